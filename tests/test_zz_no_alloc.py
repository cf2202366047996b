"""The allocation-free reduction entry point (dns_flow_sums_static).

It serves callers that cannot allocate device memory (a CUDA graph being
captured, a fixed device-memory budget, a pool allocator): the caller passes
the state and the output in device memory and the library uses a scratch array
compiled into it.  Its result must agree with the regular entry points, which
compute the same sums with allocated scratch: the force from dns_get_force and
the momentum and mass logged for the first step.  Two calls in a row must give
the same result, since the shared scratch keeps the previous call's contents.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]


def device_state(ch):
    """The channel's post-stream state in the library's device layout."""
    import torch

    g = ch.geom
    zds = ch.params.zds
    coarse = np.ascontiguousarray(ch.export_state(0).transpose(3, 2, 1, 0))  # [19][k][j][i]
    lo, up = ch.export_state(1), ch.export_state(2)  # (i, j, k, a)
    fine = np.concatenate([lo[:, :, 1:g.zdf, :], up[:, :, 0:zds, :]], axis=2)
    fine = np.ascontiguousarray(fine.transpose(3, 2, 1, 0))  # [19][p][j][i]
    return torch.from_numpy(coarse).cuda(), torch.from_numpy(fine).cuda()


@pytest.mark.parametrize("name,on_stream", [("t_odd", False), ("c1", False), ("c1", True)])
def test_static_reduction_matches_allocating_path(pkg, ref_configs, name, on_stream):
    import torch

    m = ref_configs[name]
    p = pkg.make_params(xdv=m["xdv"], ydv=m["ydv"], zdv=m["zdv"], zds=m["zds"], gratio=m["gratio"],
                        Rebs=float(m["Rebs"]), ub=m["ub"], CFL=m["CFL"], pattern=m.get("pattern"),
                        gyplussize=m["gyplussize"], wyplussize=m["wyplussize"], forcing=pkg.FORCING_CFR)
    ch = pkg.Channel(p)
    ch.init_seeded(11, 0.05, 0.005)
    fc, ff = device_state(ch)
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    fn = pkg.lib().dns_flow_sums_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(pkg.Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    # on_stream: the call is ordered on a caller's stream, which is then the
    # only thing synchronised before the result is read
    stream = torch.cuda.Stream() if on_stream else None
    results = []
    for _ in range(2):
        if stream is not None:
            out.fill_(float("nan"))
            torch.cuda.synchronize()
        rc = fn(C.byref(p), fc.data_ptr(), ff.data_ptr(), out.data_ptr(),
                stream.cuda_stream if stream is not None else None)
        assert rc == 0, pkg.lib().dns_last_error()
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.synchronize()
        results.append(out.cpu().numpy().copy())
    np.testing.assert_array_equal(results[0][:3], results[1][:3])
    force = ch.force()
    log = ch.step(1)
    expected = np.array([force, log[0, 2], log[0, 3]])  # force, momentum, mass of the seeded state
    np.testing.assert_allclose(results[0][:3], expected, rtol=1e-13, atol=1e-18)


def test_static_reduction_accepts_a_domain_that_fills_the_scratch(pkg):
    """64 x 4096 coarse columns, zdv 48, zds 8: exactly 262144 reduction
    blocks (the array's size).  A zero state has zero momentum and mass, so
    the constant-flow-rate force is ub."""
    import torch

    p = pkg.make_params(xdv=64, ydv=4096, zdv=48, zds=8, gratio=2, forcing=pkg.FORCING_CFR)
    g = pkg.geometry(p)
    fc = torch.zeros(19 * g.nzc * g.ny * g.nx, dtype=torch.float64, device="cuda")
    ff = torch.zeros(19 * 2 * p.zds * g.nyf * g.nxf, dtype=torch.float64, device="cuda")
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    fn = pkg.lib().dns_flow_sums_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(pkg.Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = fn(C.byref(p), fc.data_ptr(), ff.data_ptr(), out.data_ptr(), None)
    assert rc == 0, pkg.lib().dns_last_error()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy()[:3], [p.ub, 0.0, 0.0])
    del fc, ff
    torch.cuda.empty_cache()


def test_static_reduction_rejects_oversized_domains(pkg):
    p = pkg.make_params(xdv=1024, ydv=1024, zdv=200, zds=16, gratio=2)
    fn = pkg.lib().dns_flow_sums_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(pkg.Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    dummy = C.c_double()
    rc = fn(C.byref(p), C.addressof(dummy), C.addressof(dummy), C.addressof(dummy), None)
    assert rc == pkg.DNS_EINVAL
    assert b"static scratch" in pkg.lib().dns_last_error()
