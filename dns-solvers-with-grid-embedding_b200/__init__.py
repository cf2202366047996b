"""Python host side of the B200 grid-embedded D3Q19 channel solver.

A thin ctypes layer over the C ABI of ``libdnsembed.so`` (``include/dns_embed.h``).
It mirrors the reference solver's interface for the time-step path: the
parameters of ``src/definitions.h`` (:class:`Params`, same names), the restart
files read in mode ``-p`` and written every 50 unit times, the per-step log
values of ``encalc2``/``wshearstr`` and the plane statistics of
``statistics``.  Errors raise :class:`DnsError` carrying the C status code.

The CUDA library is required: if ``libdnsembed.so`` is missing or cannot be
loaded, :func:`lib` raises instead of falling back to any CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# the in-tree build; DNS_EMBED_LIBRARY selects another build of the same
# sources (e.g. one compiled with different tuning macros)
LIBPATH = Path(os.environ["DNS_EMBED_LIBRARY"]) if os.environ.get("DNS_EMBED_LIBRARY") else HERE / "libdnsembed.so"

DNS_OK, DNS_EINVAL, DNS_ENOMEM, DNS_EIO, DNS_ENAN, DNS_ETIMEOUT, DNS_ECUDA = 0, -1, -2, -3, -4, -5, -6
PATTERN_NONE, PATTERN_RSLIP, PATTERN_PSLIP, PATTERN_SSLIP = 0, 1, 2, 3
FORCING_CFR, FORCING_CONST = 0, 1
FP64, FP32 = 0, 1
NSTAT = 14
STAT_NAMES = ("z", "U", "V", "W", "rho", "uu", "vv", "ww", "uw", "rr", "uu_t", "vv_t", "ww_t", "uw_t")
NKERNEL = 7
KERNEL_NAMES = ("coarse", "extract", "fine", "interface", "inject", "finalize", "stats")
PLANE_STAT_NAMES = ("UAVG", "VAVG", "WAVG", "UTIN", "VTIN", "WTIN", "REYS", "DAVG", "DTIN")
# profiles of dns_tke_budget, in the order of the reference's turb-fld-2d (19),
# vort-fluc-2d (3) and KE-Budget-2d (30) files
TKE_FILES = (("turb-fld-2d", 19), ("vort-fluc-2d", 3), ("KE-Budget-2d", 30))
TKE_NAMES = ("UAVG", "VAVG", "WAVG", "UTIN", "VTIN", "WTIN", "uw", "DAVG", "DTIN", "SKEWu", "SKEWv", "SKEWw",
             "SKEWuw", "SKEWp", "KURTu", "KURTv", "KURTw", "KURTuw", "KURTp", "wx", "wy", "wz", "Pii", "Puu", "Pvv",
             "Pww", "Puw", "Tiir", "Tuur", "Tvvr", "Twwr", "Tuwr", "Tiipai", "Tuupai", "Tvvpai", "Twwpai", "Tuwpai",
             "Paiuu", "Paivv", "Paiww", "Paiuw", "Tiis", "Tuus", "Tvvs", "Twws", "Tuws", "Epii", "Epuu", "Epvv",
             "Epww", "Epuw", "KE")


class DnsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class Params(C.Structure):
    """``dns_params``: the reference's definitions.h macros plus run-time options."""

    _fields_ = [
        ("Rebs", C.c_double), ("ub", C.c_double), ("zdv", C.c_int), ("ydv", C.c_int), ("xdv", C.c_int),
        ("TSTR", C.c_int), ("TEND", C.c_int), ("CFL", C.c_double), ("gratio", C.c_int), ("zds", C.c_int),
        ("gyplussize", C.c_int), ("wyplussize", C.c_int), ("gxplussize", C.c_int), ("wxplussize", C.c_int),
        ("pattern", C.c_int), ("XDIM", C.c_int), ("YDIM", C.c_int), ("ITER", C.c_long),
        ("forcing", C.c_int), ("force_const", C.c_double), ("precision", C.c_int), ("device", C.c_int),
        ("xdu", C.c_int), ("ydu", C.c_int), ("zdu", C.c_int), ("fltr", C.c_int),
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nzc", C.c_int), ("nxf", C.c_int), ("nyf", C.c_int), ("zdf", C.c_int),
        ("gr", C.c_int), ("nzs", C.c_int), ("nz_profile", C.c_int), ("utime", C.c_int),
        ("omega_c", C.c_double), ("omega_f", C.c_double), ("updates_per_step", C.c_longlong),
        ("device_bytes", C.c_longlong),
    ]


class StepLog(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("time", "force", "momentum", "denst", "flowrate", "stup", "stdown", "stress", "pgrad")]


LOG_FIELDS = tuple(n for n, _ in StepLog._fields_)


class Tile(C.Structure):
    """``dns_tile``: tile shape of one batched instance."""

    _fields_ = [("cw", C.c_int), ("cjb", C.c_int), ("fw", C.c_int), ("fjb", C.c_int)]

    def as_tuple(self):
        return (self.cw, self.cjb, self.fw, self.fjb)


class BatchInfo(C.Structure):
    _fields_ = [
        ("steps_done", C.c_longlong), ("remaining", C.c_longlong), ("status", C.c_int), ("slot", C.c_int),
        ("force", C.c_double), ("flowrate", C.c_double), ("stress", C.c_double),
        ("device_bytes", C.c_longlong), ("updates_per_step", C.c_longlong), ("tile", Tile),
    ]

_lib = None


def lib() -> C.CDLL:
    """Load ``libdnsembed.so``; raise if it is absent (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBPATH.exists():
        raise DnsError(DNS_ECUDA, f"{LIBPATH.name} is not built; run build.py")
    L = C.CDLL(str(LIBPATH))
    P, I, D = C.c_void_p, C.c_int, C.c_double
    sig = {
        "dns_params_default": (I, [C.POINTER(Params)]),
        "dns_params_from_definitions": (I, [C.c_char_p, C.POINTER(Params)]),
        "dns_geometry_of": (I, [C.POINTER(Params), C.POINTER(Geometry)]),
        "dns_create": (I, [C.POINTER(Params), C.POINTER(P)]),
        "dns_destroy": (None, [P]),
        "dns_set_stream": (I, [P, P]),
        "dns_get_geometry": (I, [P, C.POINTER(Geometry)]),
        "dns_load_restart": (I, [P, C.c_char_p, I]),
        "dns_write_restart": (I, [P, C.c_char_p, I]),
        "dns_load_uniform": (I, [P, C.c_char_p, I]),
        "dns_write_fields": (I, [P, C.c_char_p, I]),
        "dns_tke_budget": (I, [P, P, P, P]),
        "dns_tke_budget_files": (I, [C.POINTER(Params), C.c_char_p, I, P, P, P]),
        "dns_write_tke_budget": (I, [C.POINTER(Params), C.c_char_p, I, P, P, P]),
        "dns_init_seeded": (I, [P, C.c_uint64, D, D]),
        "dns_export_state": (I, [P, I, P]),
        "dns_import_state": (I, [P, I, P]),
        "dns_export_history": (I, [P, P]),
        "dns_import_history": (I, [P, P]),
        "dns_get_force": (I, [P, C.POINTER(D)]),
        "dns_step": (I, [P, C.c_long, P]),
        "dns_set_sampling": (I, [P, C.c_long]),
        "dns_stats_reset": (I, [P]),
        "dns_stats": (I, [P, P, C.POINTER(C.c_long)]),
        "dns_plane_stats": (I, [P, P]),
        "dns_set_profiling": (I, [P, I]),
        "dns_kernel_times": (I, [P, P, P]),
        "dns_batch_create": (I, [I, C.POINTER(P)]),
        "dns_batch_destroy": (None, [P]),
        "dns_batch_footprint": (I, [C.POINTER(Params), C.POINTER(C.c_longlong)]),
        "dns_batch_tile_for": (I, [P, C.POINTER(Params), C.POINTER(Tile)]),
        "dns_batch_set_tile": (I, [P, C.POINTER(Params), C.POINTER(Tile)]),
        "dns_batch_autotune": (I, [P, C.POINTER(Params), I, C.POINTER(Tile), C.POINTER(D)]),
        "dns_batch_add": (I, [P, C.POINTER(Params), C.POINTER(Tile), C.c_uint64, D, D, C.c_longlong,
                              C.c_longlong, C.POINTER(I)]),
        "dns_batch_remove": (I, [P, I]),
        "dns_batch_run": (I, [P, C.c_longlong, C.POINTER(I)]),
        "dns_batch_info_of": (I, [P, I, C.POINTER(BatchInfo)]),
        "dns_batch_stats": (I, [P, I, P, C.POINTER(C.c_long)]),
        "dns_batch_stats_reset": (I, [P, I]),
        "dns_batch_export_state": (I, [P, I, I, P]),
        "dns_batch_import_state": (I, [P, I, I, P]),
        "dns_batch_log": (I, [P, I, C.c_longlong, C.c_longlong, P]),
        "dns_batch_stream": (I, [P, C.POINTER(P)]),
        "dns_error_string": (C.c_char_p, [I]),
        "dns_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != DNS_OK:
        msg = lib().dns_last_error().decode(errors="replace")
        raise DnsError(rc, f"{what}: {msg or lib().dns_error_string(rc).decode()}")


def default_params() -> Params:
    p = Params()
    _check(lib().dns_params_default(C.byref(p)), "dns_params_default")
    return p


def params_from_definitions(path) -> Params:
    """Read a reference-style ``definitions.h``."""
    p = Params()
    _check(lib().dns_params_from_definitions(str(path).encode(), C.byref(p)), "dns_params_from_definitions")
    return p


def make_params(**kw) -> Params:
    """Defaults of the reference, overridden by keyword (macro names, e.g. xdv=64)."""
    p = default_params()
    for k, v in kw.items():
        if k == "pattern" and isinstance(v, str):
            v = {"RSLIP": PATTERN_RSLIP, "PSLIP": PATTERN_PSLIP, "SSLIP": PATTERN_SSLIP}[v]
        if k == "pattern" and v is None:
            v = PATTERN_NONE
        setattr(p, k, v)
    return p


def geometry(p: Params) -> Geometry:
    g = Geometry()
    _check(lib().dns_geometry_of(C.byref(p), C.byref(g)), "dns_geometry_of")
    return g


class Channel:
    """One grid-embedded channel resident on a GPU (a ``dns_handle``)."""

    def __init__(self, params: Params):
        self.params = params
        h = C.c_void_p()
        _check(lib().dns_create(C.byref(params), C.byref(h)), "dns_create")
        self.h = h
        self.geom = Geometry()
        _check(lib().dns_get_geometry(self.h, C.byref(self.geom)), "dns_get_geometry")

    def close(self):
        if getattr(self, "h", None):
            lib().dns_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state
    def set_stream(self, stream_handle: int | None):
        _check(lib().dns_set_stream(self.h, C.c_void_p(stream_handle or 0)), "dns_set_stream")

    def init_seeded(self, seed: int = 42, uc: float = 0.05, amp: float = 0.005):
        _check(lib().dns_init_seeded(self.h, seed, uc, amp), "dns_init_seeded")

    def load_restart(self, directory, cntr: int):
        _check(lib().dns_load_restart(self.h, str(directory).encode(), cntr), "dns_load_restart")

    def load_uniform(self, directory, cntr: int):
        """Mode -i start from the uniform-grid file lbf.cntr in directory."""
        _check(lib().dns_load_uniform(self.h, str(directory).encode(), cntr), "dns_load_uniform")

    def write_restart(self, directory, cntr: int):
        _check(lib().dns_write_restart(self.h, str(directory).encode(), cntr), "dns_write_restart")

    def write_fields(self, directory, cntr: int):
        """vel-{c,slf,suf} / den-{c,slf,suf} field files (the reference's vel_print)."""
        _check(lib().dns_write_fields(self.h, str(directory).encode(), cntr), "dns_write_fields")

    def tke_budget(self, fluct_plane: bool = False):
        """Turbulence statistics and kinetic-energy budget of the current state
        (the reference's TKE-budget/computations on the fields vel_print would
        write): (TKE_NAMES x NZ) profiles, plus the u / v fluctuations of the
        lower fine plane k = 4 when fluct_plane."""
        return _tke_call(self.params, lambda pr, u, v: lib().dns_tke_budget(self.h, pr, u, v), fluct_plane)

    def _level_shape(self, level: int):
        g = self.geom
        return (g.nx, g.ny, g.nzc, 19) if level == 0 else (g.nxf, g.nyf, g.zdf, 19)

    def export_state(self, level: int) -> np.ndarray:
        out = np.empty(self._level_shape(level), dtype=np.float64)
        _check(lib().dns_export_state(self.h, level, out.ctypes.data), "dns_export_state")
        return out

    def import_state(self, level: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self._level_shape(level):
            raise DnsError(DNS_EINVAL, f"state shape {a.shape} != {self._level_shape(level)}")
        _check(lib().dns_import_state(self.h, level, a.ctypes.data), "dns_import_state")

    def export_history(self) -> np.ndarray:
        g = self.geom
        out = np.empty((3, 2, g.nx, g.ny, 23), dtype=np.float64)
        _check(lib().dns_export_history(self.h, out.ctypes.data), "dns_export_history")
        return out

    def import_history(self, arr: np.ndarray):
        g = self.geom
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (3, 2, g.nx, g.ny, 23):
            raise DnsError(DNS_EINVAL, f"history shape {a.shape} != {(3, 2, g.nx, g.ny, 23)}")
        _check(lib().dns_import_history(self.h, a.ctypes.data), "dns_import_history")

    def force(self) -> float:
        f = C.c_double()
        _check(lib().dns_get_force(self.h, C.byref(f)), "dns_get_force")
        return f.value

    # ---- hot path
    def step(self, n: int = 1, log: bool = True) -> np.ndarray | None:
        """Advance n coarse steps; returns the per-step log (n x 9) when asked."""
        if log:
            buf = (StepLog * max(n, 1))()
            _check(lib().dns_step(self.h, n, buf), "dns_step")
            return np.frombuffer(buf, dtype=np.float64).reshape(-1, len(LOG_FIELDS))[:n].copy()
        _check(lib().dns_step(self.h, n, None), "dns_step")
        return None

    # ---- statistics
    def set_sampling(self, every: int):
        _check(lib().dns_set_sampling(self.h, every), "dns_set_sampling")

    def stats_reset(self):
        _check(lib().dns_stats_reset(self.h), "dns_stats_reset")

    def stats(self):
        nz = self.geom.nz_profile
        out = np.zeros((NSTAT, nz))
        ns = C.c_long()
        _check(lib().dns_stats(self.h, out.ctypes.data, C.byref(ns)), "dns_stats")
        return out, ns.value

    # ---- measurement
    def set_profiling(self, on: bool):
        _check(lib().dns_set_profiling(self.h, 1 if on else 0), "dns_set_profiling")

    def kernel_times(self):
        """{kernel class: (total ms, launches)} since profiling was switched on."""
        ms = np.zeros(NKERNEL)
        n = np.zeros(NKERNEL, dtype=np.int64)
        _check(lib().dns_kernel_times(self.h, ms.ctypes.data, n.ctypes.data), "dns_kernel_times")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNEL_NAMES)}

    def plane_stats(self) -> np.ndarray:
        out = np.zeros((9, self.geom.nz_profile))
        _check(lib().dns_plane_stats(self.h, out.ctypes.data), "dns_plane_stats")
        return out


def _tke_call(p: Params, fn, fluct_plane: bool):
    g = geometry(p)
    prof = np.zeros((len(TKE_NAMES), g.nz_profile))
    ufl = vfl = None
    if fluct_plane:
        ufl = np.zeros((g.nxf, g.nyf))
        vfl = np.zeros((g.nxf, g.nyf))
    ptr = lambda a: None if a is None else a.ctypes.data
    _check(fn(prof.ctypes.data, ptr(ufl), ptr(vfl)), "dns_tke_budget")
    return (prof, ufl, vfl) if fluct_plane else prof


def tke_budget_files(p: Params, directory, cntr: int, fluct_plane: bool = False):
    """The budget from vel-* / den-* files of snapshot cntr in directory."""
    d = str(directory).encode()
    return _tke_call(p, lambda pr, u, v: lib().dns_tke_budget_files(C.byref(p), d, cntr, pr, u, v), fluct_plane)


def write_tke_budget(p: Params, directory, cntr: int, prof, ufl=None, vfl=None):
    """turb-fld-2d / vort-fluc-2d / KE-Budget-2d (.000.cntr) and ufl4 / vfl4 files."""
    prof, ufl, vfl = (None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (prof, ufl, vfl))
    ptr = lambda a: None if a is None else a.ctypes.data
    _check(lib().dns_write_tke_budget(C.byref(p), str(directory).encode(), cntr, prof.ctypes.data, ptr(ufl), ptr(vfl)),
           "dns_write_tke_budget")


def batch_footprint(p: Params) -> int:
    """Device bytes one batched (FP32) instance of these parameters holds."""
    b = C.c_longlong()
    _check(lib().dns_batch_footprint(C.byref(p), C.byref(b)), "dns_batch_footprint")
    return b.value


class Batch:
    """Many independent channels stepped together in the FP32 form (a ``dns_batch``).

    ``add`` makes a seeded instance with its own step budget and returns its
    id; ``run(n)`` advances every instance with budget left by up to n coarse
    steps (captured CUDA graphs of persistent kernels over a per-instance
    block table); results stay on the device until read or removed.
    """

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().dns_batch_create(device, C.byref(h)), "dns_batch_create")
        self.h = h
        self.geoms = {}

    def close(self):
        if getattr(self, "h", None):
            lib().dns_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().dns_batch_stream(self.h, C.byref(s)), "dns_batch_stream")
        return s.value or 0

    def tile_for(self, p: Params) -> Tile:
        t = Tile()
        _check(lib().dns_batch_tile_for(self.h, C.byref(p), C.byref(t)), "dns_batch_tile_for")
        return t

    def set_tile(self, p: Params, tile):
        t = tile if isinstance(tile, Tile) else Tile(*tile)
        _check(lib().dns_batch_set_tile(self.h, C.byref(p), C.byref(t)), "dns_batch_set_tile")

    def autotune(self, p: Params, steps: int = 10):
        """Time tile shapes for this grid shape; returns (tile tuple, ms per step)."""
        t, ms = Tile(), C.c_double()
        _check(lib().dns_batch_autotune(self.h, C.byref(p), steps, C.byref(t), C.byref(ms)), "dns_batch_autotune")
        return t.as_tuple(), ms.value

    def add(self, p: Params, steps: int, seed: int = 42, uc: float = 0.05, amp: float = 0.005,
            sample_every: int = 0, tile=None) -> int:
        i = C.c_int()
        t = None if tile is None else C.byref(tile if isinstance(tile, Tile) else Tile(*tile))
        _check(lib().dns_batch_add(self.h, C.byref(p), t, seed, uc, amp, steps, sample_every, C.byref(i)),
               "dns_batch_add")
        q = Params.from_buffer_copy(p)
        q.precision = FP32
        self.geoms[i.value] = geometry(q)
        return i.value

    def remove(self, i: int):
        _check(lib().dns_batch_remove(self.h, i), "dns_batch_remove")
        self.geoms.pop(i, None)

    def run(self, n: int) -> int:
        """Advance up to n steps; returns the number of instances with budget left."""
        a = C.c_int()
        _check(lib().dns_batch_run(self.h, n, C.byref(a)), "dns_batch_run")
        return a.value

    def info(self, i: int) -> BatchInfo:
        out = BatchInfo()
        _check(lib().dns_batch_info_of(self.h, i, C.byref(out)), "dns_batch_info_of")
        return out

    def stats(self, i: int):
        nz = self.geoms[i].nz_profile
        out = np.zeros((NSTAT, nz))
        ns = C.c_long()
        _check(lib().dns_batch_stats(self.h, i, out.ctypes.data, C.byref(ns)), "dns_batch_stats")
        return out, ns.value

    def stats_reset(self, i: int):
        _check(lib().dns_batch_stats_reset(self.h, i), "dns_batch_stats_reset")

    def export_state(self, i: int, level: int) -> np.ndarray:
        g = self.geoms[i]
        shape = (g.nx, g.ny, g.nzc, 19) if level == 0 else (g.nxf, g.nyf, g.zdf, 19)
        out = np.empty(shape, dtype=np.float64)
        _check(lib().dns_batch_export_state(self.h, i, level, out.ctypes.data), "dns_batch_export_state")
        return out

    def import_state(self, i: int, level: int, arr: np.ndarray):
        g = self.geoms[i]
        shape = (g.nx, g.ny, g.nzc, 19) if level == 0 else (g.nxf, g.nyf, g.zdf, 19)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != shape:
            raise DnsError(DNS_EINVAL, f"state shape {a.shape} != {shape}")
        _check(lib().dns_batch_import_state(self.h, i, level, a.ctypes.data), "dns_batch_import_state")

    def log(self, i: int, first: int = 0, n: int | None = None) -> np.ndarray:
        if n is None:
            n = self.info(i).steps_done - first
        buf = (StepLog * max(n, 1))()
        _check(lib().dns_batch_log(self.h, i, first, n, buf), "dns_batch_log")
        return np.frombuffer(buf, dtype=np.float64).reshape(-1, len(LOG_FIELDS))[:n].copy()
