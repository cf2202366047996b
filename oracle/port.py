"""ctypes wrapper of the oracle's CPU restatement — TEST INFRASTRUCTURE ONLY.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module, and only as the checker.  ``build_port()`` compiles
``oracle/dnsport.c`` into ``oracle/libdnsport.so`` (gcc, ``-ffp-contract=off``
so no fused multiply-add changes the reference's rounding).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libdnsport.so"

PATTERNS = {None: 0, "RSLIP": 1, "PSLIP": 2, "SSLIP": 3}


class PortCfg(C.Structure):
    _fields_ = [("xdv", C.c_int), ("ydv", C.c_int), ("zdc", C.c_int), ("zds", C.c_int), ("gr", C.c_int),
                ("Reb", C.c_double), ("ub", C.c_double), ("CFL", C.c_double), ("pattern", C.c_int),
                ("gy", C.c_int), ("wy", C.c_int), ("gx", C.c_int), ("wx", C.c_int), ("fltr", C.c_int)]

    @classmethod
    def from_macros(cls, m: dict) -> "PortCfg":
        return cls(int(m["xdv"]), int(m["ydv"]), int(m["zdv"]), int(m["zds"]), int(m["gratio"]),
                   float(m["Rebs"]), float(m["ub"]), float(m["CFL"]), PATTERNS[m.get("pattern")],
                   int(m["gyplussize"]), int(m["wyplussize"]), int(m["gxplussize"]), int(m["wxplussize"]),
                   1 if m.get("fltr") else 0)


class PortLog(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("force", "momentum", "denst", "flowrate", "stup", "stdown", "stress", "pgrad")]


def build_port(force: bool = False) -> Path:
    src = [HERE / "dnsport.c", HERE / "dnsport.h"]
    if force or not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in src):
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-Wall", "-o", str(LIB),
                        str(HERE / "dnsport.c"), "-lm"], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build_port()
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        L.port_create.restype = P
        L.port_create.argtypes = [C.POINTER(PortCfg)]
        L.port_destroy.argtypes = [P]
        L.port_load_restart.argtypes = [P, C.c_char_p, C.c_int]
        L.port_save_restart.argtypes = [P, C.c_char_p, C.c_int]
        L.port_init_seeded.argtypes = [P, C.c_uint64, C.c_double, C.c_double, C.c_double]
        L.port_set_forcing.argtypes = [P, C.c_int, C.c_double]
        L.port_init_uniform.restype = C.c_int
        L.port_init_uniform.argtypes = [P, C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.port_step.argtypes = [P, C.c_long, C.POINTER(PortLog)]
        L.port_export.restype = C.c_long
        L.port_export.argtypes = [P, C.c_int, C.c_void_p]
        L.port_export_history.restype = C.c_long
        L.port_export_history.argtypes = [P, C.c_void_p]
        L.port_force.restype = C.c_double
        L.port_force.argtypes = [P]
        L.port_plane_stats.restype = C.c_int
        L.port_plane_stats.argtypes = [P, C.c_void_p]
        L.port_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.port_params.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        _lib = L
    return _lib


class Port:
    """One channel held by the CPU restatement."""

    def __init__(self, macros: dict):
        self.macros = dict(macros)
        self.cfg = PortCfg.from_macros(macros)
        self.h = lib().port_create(C.byref(self.cfg))
        gr = self.cfg.gr
        self.nx, self.ny, self.zdc = self.cfg.xdv, self.cfg.ydv, self.cfg.zdc
        self.nxf, self.nyf, self.zdf = gr * self.nx, gr * self.ny, self.cfg.zds + 1

    def close(self):
        if self.h:
            lib().port_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self):
        oc, of, nz = C.c_double(), C.c_double(), C.c_int()
        lib().port_params(self.h, C.byref(oc), C.byref(of), C.byref(nz))
        return oc.value, of.value, nz.value

    def init_seeded(self, seed=42, uc=0.05, amp=0.005, force=0.0):
        lib().port_init_seeded(self.h, seed, uc, amp, force)

    def init_uniform(self, uni: np.ndarray):
        """Mode -i start from the uniform-grid state uni[xdu, ydu, zdu + 2, 19]."""
        u = np.ascontiguousarray(uni, dtype=np.float64)
        xu, yu, zd, _ = u.shape
        if lib().port_init_uniform(self.h, u.ctypes.data, xu, yu, zd - 2) != 0:
            raise ValueError("the uniform grid does not cover the embedded grid")

    def set_forcing(self, cfr: bool, g: float = 0.0):
        lib().port_set_forcing(self.h, 1 if cfr else 0, g)

    def load(self, d, cntr):
        if lib().port_load_restart(self.h, str(d).encode(), cntr) != 0:
            raise IOError(f"cannot load restart {cntr} from {d}")

    def save(self, d, cntr):
        if lib().port_save_restart(self.h, str(d).encode(), cntr) != 0:
            raise IOError(f"cannot save restart {cntr} to {d}")

    def step(self, n: int):
        log = (PortLog * max(n, 1))()
        lib().port_step(self.h, n, log)
        return np.array([[getattr(log[i], f) for f, _ in PortLog._fields_] for i in range(n)])

    def export(self, level: int) -> np.ndarray:
        n = lib().port_export(self.h, level, None)
        out = np.empty(n, dtype=np.float64)
        lib().port_export(self.h, level, out.ctypes.data)
        if level == 0:
            return out.reshape(self.nx, self.ny, self.zdc, 19)
        return out.reshape(self.nxf, self.nyf, self.zdf, 19)

    def history(self) -> np.ndarray:
        n = lib().port_export_history(self.h, None)
        out = np.empty(n, dtype=np.float64)
        lib().port_export_history(self.h, out.ctypes.data)
        return out.reshape(3, 2, self.nx, self.ny, 23)

    def force(self) -> float:
        return lib().port_force(self.h)

    def plane_stats(self) -> np.ndarray:
        nz = 2 * self.zdf + self.zdc - 4
        out = np.zeros(9 * nz)
        lib().port_plane_stats(self.h, out.ctypes.data)
        return out.reshape(9, nz)


_EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0], dtype=np.float64)
_EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1], dtype=np.float64)
_EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], dtype=np.float64)
_W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)


def _uniform01(idx: np.ndarray, seed: int) -> np.ndarray:
    """splitmix64 of (seed, idx) mapped to [0, 1): integer arithmetic and one
    exact scaling, so the values are the same on every machine."""
    with np.errstate(over="ignore"):
        z = idx.astype(np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def uniform_state(xu: int, yu: int, zu: int, seed: int, uc: float = 0.05) -> np.ndarray:
    """A uniform-grid state [xu, yu, zu + 2, 19] for mode -i starts: density
    1 +- 0.005, laminar profile of centreline uc on the wall-normal node
    positions (k - 1/2) / zu plus +-0.005 in each velocity component, the
    equilibrium of that, plus +-5e-5 in every population.  Built from
    additions and multiplications of hashed integers only."""
    zd = zu + 2
    n = xu * yu * zd
    r = _uniform01(np.arange(n * 23, dtype=np.uint64), seed).reshape(xu, yu, zd, 23)
    zeta = (np.arange(zd, dtype=np.float64) - 0.5) / zu
    rho = 1.0 + 0.01 * (r[..., 0] - 0.5)
    u0 = (4.0 * uc) * zeta * (1.0 - zeta) + 0.01 * (r[..., 1] - 0.5)
    u1 = 0.01 * (r[..., 2] - 0.5)
    u2 = 0.01 * (r[..., 3] - 0.5)
    v = u0 * u0 + u1 * u1 + u2 * u2
    f = np.empty((xu, yu, zd, 19))
    for a in range(19):
        eu = _EX[a] * u0 + _EY[a] * u1 + _EZ[a] * u2
        f[..., a] = _W[a] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * v) + 1e-4 * (r[..., 4 + a] - 0.5)
    return f


def write_uniform_file(path, first: np.ndarray, second: np.ndarray) -> None:
    """lbf.TTTT of a uniform-grid run: [ftemp | f] in C order, native doubles."""
    np.concatenate([first.reshape(-1), second.reshape(-1)]).astype(np.float64).tofile(path)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().port_philox4x32_10(c, k, o)
    return tuple(o)
