"""ctypes wrapper of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs, as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "general-simulator_b200"))
import gs_b200 as gb  # noqa: E402  (struct layouts shared with the C ABI)

LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import subprocess
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB)
        P, S = C.POINTER(gb.GsParams), C.POINTER(gb.GsStats)
        dp = C.POINTER(C.c_double)
        L.or_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.or_normals4.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, dp]
        L.or_fft3.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_bmat_at.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.or_mart_run.argtypes = [P, dp, dp, dp, C.c_int, C.c_int64]
        L.or_mart_stats.argtypes = [P, dp, dp, dp, S]
        L.or_mart_potential.argtypes = [P, dp, dp]
        L.or_precip_run.argtypes = [P, dp, dp, C.c_int, C.c_int64]
        L.or_precip_stats.argtypes = [P, dp, dp, S]
        L.or_stress.argtypes = [P, dp, dp, dp]
        L.or_mart_adjoint.argtypes = [P, dp, C.c_int, dp, C.c_double, C.c_double, dp, C.c_double, dp, dp, dp]
        ip = C.POINTER(C.c_int)
        fp = C.POINTER(C.c_float)
        L.or_cores_paint.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, C.c_double, C.c_double,
                                     C.c_double, fp, fp]
        L.or_cores_marked.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, C.c_double, C.c_int, C.c_int, C.c_int]
        L.or_precip_adjoint.argtypes = [P, dp, dp, C.c_int, dp, dp, dp, dp, dp]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().or_philox4x32_10(c, k, o)
    return [o[i] for i in range(4)]


def normals4(seed, cell, step, sim, block):
    z = np.zeros(4)
    lib().or_normals4(seed, cell, step, sim, block, _dp(z))
    return z


def fft3(a: np.ndarray, sign: int) -> np.ndarray:
    b = np.ascontiguousarray(a, dtype=np.complex128).copy()
    n0, n1, n2 = b.shape
    lib().or_fft3(b.ctypes.data_as(C.POINTER(C.c_double)), n0, n1, n2, sign)
    return b


def bmat(p: gb.GsParams, which: int, m) -> np.ndarray:
    B = np.zeros(100)
    na, nb = C.c_int(), C.c_int()
    lib().or_bmat_at(C.byref(p), which, int(m[0]), int(m[1]), int(m[2]), _dp(B), C.byref(na), C.byref(nb))
    return B[: na.value * nb.value].reshape(na.value, nb.value)


def mart_run(p, eta, nsteps, step0=0, defect=None, dstress=None) -> np.ndarray:
    e = _f64(eta).copy()
    d = None if defect is None else _f64(defect)
    s = None if dstress is None else _f64(dstress)
    lib().or_mart_run(C.byref(p), _dp(e), _dp(d), _dp(s), nsteps, step0)
    return e


def mart_stats(p, eta, defect=None, dstress=None) -> dict:
    st = gb.GsStats()
    e = _f64(eta)
    d = None if defect is None else _f64(defect)
    s = None if dstress is None else _f64(dstress)
    lib().or_mart_stats(C.byref(p), _dp(e), _dp(d), _dp(s), C.byref(st))
    return st.as_dict(p.nvariants)


def mart_potential(p, eta) -> np.ndarray:
    e = _f64(eta)
    R = np.zeros_like(e)
    lib().or_mart_potential(C.byref(p), _dp(e), _dp(R))
    return R


def precip_run(p, c, eta, nsteps, step0=0):
    cc = _f64(c).copy()
    e = _f64(eta).copy()
    lib().or_precip_run(C.byref(p), _dp(cc), _dp(e), nsteps, step0)
    return cc, e


def precip_stats(p, c, eta) -> dict:
    st = gb.GsStats()
    lib().or_precip_stats(C.byref(p), _dp(_f64(c)), _dp(_f64(eta)), C.byref(st))
    return st.as_dict(p.nvariants)


def stress(p, eta):
    e = _f64(eta)
    n = p.nx * p.ny * p.nz
    s = np.zeros((6, n))
    d = np.zeros(n)
    lib().or_stress(C.byref(p), _dp(e), _dp(s), _dp(d))
    return s.reshape(6, p.nx, p.ny, p.nz), d.reshape(p.nx, p.ny, p.nz)


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def get_threads() -> int:
    return lib().or_get_threads()


def mart_adjoint(p, eta0, nsteps, target=None, lam_el=0.0, e_target=0.0, seed=None, seed_e=0.0):
    """(loss, field term, E_el(T)), grads[6], dJ/deta0 of the baseline martensite run."""
    e = _f64(eta0)
    g = np.zeros(6)
    ge = np.zeros_like(e)
    lo = np.zeros(3)
    t = None if target is None else _f64(target)
    sd = None if seed is None else _f64(seed)
    lib().or_mart_adjoint(C.byref(p), _dp(e), nsteps, _dp(t), lam_el, e_target, _dp(sd), seed_e, _dp(g), _dp(ge), _dp(lo))
    return lo, g, ge


def mart_loss(p, eta0, nsteps, target, lam_el, e_target):
    eT = mart_run(p, eta0, nsteps)
    st = mart_stats(p, eT)
    return ((eT - target) ** 2).sum() + lam_el * (st["e_el"] - e_target) ** 2


def cores_paint(shape, V, centers, variants, radius, c_matrix, c_core):
    """(eta [V][nx][ny][nz], concentration [nx][ny][nz]) as float32."""
    nx, ny, nz = shape
    n = len(variants)
    cen = np.ascontiguousarray(np.asarray(centers, dtype=np.int32).reshape(n * 3) if n else np.zeros(3, np.int32))
    var = np.ascontiguousarray(np.asarray(variants, dtype=np.int32) if n else np.zeros(1, np.int32))
    eta = np.zeros((V, nx, ny, nz), dtype=np.float32)
    conc = np.zeros((nx, ny, nz), dtype=np.float32)
    ip = C.POINTER(C.c_int)
    fp = C.POINTER(C.c_float)
    lib().or_cores_paint(nx, ny, nz, V, n, cen.ctypes.data_as(ip), var.ctypes.data_as(ip), radius, c_matrix, c_core,
                         eta.ctypes.data_as(fp), conc.ctypes.data_as(fp))
    return eta, conc


def cores_place(shape, V, ncores, radius, method, rand):
    """Nucleus centres and variants in the order the reference draws them;
    rand() returns the next value of the C library's random()."""
    nx, ny, nz = shape
    centers, variants = [], []
    ip = C.POINTER(C.c_int)
    if method == "random":
        for _ in range(ncores):
            cen = np.ascontiguousarray(np.asarray(centers, dtype=np.int32).reshape(-1) if centers else np.zeros(3, np.int32))
            for _ in range(100000):
                o = (rand() % nx, rand() % ny, rand() % nz)
                if not lib().or_cores_marked(nx, ny, nz, len(centers), cen.ctypes.data_as(ip), radius, *o):
                    break
            centers.append(o)
            variants.append(rand() % V)
    elif method == "regular":
        for cn in range(ncores):
            rand()
            centers.append((nx // 2, ny // 2, nz // ncores // 2 + nx // ncores * cn))
            variants.append(cn % V)
    return centers, variants


def precip_adjoint(p, c0, eta0, nsteps, seed_c, seed_eta):
    """grads[9] (kappa_c, kappa_eta, coef[1..7]), dJ/dc0, dJ/deta0 of
    J = <seed_c, c_T> + <seed_eta, eta_T> (baseline precipitate run)."""
    c = _f64(c0)
    e = _f64(eta0)
    gc = np.zeros_like(c)
    ge = np.zeros_like(e)
    g = np.zeros(9)
    lib().or_precip_adjoint(C.byref(p), _dp(c), _dp(e), nsteps, _dp(_f64(seed_c)), _dp(_f64(seed_eta)), _dp(gc),
                            _dp(ge), _dp(g))
    return g, gc, ge
