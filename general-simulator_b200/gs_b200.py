"""ctypes binding of the B200-native phase-field step (include/gs_capi.h).

The C ABI is the product boundary; this module only mirrors its POD structs
and wraps the handles for Python callers (tests, bench.py, the calibration
harness).  Loading fails loudly when libgsb200.so is missing: there is no
Python or CPU fallback for the step.

The reference drives the same work through GS_NS::Dynamics
(src/dynamics.h:9-25); `Sim` mirrors that lifecycle: create = Initialize,
step = Calculate, stats = Get.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# GS_BOUNDS_CHECK=1 loads the bounds-check build (index asserts in the kernels,
# GS_EBOUNDS from the step entries, the launch-range check on)
BOUNDS_CHECK_BUILD = os.environ.get("GS_BOUNDS_CHECK", "0") not in ("", "0")
LIB_PATH = os.path.join(HERE, "libgsb200_bc.so" if BOUNDS_CHECK_BUILD else "libgsb200.so")

GS_OK = 0
GS_EINVAL = -10
GS_ENOTSUP = -14
GS_EBOUNDS = -16
GS_MODEL_MART, GS_MODEL_PRECIPITATE, GS_MODEL_STRESS = 1, 2, 3
GS_MODE_BASELINE, GS_MODE_REFCOMPAT = 0, 1
GS_DTYPE_F32, GS_DTYPE_F64 = 0, 1
GS_MAX_V = 8


class GsSchedule(C.Structure):
    _fields_ = [("z_lines", C.c_int), ("y_cols", C.c_int), ("x_cols", C.c_int), ("update_rows", C.c_int),
                ("y_radix", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GsParams(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("mode", C.c_int), ("dtype", C.c_int), ("nvariants", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("eigenstrain", C.c_double * 9 * GS_MAX_V),
        ("cijkl", C.c_double * 81),
        ("applied_stress", C.c_double * 9),
        ("weight_elastic", C.c_double),
        ("landau", C.c_double * 4), ("kappa", C.c_double), ("mobility", C.c_double),
        ("weight_gradient", C.c_double), ("weight_chemical", C.c_double),
        ("weight_dislocation", C.c_double), ("lpc", C.c_double * 4),
        ("transition_temperature", C.c_double), ("temperature", C.c_double),
        ("noise_amp", C.c_double), ("seed", C.c_uint64), ("sim_id", C.c_uint32), ("pad0", C.c_uint32),
        ("coef", C.c_double * 8), ("c1", C.c_double), ("c2", C.c_double),
        ("kappa_c", C.c_double), ("kappa_eta", C.c_double),
        ("mobility_c", C.c_double), ("mobility_eta", C.c_double),
        ("xi", C.c_double), ("misfit_c", C.c_double),
        ("c_elastic", C.c_int), ("mass_projection", C.c_int),
    ]

    # numpy views of the array members
    def set_eigenstrain(self, eps: np.ndarray) -> None:
        eps = np.asarray(eps, dtype=np.float64).reshape(-1, 3, 3)
        flat = np.zeros((GS_MAX_V, 9))
        flat[: eps.shape[0]] = eps.reshape(-1, 9)
        for v in range(GS_MAX_V):
            for i in range(9):
                self.eigenstrain[v][i] = flat[v, i]

    def get_eigenstrain(self) -> np.ndarray:
        return np.array([[self.eigenstrain[v][i] for i in range(9)] for v in range(self.nvariants)]).reshape(-1, 3, 3)

    def set_cijkl(self, c: np.ndarray) -> None:
        c = np.asarray(c, dtype=np.float64).reshape(81)
        for i in range(81):
            self.cijkl[i] = c[i]

    def get_cijkl(self) -> np.ndarray:
        return np.array([self.cijkl[i] for i in range(81)]).reshape(3, 3, 3, 3)

    def set_applied_stress(self, s: np.ndarray) -> None:
        s = np.asarray(s, dtype=np.float64).reshape(9)
        for i in range(9):
            self.applied_stress[i] = s[i]

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    def copy(self) -> "GsParams":
        q = GsParams()
        C.memmove(C.byref(q), C.byref(self), C.sizeof(GsParams))
        return q


class GsStats(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("eta_mean", C.c_double),
        ("eta2", C.c_double * GS_MAX_V), ("vf", C.c_double * GS_MAX_V),
        ("e_el", C.c_double), ("e_chem", C.c_double), ("e_grad", C.c_double),
        ("e_appl", C.c_double), ("e_tot", C.c_double),
        ("gradient_mean", C.c_double), ("chemical_mean", C.c_double),
        ("elastic_mean", C.c_double), ("dislocation_mean", C.c_double),
        ("c_mean", C.c_double), ("step", C.c_int64),
    ]

    def as_dict(self, nv: int) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("eta2", "vf")}
        d["eta2"] = [self.eta2[i] for i in range(nv)]
        d["vf"] = [self.vf[i] for i in range(nv)]
        return d


class GsSlabGeometry(C.Structure):
    _fields_ = [("rank", C.c_int), ("nranks", C.c_int), ("x0", C.c_int), ("nx_local", C.c_int),
                ("kz0", C.c_int), ("nkz_local", C.c_int), ("a2a_bytes", C.c_size_t), ("halo_bytes", C.c_size_t),
                ("step", C.c_int64)]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load libgsb200.so (libgsb200_bc.so under GS_BOUNDS_CHECK=1; built
    in-tree by build.py); raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{os.path.basename(LIB_PATH)} not built at {LIB_PATH}; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    P, S = C.POINTER(GsParams), C.POINTER(GsStats)
    vp = C.c_void_p
    sig = {
        "gs_version": (C.c_int, []),
        "gs_sizeof_params": (C.c_size_t, []),
        "gs_sizeof_stats": (C.c_size_t, []),
        "gs_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
        "gs_params_default": (C.c_int, [P, C.c_int, C.c_int]),
        "gs_sim_create": (C.c_int, [P, C.POINTER(vp)]),
        "gs_sim_destroy": (C.c_int, [vp]),
        "gs_sim_set_field": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_sim_get_field": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_sim_set_scalar": (C.c_int, [vp, C.c_char_p, C.c_double]),
        "gs_sim_step": (C.c_int, [vp, C.c_int, vp]),
        "gs_sim_stats": (C.c_int, [vp, S, vp]),
        "gs_sim_device_field": (C.c_int, [vp, C.c_char_p, C.POINTER(vp), C.POINTER(C.c_size_t)]),
        "gs_sim_launch_count": (C.c_int64, [vp]),
        "gs_sim_profile_step": (C.c_int, [vp, vp, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int)]),
        "gs_sim_use_graph": (C.c_int, [vp, C.c_int]),
        "gs_set_device": (C.c_int, [C.c_int]),
        "gs_batch_create": (C.c_int, [P, C.c_int, C.POINTER(vp)]),
        "gs_batch_destroy": (C.c_int, [vp]),
        "gs_batch_set_field": (C.c_int, [vp, C.c_int, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_batch_get_field": (C.c_int, [vp, C.c_int, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_batch_step": (C.c_int, [vp, C.c_int, vp]),
        "gs_batch_stats": (C.c_int, [vp, C.c_int, S, vp]),
        "gs_batch_use_graph": (C.c_int, [vp, C.c_int]),
        "gs_batch_groups": (C.c_int, [vp]),
        "gs_batch_set_concurrent": (C.c_int, [vp, C.c_int]),
        "gs_batch_launch_count": (C.c_int64, [vp]),
        "gs_plain_create": (C.c_int, [P, C.POINTER(vp)]),
        "gs_plain_step": (C.c_int, [vp, C.c_int, vp]),
        "gs_sim_pass_name": (C.c_char_p, [vp, C.c_int]),
        "gs_sim_stage_field_async": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_cufft_create": (C.c_int, [P, C.POINTER(vp)]),
        "gs_cufft_step": (C.c_int, [vp, C.c_int, vp]),
        "gs_adjoint_create": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(vp)]),
        "gs_adjoint_destroy": (C.c_int, [vp]),
        "gs_adjoint_set_params": (C.c_int, [vp, P]),
        "gs_adjoint_set_loss": (C.c_int, [vp, vp, C.c_int, C.c_double, C.c_double]),
        "gs_adjoint_forward": (C.c_int, [vp, vp, C.c_int, vp, C.POINTER(C.c_double), vp]),
        "gs_adjoint_backward": (C.c_int, [vp, vp, C.c_int, C.c_double, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), vp, C.c_int, vp]),
        "gs_adjoint_device_bytes": (C.c_size_t, [vp]),
        "gs_adjoint_use_graph": (C.c_int, [vp, C.c_int]),
        "gs_adjoint_launch_count": (C.c_int64, [vp]),
        "gs_precip_adjoint_create": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(vp)]),
        "gs_precip_adjoint_use_graph": (C.c_int, [vp, C.c_int]),
        "gs_precip_adjoint_destroy": (C.c_int, [vp]),
        "gs_precip_adjoint_forward": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, vp]),
        "gs_precip_adjoint_backward": (C.c_int, [vp, vp, vp, C.c_int, C.POINTER(C.c_double), vp, vp, vp]),
        "gs_precip_adjoint_device_bytes": (C.c_size_t, [vp]),
        "gs_precip_adjoint_set_seed": (C.c_int, [vp, vp, vp, C.c_int]),
        "gs_set_x_prefetch": (None, [C.c_int]),
        "gs_sim_copy_field_async": (C.c_int, [vp, C.c_char_p, vp, vp, C.POINTER(C.c_int)]),
        "gs_sim_copy_field_wait": (C.c_int, [vp, C.c_int, vp, C.c_size_t, C.c_int]),
        "gs_sim_set_field_async": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int, vp]),
        "gs_x_prefetch_timeouts": (C.c_uint, []),
        "gs_sim_set_schedule": (C.c_int, [vp, C.POINTER(GsSchedule)]),
        "gs_sim_get_schedule": (C.c_int, [vp, C.POINTER(GsSchedule)]),
        "gs_sim_autotune": (C.c_int, [vp, C.c_int, vp, C.POINTER(GsSchedule)]),
        "gs_batch_autotune": (C.c_int, [vp, C.c_int, vp]),
        "gs_batch_get_schedule": (C.c_int, [vp, C.c_int, C.POINTER(GsSchedule)]),
        "gs_sim_take_field": (C.c_int, [vp, C.c_char_p, vp, C.c_char_p]),
        "gs_cores_paint": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, C.c_double, C.c_double,
                                     C.c_double, vp, vp]),
        "gs_slab_create": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(vp)]),
        "gs_slab_destroy": (C.c_int, [vp]),
        "gs_slab_info": (C.c_int, [vp, C.POINTER(GsSlabGeometry)]),
        "gs_slab_set_field": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_slab_get_field": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.c_int]),
        "gs_slab_set_step": (C.c_int, [vp, C.c_int64]),
        "gs_slab_begin": (C.c_int, [vp, vp, vp, vp]),
        "gs_slab_xpass": (C.c_int, [vp, vp, vp, vp]),
        "gs_slab_end": (C.c_int, [vp, vp, vp, vp]),
        "gs_noise_block": (C.c_int, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                     vp, vp]),
        "gs_mart_step_noalloc": (C.c_int, [P, vp, vp, C.c_int64, vp]),
        "gs_mart_step_noalloc_max_bytes": (C.c_size_t, []),
        "gs_set_bounds_check": (None, [C.c_int]),
        "gs_bounds_check_enabled": (C.c_int, []),
        "gs_bounds_check_build": (C.c_int, []),
        "gs_bounds_check_read": (C.c_int, [C.POINTER(C.c_longlong), C.c_int]),
        "gs_bounds_site_name": (C.c_char_p, [C.c_int]),
        "gs_bounds_selftest": (C.c_int, [vp, C.c_int, C.c_int, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().gs_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


class GsError(RuntimeError):
    pass


def check(rc: int, what: str) -> None:
    if rc != GS_OK:
        raise GsError(f"{what} failed with status {rc}: {last_error()}")


def set_bounds_check(on: bool) -> None:
    """The launch-range check (every build): each pass launcher checks that
    its buffers' ranges lie inside their allocations before it launches."""
    lib().gs_set_bounds_check(1 if on else 0)


def bounds_record(clear: bool = False) -> dict:
    """The bounds-check build's index-assert record of the current device
    (synchronises it): violations, the first one's site, index, extent,
    block and thread.  GsError in a normal build."""
    out = (C.c_longlong * 6)()
    check(lib().gs_bounds_check_read(out, 1 if clear else 0), "gs_bounds_check_read")
    site = int(out[1])
    return {"violations": int(out[0]), "site": site, "site_name": lib().gs_bounds_site_name(site).decode(),
            "index": int(out[2]), "extent": int(out[3]), "block": int(out[4]), "thread": int(out[5])}


def default_params(model: int, mode: int = GS_MODE_BASELINE) -> GsParams:
    p = GsParams()
    check(lib().gs_params_default(C.byref(p), model, mode), "gs_params_default")
    return p


def _np_dtype(code: int):
    return np.float64 if code == GS_DTYPE_F64 else np.float32


class Adjoint:
    """Checkpointed adjoint of a martensite run (gs_adjoint*): forward() runs
    eta0 -> eta_T keeping a checkpoint every `checkpoint_every` steps;
    backward() returns (loss[3], grads[6], dJ/deta0) with grads over
    (kappa, A2, A4, A6, Ac, eigenstrain scale s)."""

    PARAM_NAMES = ("kappa", "A2", "A4", "A6", "Ac", "s")

    def __init__(self, params: GsParams, nsteps: int, checkpoint_every: int):
        self.params = params.copy()
        self.nsteps = nsteps
        h = C.c_void_p()
        check(lib().gs_adjoint_create(C.byref(self.params), nsteps, checkpoint_every, C.byref(h)), "gs_adjoint_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().gs_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        p = self.params
        return (p.nvariants, p.nx, p.ny, p.nz)

    def set_params(self, params: GsParams) -> None:
        self.params = params.copy()
        check(lib().gs_adjoint_set_params(self.h, C.byref(self.params)), "gs_adjoint_set_params")

    def set_loss(self, target: np.ndarray, lam_el: float, e_target: float) -> None:
        t = np.ascontiguousarray(target, dtype=np.float64)
        check(lib().gs_adjoint_set_loss(self.h, t.ctypes.data, GS_DTYPE_F64, lam_el, e_target), "gs_adjoint_set_loss")

    def forward(self, eta0: np.ndarray, stream: int = 0):
        e = np.ascontiguousarray(eta0, dtype=np.float64)
        out = np.empty(self.shape, dtype=np.float64)
        eel = C.c_double()
        check(lib().gs_adjoint_forward(self.h, e.ctypes.data, GS_DTYPE_F64, out.ctypes.data, C.byref(eel),
                                       C.c_void_p(stream)), "gs_adjoint_forward")
        return out, eel.value

    def backward(self, seed: Optional[np.ndarray] = None, seed_e: float = 0.0, stream: int = 0):
        loss = (C.c_double * 3)()
        g = (C.c_double * 6)()
        ge = np.empty(self.shape, dtype=np.float64)
        sd = None
        if seed is not None:
            sd = np.ascontiguousarray(seed, dtype=np.float64)
        check(lib().gs_adjoint_backward(self.h, None if sd is None else sd.ctypes.data, GS_DTYPE_F64, seed_e, loss, g,
                                        ge.ctypes.data, GS_DTYPE_F64, C.c_void_p(stream)), "gs_adjoint_backward")
        return np.array(loss[:]), np.array(g[:]), ge

    def device_bytes(self) -> int:
        return int(lib().gs_adjoint_device_bytes(self.h))

    def use_graph(self, on: bool) -> None:
        check(lib().gs_adjoint_use_graph(self.h, int(bool(on))), "gs_adjoint_use_graph")

    def launch_count(self) -> int:
        return int(lib().gs_adjoint_launch_count(self.h))


class PrecipAdjoint:
    """Adjoint of a precipitate run (gs_precip_adjoint*): forward() runs
    (c0, eta0) -> (c_T, eta_T) keeping a checkpoint every `checkpoint_every`
    steps; backward(seed_c, seed_eta) recomputes each segment and returns
    (grads[9], dJ/dc0, dJ/deta0) for J = <seed_c, c_T> + <seed_eta, eta_T>,
    grads over (kappa_c, kappa_eta, coef[1..7])."""

    PARAM_NAMES = ("kappa_c", "kappa_eta", "A1", "A2", "A3", "A4", "A5", "A6", "A7")

    def __init__(self, params: GsParams, nsteps: int, checkpoint_every: int = 1):
        self.params = params.copy()
        self.nsteps = nsteps
        h = C.c_void_p()
        check(lib().gs_precip_adjoint_create(C.byref(self.params), nsteps, checkpoint_every, C.byref(h)),
              "gs_precip_adjoint_create")
        self.h = h

    def use_graph(self, on: bool) -> None:
        check(lib().gs_precip_adjoint_use_graph(self.h, 1 if on else 0), "gs_precip_adjoint_use_graph")

    def close(self) -> None:
        if self.h:
            lib().gs_precip_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        p = self.params
        return (p.nx, p.ny, p.nz)

    def forward(self, c0: Optional[np.ndarray] = None, eta0: Optional[np.ndarray] = None, stream: int = 0,
                outputs: bool = True):
        """c0 = eta0 = None: again from the previous initial state (device);
        outputs=False: keep (c_T, eta_T) on the device and return None."""
        c = e = None
        if c0 is not None:
            c = np.ascontiguousarray(c0, dtype=np.float64)
            e = np.ascontiguousarray(eta0, dtype=np.float64)
        co = eo = None
        if outputs:
            co = np.empty(self.shape, dtype=np.float64)
            eo = np.empty((self.params.nvariants,) + self.shape, dtype=np.float64)
        check(lib().gs_precip_adjoint_forward(self.h, None if c is None else c.ctypes.data,
                                              None if e is None else e.ctypes.data, GS_DTYPE_F64,
                                              None if co is None else co.ctypes.data,
                                              None if eo is None else eo.ctypes.data, C.c_void_p(stream)),
              "gs_precip_adjoint_forward")
        return (co, eo) if outputs else None

    def set_seed(self, seed_c: np.ndarray, seed_eta: np.ndarray) -> None:
        sc = np.ascontiguousarray(seed_c, dtype=np.float64)
        se = np.ascontiguousarray(seed_eta, dtype=np.float64)
        check(lib().gs_precip_adjoint_set_seed(self.h, sc.ctypes.data, se.ctypes.data, GS_DTYPE_F64),
              "gs_precip_adjoint_set_seed")

    def backward(self, seed_c: Optional[np.ndarray] = None, seed_eta: Optional[np.ndarray] = None, stream: int = 0,
                 outputs: bool = True):
        """Seeds None: the last ones given.  Returns (grads[9], dJ/dc0,
        dJ/deta0); the fields are None with outputs=False."""
        if seed_c is not None:
            self.set_seed(seed_c, seed_eta)
        g = (C.c_double * 9)()
        gc = ge = None
        if outputs:
            gc = np.empty(self.shape, dtype=np.float64)
            ge = np.empty((self.params.nvariants,) + self.shape, dtype=np.float64)
        check(lib().gs_precip_adjoint_backward(self.h, None, None, GS_DTYPE_F64, g,
                                               None if gc is None else gc.ctypes.data,
                                               None if ge is None else ge.ctypes.data, C.c_void_p(stream)),
              "gs_precip_adjoint_backward")
        return np.array(g[:]), gc, ge

    def device_bytes(self) -> int:
        return int(lib().gs_precip_adjoint_device_bytes(self.h))


class Sim:
    """One simulation handle (gs_sim*).  `plain=True` builds the comparator
    in the reference's structure (cuFFT C2C, B streamed, unfused sweeps);
    `cufft=True` the cuFFT R2C/C2R comparator with this project's contraction
    and fused update; neither is the product step."""

    def __init__(self, params: GsParams, plain: bool = False, cufft: bool = False):
        self.params = params.copy()
        h = C.c_void_p()
        if plain:
            check(lib().gs_plain_create(C.byref(self.params), C.byref(h)), "gs_plain_create")
        elif cufft:
            check(lib().gs_cufft_create(C.byref(self.params), C.byref(h)), "gs_cufft_create")
        else:
            check(lib().gs_sim_create(C.byref(self.params), C.byref(h)), "gs_sim_create")
        self.h = h
        self.plain = plain
        self.cufft = cufft

    def close(self) -> None:
        if self.h:
            lib().gs_sim_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr)
        code = GS_DTYPE_F64 if a.dtype == np.float64 else GS_DTYPE_F32
        a = np.ascontiguousarray(a, dtype=_np_dtype(code))
        check(lib().gs_sim_set_field(self.h, name.encode(), a.ctypes.data, a.size, code), f"set_field({name})")

    def get_field(self, name: str, count: int, dtype=np.float64) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        code = GS_DTYPE_F64 if dtype == np.float64 else GS_DTYPE_F32
        check(lib().gs_sim_get_field(self.h, name.encode(), out.ctypes.data, count, code), f"get_field({name})")
        return out

    def eta(self, dtype=np.float64) -> np.ndarray:
        p = self.params
        return self.get_field("eta", p.nvariants * p.ncells, dtype).reshape(p.nvariants, p.nx, p.ny, p.nz)

    def concentration(self, dtype=np.float64) -> np.ndarray:
        p = self.params
        return self.get_field("concentration", p.ncells, dtype).reshape(p.nx, p.ny, p.nz)

    def set_scalar(self, name: str, value: float) -> None:
        check(lib().gs_sim_set_scalar(self.h, name.encode(), float(value)), f"set_scalar({name})")

    def step(self, n: int = 1, stream: int = 0) -> None:
        if self.plain:
            check(lib().gs_plain_step(self.h, n, C.c_void_p(stream)), "gs_plain_step")
        elif self.cufft:
            check(lib().gs_cufft_step(self.h, n, C.c_void_p(stream)), "gs_cufft_step")
        else:
            check(lib().gs_sim_step(self.h, n, C.c_void_p(stream)), "gs_sim_step")

    def stats(self, stream: int = 0) -> dict:
        s = GsStats()
        check(lib().gs_sim_stats(self.h, C.byref(s), C.c_void_p(stream)), "gs_sim_stats")
        return s.as_dict(self.params.nvariants)

    def device_field(self, name: str):
        ptr = C.c_void_p()
        nb = C.c_size_t()
        check(lib().gs_sim_device_field(self.h, name.encode(), C.byref(ptr), C.byref(nb)), "device_field")
        return ptr.value, nb.value

    def profile_step(self, stream: int = 0) -> list:
        buf = (C.c_double * 32)()
        n = C.c_int()
        check(lib().gs_sim_profile_step(self.h, C.c_void_p(stream), buf, 32, C.byref(n)), "profile_step")
        return [buf[i] for i in range(n.value)]

    def pass_names(self) -> list:
        """Names of the passes of the last profile_step, in launch order."""
        out = []
        while True:
            nm = lib().gs_sim_pass_name(self.h, len(out))
            if nm is None:
                return out
            out.append(nm.decode())

    def launch_count(self) -> int:
        return int(lib().gs_sim_launch_count(self.h))

    def autotune(self, reps: int = 5, stream: int = 0) -> dict:
        sc = GsSchedule()
        check(lib().gs_sim_autotune(self.h, reps, C.c_void_p(stream), C.byref(sc)), "gs_sim_autotune")
        return sc.as_dict()

    def schedule(self) -> dict:
        sc = GsSchedule()
        check(lib().gs_sim_get_schedule(self.h, C.byref(sc)), "gs_sim_get_schedule")
        return sc.as_dict()

    def set_schedule(self, **kw) -> None:
        sc = GsSchedule(**{k: int(kw.get(k, 0)) for k, _ in GsSchedule._fields_})
        check(lib().gs_sim_set_schedule(self.h, C.byref(sc)), "gs_sim_set_schedule")

    def use_graph(self, on: bool) -> None:
        check(lib().gs_sim_use_graph(self.h, 1 if on else 0), "use_graph")

    def take_field(self, name: str, src: "Sim", src_name: str) -> None:
        check(lib().gs_sim_take_field(self.h, name.encode(), src.h, src_name.encode()), f"take_field({name})")


class Batch:
    """Many independent martensite simulations advanced together (gs_batch*)."""

    def __init__(self, params: list):
        arr = (GsParams * len(params))()
        for i, p in enumerate(params):
            C.memmove(C.byref(arr[i]), C.byref(p), C.sizeof(GsParams))
        self.params = [p.copy() for p in params]
        h = C.c_void_p()
        check(lib().gs_batch_create(arr, len(params), C.byref(h)), "gs_batch_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().gs_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_eta(self, sim: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr)
        code = GS_DTYPE_F64 if a.dtype == np.float64 else GS_DTYPE_F32
        a = np.ascontiguousarray(a, dtype=_np_dtype(code))
        check(lib().gs_batch_set_field(self.h, sim, b"eta", a.ctypes.data, a.size, code), "batch set_field")

    def eta(self, sim: int, dtype=np.float64) -> np.ndarray:
        p = self.params[sim]
        n = p.nvariants * p.ncells
        out = np.empty(n, dtype=dtype)
        code = GS_DTYPE_F64 if dtype == np.float64 else GS_DTYPE_F32
        check(lib().gs_batch_get_field(self.h, sim, b"eta", out.ctypes.data, n, code), "batch get_field")
        return out.reshape(p.nvariants, p.nx, p.ny, p.nz)

    def step(self, n: int = 1, stream: int = 0) -> None:
        check(lib().gs_batch_step(self.h, n, C.c_void_p(stream)), "gs_batch_step")

    def stats(self, sim: int) -> dict:
        s = GsStats()
        check(lib().gs_batch_stats(self.h, sim, C.byref(s), None), "gs_batch_stats")
        return s.as_dict(self.params[sim].nvariants)

    def use_graph(self, on: bool) -> None:
        check(lib().gs_batch_use_graph(self.h, 1 if on else 0), "use_graph")

    def groups(self) -> int:
        return int(lib().gs_batch_groups(self.h))

    def set_concurrent(self, on: bool) -> None:
        check(lib().gs_batch_set_concurrent(self.h, 1 if on else 0), "gs_batch_set_concurrent")

    def autotune(self, reps: int = 5, stream: int = 0) -> list:
        check(lib().gs_batch_autotune(self.h, reps, C.c_void_p(stream)), "gs_batch_autotune")
        out = []
        for g in range(self.groups()):
            sc = GsSchedule()
            check(lib().gs_batch_get_schedule(self.h, g, C.byref(sc)), "gs_batch_get_schedule")
            out.append(sc.as_dict())
        return out

    def launch_count(self) -> int:
        return int(lib().gs_batch_launch_count(self.h))


# ---------------------------------------------------------------------------
# workload builders: the configurations the step is measured and tested on
# ---------------------------------------------------------------------------

def cubic_cijkl(c11: float, c12: float, c44: float) -> np.ndarray:
    C4 = np.zeros((3, 3, 3, 3))
    for i in range(3):
        for j in range(3):
            C4[i, i, j, j] = c12
        C4[i, i, i, i] = c11
    for i in range(3):
        for j in range(3):
            if i != j:
                C4[i, j, i, j] = c44
                C4[i, j, j, i] = c44
    return C4


def tetragonal_eigenstrains(nv: int, along: float, other: float) -> np.ndarray:
    """Variant p: `along` on axis p mod 3, `other` on the two other axes."""
    eps = np.zeros((nv, 3, 3))
    for p in range(nv):
        for a in range(3):
            eps[p, a, a] = along if a == p % 3 else other
    return eps


def mart2d_params(n: int = 128, dtype: int = GS_DTYPE_F64) -> GsParams:
    """2D square-to-rectangle martensite, 2 variants, FP64, 1000 explicit steps."""
    p = default_params(GS_MODEL_MART, GS_MODE_BASELINE)
    p.dtype = dtype
    p.nvariants = 2
    p.nx, p.ny, p.nz = n, n, 1
    p.dx = p.dy = p.dz = 1.0
    p.dt = 0.01
    p.landau[0], p.landau[1], p.landau[2], p.landau[3] = 0.2, 3.0, 2.0, 1.0
    p.kappa = 1.0
    p.mobility = 1.0
    eps = np.zeros((2, 3, 3))
    eps[0, 0, 0], eps[0, 1, 1] = 0.02, -0.02
    eps[1, 0, 0], eps[1, 1, 1] = -0.02, 0.02
    p.set_eigenstrain(eps)
    p.set_cijkl(cubic_cijkl(1.4, 0.84, 0.28))
    p.set_applied_stress(np.zeros(9))
    p.noise_amp = 0.0
    p.seed = 0
    return p


def _mart_baseline_defaults_host() -> GsParams:
    """The baseline-mode martensite defaults of gs_params_default, filled in
    Python without loading libgsb200.so (a CPU-only caller such as the
    benchmark's CPU arm must not map the product library).  A CPU test keeps
    the two byte-identical."""
    p = GsParams()  # zero-filled, like the C function's memset
    p.model, p.mode, p.dtype = GS_MODEL_MART, GS_MODE_BASELINE, GS_DTYPE_F32
    p.dx = p.dy = p.dz = 1.0
    p.weight_elastic = 1.0
    p.xi = 1.0
    p.nvariants = 3
    p.nx = p.ny = p.nz = 256
    p.dt = 0.005
    p.landau[0], p.landau[1], p.landau[2], p.landau[3] = 0.2, 3.0, 2.0, 1.0
    p.kappa = 0.5
    p.mobility = 1.0
    p.set_eigenstrain(tetragonal_eigenstrains(3, 0.02, -0.01))
    p.set_cijkl(cubic_cijkl(1.4, 0.84, 0.56))
    p.applied_stress[8] = 0.005
    p.noise_amp = 1e-3
    p.seed = 1
    return p


def mart3d_params(n: int = 256, dtype: int = GS_DTYPE_F32, noise: float = 1e-3,
                  host_only: bool = False) -> GsParams:
    """3D cubic-to-tetragonal martensite, 3 variants, sigma_zz = 0.005.
    host_only: start from the Python copy of the defaults (no library load)."""
    p = _mart_baseline_defaults_host() if host_only else default_params(GS_MODEL_MART, GS_MODE_BASELINE)
    p.dtype = dtype
    p.nvariants = 3
    p.nx = p.ny = p.nz = n
    p.dx = p.dy = p.dz = 1.0
    p.dt = 0.005
    p.landau[0], p.landau[1], p.landau[2], p.landau[3] = 0.2, 3.0, 2.0, 1.0
    p.kappa = 0.5
    p.mobility = 1.0
    p.set_eigenstrain(tetragonal_eigenstrains(3, 0.02, -0.01))
    p.set_cijkl(cubic_cijkl(1.4, 0.84, 0.56))
    s = np.zeros((3, 3))
    s[2, 2] = 0.005
    p.set_applied_stress(s)
    p.noise_amp = noise
    p.seed = 1
    return p


def precip3d_params(n: int = 256, dtype: int = GS_DTYPE_F32) -> GsParams:
    """3D precipitate: CH concentration + 4 AC variants, semi-implicit."""
    p = default_params(GS_MODEL_PRECIPITATE, GS_MODE_BASELINE)
    p.dtype = dtype
    p.nvariants = 4
    p.nx = p.ny = p.nz = n
    return p


def ensemble_params(dtype: int = GS_DTYPE_F32, steps_noise: float = 1e-3, seed0: int = 100,
                    counts=(32, 16, 12, 4)) -> list:
    """64 uneven martensite simulations: 32 x 128^2 and 16 x 256^2 (2D, 2
    variants), 12 x 64^3 and 4 x 128^3 (3D, 3 variants); per-simulation
    seeds seed0.., coefficients drawn uniformly (A2 in [0.1,0.4], A4 in
    [2,4], kappa in [0.5,2], eigenstrain magnitude in [0.01,0.03]) from a
    seeded host generator; noise 1e-3, dt 0.005."""
    rng = np.random.default_rng(2024)
    shapes = [((128, 128, 1), 2)] * counts[0] + [((256, 256, 1), 2)] * counts[1] + \
             [((64, 64, 64), 3)] * counts[2] + [((128, 128, 128), 3)] * counts[3]
    out = []
    for i, (shape, V) in enumerate(shapes):
        if V == 2:
            p = mart2d_params(shape[0], dtype=dtype)
            base = np.zeros((2, 3, 3))
            base[0, 0, 0], base[0, 1, 1], base[1, 0, 0], base[1, 1, 1] = 1, -1, -1, 1
        else:
            p = mart3d_params(shape[0], dtype=dtype, noise=steps_noise)
            base = tetragonal_eigenstrains(3, 1.0, -0.5)
        p.nx, p.ny, p.nz = shape
        p.dt = 0.005
        p.noise_amp = steps_noise
        p.landau[0] = rng.uniform(0.1, 0.4)
        p.landau[1] = rng.uniform(2.0, 4.0)
        p.kappa = rng.uniform(0.5, 2.0)
        p.set_eigenstrain(base * rng.uniform(0.01, 0.03))
        p.seed = seed0 + i
        p.sim_id = i
        out.append(p)
    return out


def initial_eta(p: GsParams, seed: int, amp: float = 0.01) -> np.ndarray:
    """eta ~ U[-amp, amp] from numpy's PCG64 with the given seed."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-amp, amp, size=(p.nvariants, p.nx, p.ny, p.nz))


def initial_c(p: GsParams, seed: int, c0: float = 0.12, amp: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return c0 + rng.uniform(-amp, amp, size=(p.nx, p.ny, p.nz))
