"""gs_mart_step_noalloc: the martensite step for callers that cannot allocate
device memory (a host whose pool allocator owns the whole GPU, a loop that
must stay out of the allocator, a plugin whose process owns the device
memory).  Its scratch is a fixed static device array, so the step needs
nothing from the allocator; these tests check, through the C ABI, that two
calls in a row give the same fields as gs_sim_step (FP64 to 1e-12, FP32 to
1e-6 relative L2, the tolerances of the other step tests), that the device's
free memory is the same before and after a run of calls (on a non-default
stream too), and that grids beyond the array's size, overlapping buffers and
buffers off a 16-byte boundary are refused before anything is launched."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

F64, F32 = 1, 0


def _params(gb, shape, V, dtype, noise):
    p = gb.mart3d_params(16, dtype=dtype, noise=noise)
    p.nx, p.ny, p.nz = shape
    if V != 3:
        p.nvariants = V
        p.set_eigenstrain(gb.tetragonal_eigenstrains(V, 0.02, -0.01))
    return p


def _sim_two_steps(gb, p, eta0):
    s = gb.Sim(p)
    try:
        s.set_field("eta", eta0)
        s.step(1)
        e1 = s.eta(np.float64)
        s.step(1)
        e2 = s.eta(np.float64)
        return e1, e2
    finally:
        s.close()


@pytest.mark.parametrize("shape,V,dtype,noise", [
    ((32, 32, 32), 3, F32, 1e-3),
    ((16, 24, 32), 3, F64, 1e-3),
    ((1, 64, 48), 2, F64, 0.0),
    ((48, 64, 1), 4, F32, 1e-3),
])
def test_noalloc_step_matches_sim_step(gb, shape, V, dtype, noise):
    import torch

    p = _params(gb, shape, V, dtype, noise)
    eta0 = gb.initial_eta(p, 11, 0.1)
    e1, e2 = _sim_two_steps(gb, p, eta0)
    tdt = torch.float64 if dtype == F64 else torch.float32
    d0 = torch.from_numpy(np.ascontiguousarray(eta0)).to(device="cuda", dtype=tdt)
    d1 = torch.empty_like(d0)
    d2 = torch.empty_like(d0)
    torch.cuda.synchronize()
    L = gb.lib()
    rc = L.gs_mart_step_noalloc(C.byref(p), d0.data_ptr(), d1.data_ptr(), 0, None)
    assert rc == gb.GS_OK, gb.last_error()
    rc = L.gs_mart_step_noalloc(C.byref(p), d1.data_ptr(), d2.data_ptr(), 1, None)
    assert rc == gb.GS_OK, gb.last_error()
    torch.cuda.synchronize()
    tol = 1e-12 if dtype == F64 else 1e-6
    assert rel_l2(d1.double().cpu().numpy().reshape(e1.shape), e1) < tol
    assert rel_l2(d2.double().cpu().numpy().reshape(e2.shape), e2) < tol


def test_noalloc_rejects_oversize_and_overlap(gb):
    import torch

    L = gb.lib()
    cap = L.gs_mart_step_noalloc_max_bytes()
    assert cap == 16 << 20
    p = _params(gb, (16, 16, 16), 3, F32, 0.0)
    n = 3 * 16 ** 3
    buf = torch.zeros(2 * n, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    # the output starting half-way into the input
    rc = L.gs_mart_step_noalloc(C.byref(p), buf.data_ptr(), buf.data_ptr() + 4 * (n // 2), 0, None)
    assert rc == gb.GS_EINVAL and "overlap" in gb.last_error()
    big = _params(gb, (128, 128, 128), 3, F32, 0.0)  # 25 MB of spectra
    rc = L.gs_mart_step_noalloc(C.byref(big), buf.data_ptr(), buf.data_ptr() + 4 * n, 0, None)
    assert rc == gb.GS_EINVAL and "static scratch holds" in gb.last_error()


def test_noalloc_rejects_misaligned_buffers(gb):
    import torch

    L = gb.lib()
    p = _params(gb, (16, 16, 16), 3, F32, 0.0)
    n = 3 * 16 ** 3
    buf = torch.zeros(2 * n + 8, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    base = buf.data_ptr()
    assert base % 16 == 0
    # 4 bytes off a 16-byte boundary: refused by the host check, nothing launched
    rc = L.gs_mart_step_noalloc(C.byref(p), base + 4, base + 4 * (n + 4), 0, None)
    assert rc == gb.GS_EINVAL and "16-byte" in gb.last_error()
    rc = L.gs_mart_step_noalloc(C.byref(p), base, base + 4 * (n + 1), 0, None)
    assert rc == gb.GS_EINVAL and "16-byte" in gb.last_error()


def test_noalloc_steps_allocate_nothing(gb):
    """After a first call (which looks up the scratch array's address), a run
    of calls, on the default stream and on a torch side stream, leaves the
    device's free memory and torch's allocator unchanged."""
    import torch

    L = gb.lib()
    p = _params(gb, (32, 32, 32), 3, F32, 1e-3)
    eta0 = gb.initial_eta(p, 5, 0.1)
    a = torch.from_numpy(np.ascontiguousarray(eta0)).to(device="cuda", dtype=torch.float32)
    b = torch.empty_like(a)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    # warm-up calls on both streams: the first looks up the scratch address
    # and loads the kernels' modules
    assert L.gs_mart_step_noalloc(C.byref(p), a.data_ptr(), b.data_ptr(), 0, None) == gb.GS_OK, gb.last_error()
    rc = L.gs_mart_step_noalloc(C.byref(p), b.data_ptr(), a.data_ptr(), 1, C.c_void_p(side.cuda_stream))
    assert rc == gb.GS_OK, gb.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for k in range(2, 8):
        src, dst = (a, b) if k % 2 == 0 else (b, a)
        stream = None if k < 5 else C.c_void_p(side.cuda_stream)
        rc = L.gs_mart_step_noalloc(C.byref(p), src.data_ptr(), dst.data_ptr(), k, stream)
        assert rc == gb.GS_OK, gb.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.isfinite(a).all() and torch.isfinite(b).all()
