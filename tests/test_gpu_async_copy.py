"""Field copies that overlap stepping (gs_sim_copy_field_async / _wait) and
the stream upload (gs_sim_set_field_async), through the C ABI, against the
synchronous gs_sim_get_field / gs_sim_set_field: the same values."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(gb, n=32, dtype=0):
    p = gb.mart3d_params(n, dtype=dtype, noise=1e-3)
    sim = gb.Sim(p)
    sim.set_field("eta", gb.initial_eta(p, 2, 0.3))
    return p, sim


def test_copy_into_library_staging_and_converted(gb):
    p, sim = _sim(gb)
    L = gb.lib()
    try:
        sim.step(3)
        want = sim.eta(np.float32)
        t = C.c_int(0)
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t)), "async")
        sim.step(2)  # overwrites the field: the copy holds the snapshot
        got32 = np.empty(want.size, np.float32)
        gb.check(L.gs_sim_copy_field_wait(sim.h, t.value, got32.ctypes.data, got32.size, 0), "wait")
        assert np.array_equal(got32.reshape(want.shape), want)
        # two in flight, waited in the other order, one converted to FP64
        t1, t2 = C.c_int(0), C.c_int(0)
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t1)), "async")
        sim.step(1)
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t2)), "async")
        later = sim.eta(np.float32)
        a = np.empty(want.size, np.float64)
        b = np.empty(want.size, np.float32)
        gb.check(L.gs_sim_copy_field_wait(sim.h, t2.value, b.ctypes.data, b.size, 0), "wait")
        gb.check(L.gs_sim_copy_field_wait(sim.h, t1.value, a.ctypes.data, a.size, 1), "wait")
        assert np.array_equal(b.reshape(want.shape), later)
        assert not np.array_equal(a.astype(np.float32), b)
        # a ticket is waited for once
        assert L.gs_sim_copy_field_wait(sim.h, t1.value, a.ctypes.data, a.size, 1) == gb.GS_EINVAL
        assert L.gs_sim_copy_field_async(sim.h, b"nosuch", None, None, C.byref(t1)) == gb.GS_EINVAL
    finally:
        sim.close()


def test_direct_pinned_copy_and_stream_upload(gb):
    import torch

    p, sim = _sim(gb, 48)
    p2, sim2 = _sim(gb, 48)
    L = gb.lib()
    try:
        n = p.nvariants * p.ncells
        src = torch.from_numpy(gb.initial_eta(p, 9, 0.3).astype(np.float32).ravel()).pin_memory()
        dst = torch.empty(n, dtype=torch.float32).pin_memory()
        stream = torch.cuda.Stream()
        sh = C.c_void_p(stream.cuda_stream)
        t = C.c_int(0)
        gb.check(L.gs_sim_set_field_async(sim.h, b"eta", C.c_void_p(src.data_ptr()), n, 0, sh), "upload")
        gb.check(L.gs_sim_step(sim.h, 3, sh), "step")
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", sh, C.c_void_p(dst.data_ptr()), C.byref(t)), "async")
        gb.check(L.gs_sim_copy_field_wait(sim.h, t.value, None, 0, 0), "wait")
        sim2.set_field("eta", src.numpy())
        sim2.step(3)
        assert np.array_equal(dst.numpy(), sim2.eta(np.float32).ravel())
        # the upload takes the simulation's dtype only
        assert L.gs_sim_set_field_async(sim.h, b"eta", C.c_void_p(src.data_ptr()), n, 1, sh) == gb.GS_EINVAL
    finally:
        sim.close()
        sim2.close()


def test_fp64_copy_converted_and_third_copy_waits_for_a_slot(gb):
    import threading

    p, sim = _sim(gb, 24, dtype=1)
    L = gb.lib()
    try:
        sim.step(2)
        want = sim.eta(np.float32)
        t1, t2, t3 = C.c_int(0), C.c_int(0), C.c_int(0)
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t1)), "async")
        gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t2)), "async")
        rc3 = []
        th = threading.Thread(target=lambda: rc3.append(
            L.gs_sim_copy_field_async(sim.h, b"eta", None, None, C.byref(t3))))
        th.start()
        th.join(0.5)
        assert th.is_alive()  # both slots are taken until a wait frees one
        got = np.empty(want.size, np.float32)
        gb.check(L.gs_sim_copy_field_wait(sim.h, t1.value, got.ctypes.data, got.size, 0), "wait")
        th.join(30)
        assert not th.is_alive() and rc3 == [0]
        assert np.array_equal(got.reshape(want.shape), want)  # FP64 state rounded to FP32
        for t in (t2, t3):
            gb.check(L.gs_sim_copy_field_wait(sim.h, t.value, got.ctypes.data, got.size, 0), "wait")
    finally:
        sim.close()
