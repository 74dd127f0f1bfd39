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


@pytest.mark.parametrize("graph", [False, True])
def test_staged_uploads_equal_synchronous_uploads(gb, graph):
    """gs_sim_stage_field_async: each step's input staged from page-locked
    memory while the previous step runs and its output downloads; the steps
    give the same bits as uploading with gs_sim_set_field before each step.
    A set_field after staging drops the staged set; a second stage before a
    step is refused."""
    import torch

    p = gb.mart3d_params(32, dtype=0, noise=1e-3)
    n = p.nvariants * p.ncells
    L = gb.lib()
    inputs = [torch.from_numpy(gb.initial_eta(p, 30 + k, 0.3).astype(np.float32).ravel()).pin_memory()
              for k in range(4)]
    outs = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(4)]
    ref = []
    s = gb.Sim(p)
    try:
        for k in range(4):
            s.set_field("eta", inputs[k].numpy())
            s.step(1)
            ref.append(s.eta(np.float32).ravel())
    finally:
        s.close()
    s = gb.Sim(p)
    try:
        s.use_graph(graph)
        tk = C.c_int(0)
        gb.check(L.gs_sim_stage_field_async(s.h, b"eta", C.c_void_p(inputs[0].data_ptr()), n, 0), "stage")
        assert L.gs_sim_stage_field_async(s.h, b"eta", C.c_void_p(inputs[0].data_ptr()), n, 0) == gb.GS_EINVAL
        tickets = []
        for k in range(4):
            s.step(1)
            gb.check(L.gs_sim_copy_field_async(s.h, b"eta", None, C.c_void_p(outs[k].data_ptr()), C.byref(tk)), "dl")
            tickets.append(tk.value)
            if k + 1 < 4:
                gb.check(L.gs_sim_stage_field_async(s.h, b"eta", C.c_void_p(inputs[k + 1].data_ptr()), n, 0), "stage")
            if len(tickets) == 2:
                gb.check(L.gs_sim_copy_field_wait(s.h, tickets.pop(0), None, 0, 0), "wait")
        for t in tickets:
            gb.check(L.gs_sim_copy_field_wait(s.h, t, None, 0, 0), "wait")
        for k in range(4):
            assert np.array_equal(outs[k].numpy(), ref[k]), k
        # a staged set dropped by a direct upload
        gb.check(L.gs_sim_stage_field_async(s.h, b"eta", C.c_void_p(inputs[3].data_ptr()), n, 0), "stage")
        s.set_field("eta", inputs[0].numpy())
        s.set_scalar("step", 0)
        s.step(1)
        assert np.array_equal(s.eta(np.float32).ravel(), ref[0])
    finally:
        s.close()
