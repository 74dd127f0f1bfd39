"""The bounds checks of the pass kernels on the GPU.

Two halves.  The launch-range check (every build, gs_set_bounds_check):
before a pass kernel launches, each buffer range its launch reaches must lie
inside one device allocation; a caller buffer that is too small is refused
before anything runs.  The bounds-check build (libgsb200_bc.so, loaded under
GS_BOUNDS_CHECK=1): every index a pass kernel forms is checked against the
launch's extents; a violation is recorded (site, index, extent) and the
access kept inside the buffer, never trapped.  The build is run here on its
self-test kernel, whose violations are planted by its arguments and whose
accesses all stay inside the buffer, and on the oracle parity suites of every
step kind, which must pass with no violation recorded.

Nothing here reads or writes outside an allocation: the refused launch never
runs, and the self-test's out-of-range indices are redirected in-bounds."""
import json
import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

F32 = 0


def _bc_env():
    env = dict(os.environ)
    env["GS_BOUNDS_CHECK"] = "1"
    return env


_SELFTEST = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import torch, gs_b200 as gb
assert gb.BOUNDS_CHECK_BUILD and gb.lib().gs_bounds_check_build() == 1
cap, n = 1000, 1500
buf = torch.full((cap + 64,), -1, dtype=torch.int32, device="cuda")
gb.bounds_record(clear=True)
gb.check(gb.lib().gs_bounds_selftest(buf.data_ptr(), cap, n, None), "gs_bounds_selftest")
rec = gb.bounds_record(clear=True)
after = gb.bounds_record()
b = buf.cpu().numpy()
print(json.dumps({"rec": rec, "after": after["violations"],
                  "inside_ok": bool((b[1:cap] == range(1, cap)).all()),
                  "tail_untouched": bool((b[cap:] == -1).all())}))
"""


def test_selftest_records_planted_violations():
    """n - cap indices beyond cap: each is counted, the first recorded, none
    written past cap (the redirected stores land on element 0)."""
    r = subprocess.run([sys.executable, "-c", _SELFTEST, os.path.join(ROOT, "general-simulator_b200")],
                       capture_output=True, text=True, env=_bc_env(), timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    rec = out["rec"]
    assert rec["violations"] == 500
    assert rec["site_name"] == "selftest"
    assert 1000 <= rec["index"] < 1500 and rec["extent"] == 1000
    assert out["after"] == 0  # cleared
    assert out["inside_ok"] and out["tail_untouched"]


def test_range_check_refuses_a_short_caller_buffer(gb):
    """gs_mart_step_noalloc with an eta buffer 4 KiB shorter than the grid:
    the z forward's launch is refused, nothing runs.  The buffer is sized
    2 MiB - 4 KiB, so even the bytes the refused launch would have read lie
    in the same 2 MiB page of this allocation."""
    import ctypes as C

    import torch
    from cuda.bindings import runtime as rt

    p = gb.mart3d_params(64, dtype=F32, noise=1e-3)
    p.nvariants = 2
    p.set_eigenstrain(gb.tetragonal_eigenstrains(2, 0.02, -0.01))
    need = 2 * 64 ** 3 * 4
    assert need == 2 << 20
    err, short = rt.cudaMalloc(need - 4096)
    assert err == rt.cudaError_t.cudaSuccess
    out = torch.empty(2 * 64 ** 3, dtype=torch.float32, device="cuda")
    L = gb.lib()
    was = L.gs_bounds_check_enabled()
    try:
        gb.set_bounds_check(True)
        torch.cuda.synchronize()
        rc = L.gs_mart_step_noalloc(C.byref(p), C.c_void_p(int(short)), C.c_void_p(out.data_ptr()), 0, None)
        msg = gb.last_error()
        assert rc == gb.GS_EINVAL, (rc, msg)
        assert "bounds check" in msg and "z forward" in msg, msg
        torch.cuda.synchronize()  # the context is fine: nothing ran
    finally:
        gb.set_bounds_check(bool(was))
        rt.cudaFree(short)


def test_range_check_passes_every_step_kind(gb):
    """No false refusals: the product's own buffers fit their launches."""
    L = gb.lib()
    was = L.gs_bounds_check_enabled()
    try:
        gb.set_bounds_check(True)
        p = gb.mart3d_params(64, dtype=F32, noise=1e-3)
        s = gb.Sim(p)
        s.set_field("eta", gb.initial_eta(p, 3, 0.1))
        s.step(3)
        s.stats()
        s.use_graph(True)
        s.step(4)
        s.close()
        q = gb.precip3d_params(32, dtype=F32)
        t = gb.Sim(q)
        t.set_field("concentration", gb.initial_c(q, 5))
        t.set_field("eta", gb.initial_eta(q, 6, 0.1))
        t.step(3)
        t.stats()
        t.close()
        b = gb.Batch([gb.mart3d_params(32, dtype=F32, noise=1e-3) for _ in range(3)])
        b.step(2)
        b.close()
    finally:
        gb.set_bounds_check(bool(was))


def test_bounds_check_build_passes_the_gpu_suite():
    """The whole GPU suite (oracle parity of every step kind at test and full
    sizes, the long-run bars, graphs, ensembles, adjoints, slabs, the TMA x
    pass, the autotuner's schedules) re-run on the bounds-check build.  Under
    GS_BOUNDS_CHECK=1 every step entry waits for its kernels and returns
    GS_EBOUNDS after an index violation, so one out-of-range index anywhere
    fails it.  (The script front end links the normal library: left out.)"""
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider", "tests",
                        "--ignore=tests/test_gpu_bounds.py", "--ignore=tests/test_frontend.py"],
                       cwd=ROOT, capture_output=True, text=True, env=_bc_env(), timeout=3000)
    lines = (r.stdout + r.stderr).strip().splitlines()
    tail = "\n".join(lines[-15:])
    assert r.returncode == 0, tail
    m = re.search(r"(\d+) passed", lines[-1])
    assert m and int(m.group(1)) >= 150 and "failed" not in lines[-1], tail
    print(lines[-1])
