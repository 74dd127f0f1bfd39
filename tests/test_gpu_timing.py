"""GS_TIMING: per-pass CUDA-event timers of gs_sim_step, one JSON line per
step.  Run in a child process, since the library reads the variable once."""
import json
import os
import subprocess
import sys
import textwrap

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

CHILD = textwrap.dedent("""
    import sys
    sys.path.insert(0, {pkg!r})
    import numpy as np
    import gs_b200 as gb
    p = gb.mart3d_params(32, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    s = gb.Sim(p)
    s.set_field("eta", gb.initial_eta(p, 1))
    s.step(3)
    s.close()
    q = gb.precip3d_params(32, dtype=gb.GS_DTYPE_F32)
    s = gb.Sim(q)
    s.set_field("concentration", gb.initial_c(q, 2))
    s.set_field("eta", gb.initial_eta(q, 3))
    s.step(2)
    s.close()
""")


def test_gs_timing_writes_one_line_per_step(tmp_path):
    out = tmp_path / "timing.jsonl"
    env = dict(os.environ, GS_TIMING=str(out))
    r = subprocess.run([sys.executable, "-c", CHILD.format(pkg=PKG)], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(ln) for ln in out.read_text().splitlines()]
    assert [ln["model"] for ln in lines] == ["martensite"] * 3 + ["precipitate"] * 2
    assert [ln["step"] for ln in lines] == [0, 1, 2, 0, 1]
    first, steady = lines[0], lines[1]
    # the first martensite step runs the z forward on its own; later ones take
    # the spectra the update left behind
    assert [p["name"] for p in first["passes"]] == ["z_forward", "y_forward", "x_contraction", "y_inverse", "update"]
    assert [p["name"] for p in steady["passes"]] == ["y_forward", "x_contraction", "y_inverse", "update"]
    for ln in lines:
        assert ln["grid"] == [32, 32, 32]
        assert all(p["ms"] > 0 for p in ln["passes"])
        assert abs(sum(p["ms"] for p in ln["passes"]) - ln["step_ms"]) < 1e-3
    assert "precip_mid" in [p["name"] for p in lines[3]["passes"]]


def test_gs_timing_off_writes_nothing(tmp_path):
    env = dict(os.environ)
    env.pop("GS_TIMING", None)
    r = subprocess.run([sys.executable, "-c", CHILD.format(pkg=PKG)], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "gs_timing" not in r.stderr
