"""The C++ script front end (general-simulator_b200/gsi) against the
reference: known-answer scripts byte for byte on CPU, the three physics
scripts against the reference's own outputs on the GPU."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import refcases as rc
from conftest import PKG, ROOT, rel_l2

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_ref_fixtures as mf  # noqa: E402

GSI = os.path.join(PKG, "gsi")


@pytest.fixture(scope="module")
def gsi():
    if not os.path.exists(GSI):
        import build

        build.build_frontend()
    return GSI


def run_script(gsi, tmp_path, name, text, inputs=None):
    for fn, arr in (inputs or {}).items():
        mf.write_text_field(str(tmp_path / fn), arr)
    (tmp_path / name).write_text(text)
    r = subprocess.run([gsi, name], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    return r.stdout


# the reference's front-end scripts, recorded from its own binary
KAT_IF_LOOP_WHILE = """########################################################
set log off
expr a=3
loop (a*2)
  print {a}
  :a=a-1
end
print {a}

########################################################
:a=3
while a>0
  expr a=a-1
  print {a}
end
print {a}

########################################################
:a=2
if (a>3)
  print {a*9^2}
else
  print {a^2}
end
"""

KAT_POW = """########################################################
sys pow
########################################################
expr total_step=20
########################################################
set x 2
########################################################
readhere matrix
2 3 3
3 9 8
1 2 3
6 5 4
########################################################
info {total_step} x sum_of_matrix
dump dump_pow_matrix {total_step} matrix
########################################################
run {total_step}
"""


@pytest.mark.parametrize("name,text,golden", [("in.if.loop.while", KAT_IF_LOOP_WHILE, "frontend_in_if_loop_while.txt"),
                                              ("in.pow", KAT_POW, "frontend_in_pow.txt")])
def test_known_answer_scripts_identical(gsi, tmp_path, name, text, golden):
    out = run_script(gsi, tmp_path, name, text)
    ref = open(os.path.join(rc.GOLDEN, golden)).read()
    assert out == ref
    assert (tmp_path / (name + ".log")).read_text() == ref  # the log tee


def test_pow_dump_files(gsi, tmp_path):
    run_script(gsi, tmp_path, "in.pow", KAT_POW)
    f = (tmp_path / "dump_pow_matrix" / "matrix.20.data").read_text().split()
    assert f[:3] == ["2", "3", "3"]
    assert float(f[3]) == pytest.approx(3 * 2 ** 20, rel=1e-6)


def test_expressions_and_blocks(gsi, tmp_path):
    # arithmetic, $globals, nested loops, if/else, division by zero and the
    # reference's own reading of `z+=4` (split at the later `=`: assigns "z+")
    text = open(os.path.join(rc.GOLDEN, "scripts", "in.expr")).read()
    out = run_script(gsi, tmp_path, "in.expr", text)
    assert out == open(os.path.join(rc.GOLDEN, "frontend_in_expr.txt")).read()


def test_errors_are_reported(gsi, tmp_path):
    out = run_script(gsi, tmp_path, "in.e", "sys nosuch\n")
    assert 'Error: unknown system "nosuch"' in out and "Error: error in command" in out
    out = run_script(gsi, tmp_path, "in.e2", "run 3\n")
    assert "Error: system not set" in out
    out = run_script(gsi, tmp_path, "in.e3", "sys mart\nrun 1\n")
    assert "strain tensor does not set" in out


@pytest.mark.gpu
def test_mart_script_matches_reference(gsi, tmp_path):
    out = run_script(gsi, tmp_path, "in.mart16", mf.mart_script(), mf.mart_inputs())
    mine = rc.info_rows(out)
    ref = rc.info_rows(str(rc.load("mart")["log"]))
    assert len(mine) == 5
    for a, b in zip(mine, ref):
        assert a[0] == b[0]  # temperature
        for j in (1, 3, 4, 5):  # eta, chemical, elastic, dislocation means
            assert abs(a[j] - b[j]) <= 2e-5 * abs(b[j]), (j, a[j], b[j])
    # unlike the reference (stale host copy), the dump holds the evolved field
    d = mf.read_binary_field(str(tmp_path / "dumpdir" / "eta.5.data"))
    assert not np.array_equal(d, mf.mart_inputs()["data.eta"])


@pytest.mark.gpu
def test_precipitate_script_matches_reference(gsi, tmp_path):
    run_script(gsi, tmp_path, "in.precipitate16", mf.precip_script(), mf.precip_inputs())
    ref = rc.load("precipitate")
    for i in range(1, 6):
        e = mf.read_binary_field(str(tmp_path / "dumpdir" / f"eta.{i}.data"))
        c = mf.read_binary_field(str(tmp_path / "dumpdir" / f"concentration.{i}.data"))
        assert rel_l2(e, ref["eta_steps"][i - 1]) < 2e-6
        assert rel_l2(c, ref["con_steps"][i - 1]) < 2e-6


@pytest.mark.gpu
def test_stress_script_matches_reference(gsi, tmp_path):
    out = run_script(gsi, tmp_path, "in.stress16", mf.stress_script(), mf.stress_inputs())
    ref = rc.load("stress")
    assert out[out.find(">>>writehere"):out.find(">>>set binary on")] == \
        str(ref["log"])[str(ref["log"]).find(">>>writehere"):str(ref["log"]).find(">>>set binary on")]
    s = mf.read_binary_field(str(tmp_path / "dumpdir" / "stress.1.data"))
    d = mf.read_binary_field(str(tmp_path / "dumpdir" / "defect.1.data"))
    assert rel_l2(s, ref["stress"]) < 2e-6
    assert np.array_equal(d, ref["defect"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", mf.CORES_CASES, ids=[c[0] for c in mf.CORES_CASES])
def test_cores_script_identical_to_reference(gsi, tmp_path, case):
    """`sys cores`: the same draws and the device painting give the
    reference binary's eta and concentration dumps exactly."""
    name, grid, V, n, r, method = case
    run_script(gsi, tmp_path, "in.cores", mf.cores_script(grid, V, n, r, method))
    ref = rc.load("cores")
    eta = mf.read_binary_field(str(tmp_path / "dd" / "eta.1.data"))
    conc = mf.read_binary_field(str(tmp_path / "dd" / "concentration.1.data"))
    assert np.array_equal(eta, ref[f"{name}_eta"])
    assert np.array_equal(conc, ref[f"{name}_concentration"])


@pytest.mark.gpu
def test_cores_paint_matches_oracle_large(gb, orc):
    """gs_cores_paint through the C ABI against the oracle on a larger grid
    with overlapping nuclei of several variants."""
    import ctypes as C

    rng = np.random.default_rng(5)
    grid, V, n, r = (64, 48, 40), 4, 25, 7.5
    centers = rng.integers(0, [64, 48, 40], size=(n, 3)).astype(np.int32)
    variants = rng.integers(0, V, size=n).astype(np.int32)
    eta = np.zeros((V,) + grid, np.float32)
    conc = np.zeros(grid, np.float32)
    L = gb.lib()
    rc_ = L.gs_cores_paint(*grid, V, n, centers.ctypes.data_as(C.c_void_p), variants.ctypes.data_as(C.c_void_p),
                           C.c_double(r), C.c_double(0.2), C.c_double(0.44), eta.ctypes.data_as(C.c_void_p),
                           conc.ctypes.data_as(C.c_void_p))
    assert rc_ == gb.GS_OK, gb.last_error()
    oe, oc = orc.cores_paint(grid, V, centers.tolist(), variants.tolist(), r, 0.2, 0.44)
    assert np.array_equal(eta, oe) and np.array_equal(conc, oc)
    assert (eta.sum(axis=0) > 1).any()  # overlaps of different variants are exercised


def test_time_calculate_script(gsi, tmp_path):
    """scripts/in.time_calculate of the reference: backquoted shell output in
    variables and expressions ({x2-x1} is the seconds slept)."""
    text = """set log off
print `date`
:x1=`date +%s`
shell sleep 1
print `date`
:x2=`date +%s`
print since time point {x1} to time point {x2}, {x2-x1} seconds have passed.
"""
    out = run_script(gsi, tmp_path, "in.time_calculate", text)
    import re

    m = re.search(r"since time point (\d+) to time point (\d+), (\d+) seconds have passed\.", out)
    assert m, out
    x1, x2, d = map(int, m.groups())
    assert d == x2 - x1 and 1 <= d <= 3


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["mart", "precipitate", "stress"])
def test_async_dumps_equal_synchronous_dumps(gsi, tmp_path, case):
    """`dump` overlaps the following steps (device snapshot, copy and file
    write off the stepping thread); the files must equal those of the
    synchronous dump (`set asyncdump 0`) byte for byte."""
    script, inputs = {"mart": (mf.mart_script, mf.mart_inputs), "precipitate": (mf.precip_script, mf.precip_inputs),
                      "stress": (mf.stress_script, mf.stress_inputs)}[case]
    files = {}
    for mode in ("async", "sync"):
        d = tmp_path / mode
        d.mkdir()
        text = script()
        if mode == "sync":
            text = "set asyncdump 0\n" + text
        run_script(gsi, d, "in." + case, text, inputs())
        files[mode] = {p.name: p.read_bytes() for p in sorted((d / "dumpdir").iterdir())}
    assert files["async"] and files["async"].keys() == files["sync"].keys()
    for k in files["async"]:
        assert files["async"][k] == files["sync"][k], k
