"""The oracle pinned against outputs of the reference itself.

tests/golden/ref_*.npz were produced by the reference's own gsi (HEAD side of
its conflicts, the p++ fix, nvcc for sm_100a; oracle/build_ref.sh) on seeded
16x12x8 inputs by tests/golden/make_ref_fixtures.py.  The reference computes
in FP32 (cuFFT, FP32 B tensor); the oracle in FP64 with the reference's own
formulas (GS_MODE_REFCOMPAT).
"""
import numpy as np
import pytest

import refcases as rc
from conftest import rel_l2


def test_mart_info_means_match_reference(gb, orc):
    # The reference's `dump` of a read-in eta writes the stale host copy
    # (Data::operator+= keeps Position == Data_HOST), so its info means are
    # the golden values: eta after step i, forces of the state before step i.
    d = rc.load("mart")
    rows = rc.info_rows(str(d["log"]))
    assert len(rows) == 5
    assert np.array_equal(d["eta_steps"][4], d["eta0"])  # the stale dump itself
    p = rc.mart_params(gb)
    eta = d["eta0"].astype(np.float64)
    df = d["defect"].astype(np.float64)
    ds = d["dislocationstress"].astype(np.float64)
    for i in range(1, 6):
        p.temperature = rc.ramp_temperature(i, 5)
        assert p.temperature == rows[i - 1][0]
        st = orc.mart_stats(p, eta, defect=df, dstress=ds)
        eta = orc.mart_run(p, eta, 1, step0=i - 1, defect=df, dstress=ds)
        T, em, grad, chem, el, disl = rows[i - 1]
        # six significant digits are printed
        assert abs(eta.mean() - em) <= 1e-5 * abs(em)
        assert abs(st["chemical_mean"] - chem) <= 2e-5 * abs(chem)
        assert abs(st["elastic_mean"] - el) <= 2e-5 * abs(el)
        assert abs(st["dislocation_mean"] - disl) <= 2e-5 * abs(disl)
        assert abs(grad) < 1e-8 and abs(st["gradient_mean"]) < 1e-12  # sums of a periodic Laplacian


def test_precipitate_fields_match_reference(gb, orc):
    d = rc.load("precipitate")
    p = rc.precip_params(gb)
    c = d["con0"].astype(np.float64)
    e = d["eta0"].astype(np.float64)
    for i in range(5):
        c, e = orc.precip_run(p, c, e, 1, step0=i)
        assert rel_l2(e, d["eta_steps"][i]) < 1e-6
        assert rel_l2(c, d["con_steps"][i]) < 1e-6
    assert rel_l2(d["eta_steps"][4], d["eta0"]) > 0.5  # the fields did move


def test_stress_and_defect_match_reference(gb, orc):
    d = rc.load("stress")
    p = rc.stress_params(gb, str(d["log"]))
    st, df = orc.stress(p, d["eta0"].astype(np.float64))
    assert rel_l2(st, d["stress"]) < 1e-6
    assert np.array_equal(df, d["defect"])


@pytest.mark.gpu
def test_gpu_mart_refcompat_matches_reference(gb):
    d = rc.load("mart")
    rows = rc.info_rows(str(d["log"]))
    p = rc.mart_params(gb)
    s = gb.Sim(p)
    s.set_field("eta", d["eta0"])
    s.set_field("defect", d["defect"])
    s.set_field("dislocationstress", d["dislocationstress"])
    for i in range(1, 6):
        s.set_scalar("temperature", rc.ramp_temperature(i, 5))
        st = s.stats()
        s.step(1)
        em = s.eta(np.float64).mean()
        T, em_ref, grad, chem, el, disl = rows[i - 1]
        assert abs(em - em_ref) <= 1e-5 * abs(em_ref)
        assert abs(st["chemical_mean"] - chem) <= 5e-5 * abs(chem)
        assert abs(st["elastic_mean"] - el) <= 5e-5 * abs(el)
        assert abs(st["dislocation_mean"] - disl) <= 5e-5 * abs(disl)
    s.close()


# ---- nuclei of the precipitate chain (Dynamics_cores) ----------------------
CORES_CASES = [("random", (32, 24, 16), 4, 3, 4.5, "random"),
               ("random_dense", (16, 16, 16), 3, 8, 5.0, "random"),
               ("regular", (24, 20, 32), 4, 2, 3.0, "regular")]


def _libc_random():
    import ctypes

    libc = ctypes.CDLL(None)
    libc.random.restype = ctypes.c_long
    libc.srandom(1)  # the state of a fresh process
    return lambda: int(libc.random())


@pytest.mark.parametrize("case", CORES_CASES, ids=[c[0] for c in CORES_CASES])
def test_oracle_cores_match_reference(orc, case):
    """The oracle's placement (the reference's random() draws and marks) and
    painting reproduce the reference binary's eta and concentration."""
    name, grid, V, n, r, method = case
    ref = rc.load("cores")
    centers, variants = orc.cores_place(grid, V, n, r, method, _libc_random())
    eta, conc = orc.cores_paint(grid, V, centers, variants, r, 0.2, 0.44)
    assert np.array_equal(eta, ref[f"{name}_eta"])
    assert np.array_equal(conc, ref[f"{name}_concentration"])
