"""Parity of the CUDA precipitate and stress models (through the C ABI) with
the FP64 oracle and with the reference's own outputs (tests/golden)."""
import numpy as np
import pytest

import refcases as rc
from conftest import rel_l2

pytestmark = pytest.mark.gpu
F64, F32 = 1, 0


def run_precip(gb, p, c0, e0, steps):
    s = gb.Sim(p)
    try:
        s.set_field("concentration", c0)
        s.set_field("eta", e0)
        s.step(steps)
        return s.concentration(), s.eta()
    finally:
        s.close()


def precip_base(gb, shape, dtype, V=4):
    p = gb.precip3d_params(16, dtype=dtype)
    p.nx, p.ny, p.nz = shape
    if V != 4:
        p.nvariants = V
        p.set_eigenstrain(gb.tetragonal_eigenstrains(V, 0.005, -0.0025))
    return p


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 12, 32), (16, 1, 24), (1, 32, 16)])
def test_precip_baseline_fp64(gb, orc, shape):
    p = precip_base(gb, shape, F64)
    c0 = gb.initial_c(p, 2)
    e0 = gb.initial_eta(p, 3, 0.4)
    cr, er = orc.precip_run(p, c0, e0, 3)
    cg, eg = run_precip(gb, p, c0, e0, 3)
    assert rel_l2(cg, cr) < 1e-11 and rel_l2(eg, er) < 1e-11
    assert rel_l2(er, e0) > 1e-3


def test_precip_baseline_noise_fp64(gb, orc):
    p = precip_base(gb, (8, 8, 16), F64)
    p.noise_amp = 1e-2
    p.seed = 77
    c0 = gb.initial_c(p, 4)
    e0 = gb.initial_eta(p, 5, 0.4)
    cr, er = orc.precip_run(p, c0, e0, 2)
    cg, eg = run_precip(gb, p, c0, e0, 2)
    assert rel_l2(cg, cr) < 1e-11 and rel_l2(eg, er) < 1e-11


@pytest.mark.parametrize("shape,V", [((8, 12, 2), 4), ((8, 8, 16), 6), ((2, 4, 512), 8)])
def test_precip_fused_and_separate_passes_fp64(gb, orc, shape, V):
    """Odd runs of two cells (n2 = 2), the wide-variant instances, and the
    longest rows (512 cells, 8 variants: 10 update fields of 16 threads)."""
    p = precip_base(gb, shape, F64, V=V)
    c0 = gb.initial_c(p, 12)
    e0 = gb.initial_eta(p, 13, 0.4)
    p.noise_amp = 1e-3
    cr, er = orc.precip_run(p, c0, e0, 2)
    cg, eg = run_precip(gb, p, c0, e0, 2)
    assert rel_l2(cg, cr) < 1e-11 and rel_l2(eg, er) < 1e-11


@pytest.mark.parametrize("dtype,shape,ce", [(F64, (8, 8, 16), 1), (F32, (16, 12, 32), 1), (F64, (8, 12, 2), 0)])
def test_precip_fused_next_z_forward_same_bits(gb, dtype, shape, ce):
    """The last sweep of a step also writes the next step's chain-1 z spectra;
    uploading eta again before every step (its own values; the concentration
    and its mass stay on the device) forces the separate z forward.  Both give
    the same bits (with and without the concentration's misfit)."""
    p = precip_base(gb, shape, dtype)
    p.c_elastic = ce
    p.noise_amp = 1e-3
    c0 = gb.initial_c(p, 21)
    e0 = gb.initial_eta(p, 22, 0.4)
    if dtype == F32:
        c0 = c0.astype(np.float32).astype(np.float64)
        e0 = e0.astype(np.float32).astype(np.float64)
    s = gb.Sim(p)
    try:
        s.set_field("concentration", c0)
        s.set_field("eta", e0)
        s.step(4)
        fc, fe = s.concentration(np.float64), s.eta(np.float64)
    finally:
        s.close()
    s = gb.Sim(p)
    try:
        s.set_field("concentration", c0)
        e = e0
        for k in range(4):
            s.set_field("eta", e)
            s.step(1)
            e = s.eta(np.float64)
        c = s.concentration(np.float64)
    finally:
        s.close()
    assert np.array_equal(fc, c) and np.array_equal(fe, e)


@pytest.mark.parametrize("V", [1, 2, 3])
def test_precip_variant_counts(gb, orc, V):
    p = precip_base(gb, (8, 8, 8), F64, V=V)
    c0 = gb.initial_c(p, 6)
    e0 = gb.initial_eta(p, 7, 0.4)
    cr, er = orc.precip_run(p, c0, e0, 2)
    cg, eg = run_precip(gb, p, c0, e0, 2)
    assert rel_l2(cg, cr) < 1e-11 and rel_l2(eg, er) < 1e-11


def test_precip_refcompat_fp64(gb, orc):
    p = rc.precip_params(gb)
    p.dtype = F64
    d = rc.load("precipitate")
    c0, e0 = d["con0"].astype(np.float64), d["eta0"].astype(np.float64)
    cr, er = orc.precip_run(p, c0, e0, 3)
    cg, eg = run_precip(gb, p, c0, e0, 3)
    assert rel_l2(cg, cr) < 1e-11 and rel_l2(eg, er) < 1e-11


def test_precip_fp32_matches_reference_fixture(gb):
    p = rc.precip_params(gb)
    d = rc.load("precipitate")
    s = gb.Sim(p)
    s.set_field("concentration", d["con0"])
    s.set_field("eta", d["eta0"])
    for i in range(5):
        s.step(1)
        assert rel_l2(s.eta(), d["eta_steps"][i]) < 2e-6
        assert rel_l2(s.concentration(), d["con_steps"][i]) < 2e-6
    s.close()


@pytest.mark.parametrize("shape,steps,tol", [((128, 128, 128), 60, 1e-10), ((32, 32, 32), 300, 5e-10)])
def test_precip_fp32_mass_drift(gb, shape, steps, tol):
    """The FP64 mass projection keeps the concentration's mass to the
    rounding of the stored FP32 field, about eps_32 / sqrt(N) relative (it
    does not grow with the steps): below 1e-10 from 128^3 up (the bar is set
    for 256^3), a few 1e-10 at 32^3."""
    p = precip_base(gb, shape, F32)
    c0 = gb.initial_c(p, 2).astype(np.float32)
    e0 = gb.initial_eta(p, 3, 0.3).astype(np.float32)
    s = gb.Sim(p)
    s.set_field("concentration", c0)
    s.set_field("eta", e0)
    m0 = c0.astype(np.float64).sum()
    st0 = s.stats()
    assert abs(st0["mass"] - m0) <= 1e-12 * m0
    s.step(steps)
    st = s.stats()
    c = s.concentration()
    s.close()
    assert abs(st["mass"] - m0) / m0 < tol
    assert abs(c.sum() - m0) / m0 < tol


def test_precip_stats_match_oracle(gb, orc):
    p = precip_base(gb, (16, 16, 8), F64)
    c0 = gb.initial_c(p, 8)
    e0 = gb.initial_eta(p, 9, 0.8)
    s = gb.Sim(p)
    s.set_field("concentration", c0)
    s.set_field("eta", e0)
    st = s.stats()
    s.close()
    ref = orc.precip_stats(p, c0, e0)
    for k in ["mass", "c_mean", "eta_mean", "e_el", "e_chem", "e_grad", "e_tot"]:
        assert abs(st[k] - ref[k]) <= 1e-10 * max(1.0, abs(ref[k])), k
    assert np.allclose(st["eta2"], ref["eta2"], rtol=1e-12) and st["vf"] == ref["vf"]


def run_stress(gb, p, e0):
    s = gb.Sim(p)
    try:
        s.set_field("eta", e0)
        s.step(1)
        n = p.nx * p.ny * p.nz
        return (s.get_field("stress", 6 * n).reshape(6, p.nx, p.ny, p.nz),
                s.get_field("defect", n).reshape(p.nx, p.ny, p.nz))
    finally:
        s.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_stress_fp64_matches_oracle(gb, orc, mode):
    p = gb.default_params(gb.GS_MODEL_STRESS, mode)
    p.dtype = F64
    p.nx, p.ny, p.nz = 12, 16, 8
    p.nvariants = 3
    p.set_eigenstrain(gb.tetragonal_eigenstrains(3, 0.01, -0.004))
    e0 = gb.initial_eta(p, 10, 1.0)
    sr, dr = orc.stress(p, e0)
    sg, dg = run_stress(gb, p, e0)
    assert rel_l2(sg, sr) < 1e-11
    assert np.array_equal(dg, dr)


def test_stress_fp32_matches_reference_fixture(gb):
    d = rc.load("stress")
    p = rc.stress_params(gb, str(d["log"]))
    sg, dg = run_stress(gb, p, d["eta0"])
    assert rel_l2(sg, d["stress"]) < 2e-6
    assert np.array_equal(dg, d["defect"])


@pytest.mark.parametrize("dtype", [F64, F32])
def test_stress_to_mart_handoff_on_device(gb, dtype):
    """gs_sim_take_field: the stress stage's stress and defect handed to a
    martensite simulation on the device step it exactly as the same fields
    downloaded and uploaded through the host."""
    shape = (16, 12, 8)
    ps = gb.default_params(gb.GS_MODEL_STRESS, gb.GS_MODE_REFCOMPAT)
    ps.dtype = dtype
    ps.nx, ps.ny, ps.nz = shape
    ps.nvariants = 4
    t = 0.0063
    eps = np.array([[[0.01, t, t], [t, -0.004, t], [t, t, 0.002]],
                    [[0.0, t, -t], [t, 0.01, -t], [-t, -t, 0.0]],
                    [[0.0, -t, t], [-t, 0.0, -t], [t, -t, 0.01]],
                    [[-0.01, -t, -t], [-t, 0.0, t], [-t, t, 0.0]]])
    ps.set_eigenstrain(eps)
    rng = np.random.default_rng(3)
    eta_s = rng.uniform(0.0, 1.0, (4,) + shape)
    st = gb.Sim(ps)
    pm = gb.default_params(gb.GS_MODEL_MART, gb.GS_MODE_REFCOMPAT)
    pm.dtype = dtype
    pm.nx, pm.ny, pm.nz = shape
    pm.nvariants = 4
    pm.set_eigenstrain(eps)
    pm.weight_dislocation = 0.1
    eta0 = rng.uniform(0.0, 0.1, (4,) + shape)
    a, b = gb.Sim(pm), gb.Sim(pm)
    try:
        st.set_field("eta", eta_s)
        st.step(1)
        N = int(np.prod(shape))
        stress = st.get_field("stress", 6 * N, np.float64 if dtype == F64 else np.float32)
        defect = st.get_field("defect", N, np.float64 if dtype == F64 else np.float32)
        a.set_field("eta", eta0)
        a.set_field("dislocationstress", stress)
        a.set_field("defect", defect)
        b.set_field("eta", eta0)
        b.take_field("dislocationstress", st, "stress")
        b.take_field("defect", st, "defect")
        a.step(3)
        b.step(3)
        assert np.array_equal(a.eta(), b.eta())
        assert defect.sum() > 0 and np.abs(stress).max() > 0
    finally:
        a.close()
        b.close()
        st.close()
