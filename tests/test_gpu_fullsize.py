"""Parity at the benchmark sizes themselves: the 256^3 x 3 martensite
workload of the headline and the 256^3 precipitate (concentration + 4
variants), FP32 on the device against the FP64 oracle on all host cores, a
few steps each (about 4 s of oracle time per martensite step).

Tolerances: 1e-6 relative L2 per step for FP32 fields (the accuracy bar of
the step), statistics (mass, elastic energy, volume fractions) within 1e-3
relative; FP32 mass of the precipitate conserved to 1e-9 relative."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_headline_martensite_256_matches_oracle(gb, orc):
    """Two steps of the headline workload; after each step the device field
    is within 1e-6 of the oracle run from the device's previous state (the
    error of that step) and of the oracle run from the start (the error so
    far)."""
    p = gb.mart3d_params(256, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    eta0 = gb.initial_eta(p, 1).astype(np.float32)
    q = p.copy()
    q.dtype = gb.GS_DTYPE_F64
    steps = 2
    sim = gb.Sim(p)
    prev = eta0.astype(np.float64)
    ref = prev
    try:
        sim.set_field("eta", eta0)
        for k in range(steps):
            sim.step(1)
            got = sim.eta(np.float64)
            one = orc.mart_run(q, prev, 1, step0=k)
            ref = orc.mart_run(q, ref, 1, step0=k)
            assert rel_l2(got, one) < 1e-6, (k, rel_l2(got, one))
            assert rel_l2(got, ref) < 1e-6, (k, rel_l2(got, ref))
            prev = got
        st = sim.stats()
    finally:
        sim.close()
    rs = orc.mart_stats(q, ref)
    for k in ("e_el", "e_tot"):
        assert abs(st[k] - rs[k]) <= 1e-3 * abs(rs[k]) + 1e-12, (k, st[k], rs[k])


def test_precipitate_256_matches_oracle(gb, orc):
    p = gb.precip3d_params(256, dtype=gb.GS_DTYPE_F32)
    c0 = gb.initial_c(p, 2).astype(np.float32)
    e0 = gb.initial_eta(p, 3, 0.01).astype(np.float32)
    sim = gb.Sim(p)
    try:
        sim.set_field("concentration", c0)
        sim.set_field("eta", e0)
        sim.step(1)
        c1, e1 = sim.concentration(np.float64), sim.eta(np.float64)
    finally:
        sim.close()
    q = p.copy()
    q.dtype = gb.GS_DTYPE_F64
    rc, re = orc.precip_run(q, c0.astype(np.float64), e0.astype(np.float64), 1)
    assert rel_l2(c1, rc) < 1e-6
    assert rel_l2(e1, re) < 1e-6
    m0 = c0.astype(np.float64).sum()
    assert abs(c1.sum() - m0) <= 1e-9 * abs(m0)
