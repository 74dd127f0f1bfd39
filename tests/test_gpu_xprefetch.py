"""The TMA-fed x pass (persistent blocks that fetch their next column tile
while they transform the current one) against the one-tile-per-block x
pass: the same arithmetic, so the fields must agree bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(gb, p, eta0, steps, prefetch, graph=False):
    gb.lib().gs_set_x_prefetch(1 if prefetch else 0)
    try:
        sim = gb.Sim(p)
        try:
            sim.set_field("eta", eta0)
            sim.use_graph(graph)
            sim.step(steps)
            return sim.eta(), sim.stats()
        finally:
            sim.close()
    finally:
        gb.lib().gs_set_x_prefetch(0)  # the library's default


@pytest.mark.parametrize("n,noise,graph", [(128, 1e-3, False), (256, 0.0, False), (128, 0.0, True)])
def test_prefetched_x_pass_bits_equal_plain(gb, n, noise, graph):
    p = gb.mart3d_params(n, dtype=gb.GS_DTYPE_F32, noise=noise)
    eta0 = gb.initial_eta(p, 3, 0.3).astype(np.float32)
    t0 = gb.lib().gs_x_prefetch_timeouts()
    a, sa = run(gb, p, eta0, 4, True, graph)
    b, sb = run(gb, p, eta0, 4, False, graph)
    assert gb.lib().gs_x_prefetch_timeouts() == t0
    assert np.array_equal(a, b)
    assert sa["e_el"] == sb["e_el"]
    assert np.abs(a - eta0).max() > 0  # the steps did move the field


def test_prefetched_x_pass_rectangular(gb):
    """n0 = 256 with n1 != n2 (tiles of other widths and counts)."""
    p = gb.mart3d_params(16, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    p.nx, p.ny, p.nz = 256, 32, 48
    eta0 = gb.initial_eta(p, 5, 0.3).astype(np.float32)
    a, _ = run(gb, p, eta0, 3, True)
    b, _ = run(gb, p, eta0, 3, False)
    assert np.array_equal(a, b)


def test_prefetched_x_pass_precipitate_bits_equal_plain(gb):
    """Five fields (four variants and the concentration) in the elastic
    chain of the precipitate step."""
    p = gb.precip3d_params(128, dtype=gb.GS_DTYPE_F32)
    c0 = gb.initial_c(p, 2)
    e0 = gb.initial_eta(p, 3, 0.3)
    out = []
    for on in (1, 0):
        gb.lib().gs_set_x_prefetch(on)
        try:
            sim = gb.Sim(p)
            try:
                sim.set_field("concentration", c0)
                sim.set_field("eta", e0)
                sim.step(3)
                out.append((sim.eta(np.float32), sim.concentration(np.float32)))
            finally:
                sim.close()
        finally:
            gb.lib().gs_set_x_prefetch(0)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
