"""Batched ensembles (gs_batch_*): every simulation of a batch against the
FP64 oracle run on its own, and the captured-graph replay against direct
stepping."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
F64, F32 = 1, 0


def mixed_params(gb, dtype):
    out = []
    rng = np.random.default_rng(5)
    for i in range(6):
        if i < 3:
            p = gb.mart2d_params(16, dtype=dtype)
            base = np.zeros((2, 3, 3))
            base[0, 0, 0], base[0, 1, 1], base[1, 0, 0], base[1, 1, 1] = 1, -1, -1, 1
        else:
            p = gb.mart3d_params(8, dtype=dtype, noise=0.0)
            p.nx, p.ny, p.nz = 8, 8, 16
            base = gb.tetragonal_eigenstrains(3, 1.0, -0.5)
        p.landau[0] = rng.uniform(0.1, 0.4)
        p.landau[1] = rng.uniform(2, 4)
        p.kappa = rng.uniform(0.5, 2)
        p.weight_elastic = 50.0
        p.set_eigenstrain(base * rng.uniform(0.01, 0.03))
        p.noise_amp = 1e-3
        p.seed = 100 + i
        p.sim_id = i
        out.append(p)
    return out


def test_batch_fp64_each_sim_matches_oracle(gb, orc):
    ps = mixed_params(gb, F64)
    b = gb.Batch(ps)
    assert b.groups() == 2
    etas = [gb.initial_eta(p, 20 + i, 0.5) for i, p in enumerate(ps)]
    for i, e in enumerate(etas):
        b.set_eta(i, e)
    b.step(3)
    for i, p in enumerate(ps):
        ref = orc.mart_run(p, etas[i], 3)
        assert rel_l2(b.eta(i), ref) < 1e-11, i
    st = b.stats(4)
    ref = orc.mart_stats(ps[4], orc.mart_run(ps[4], etas[4], 3))
    for k in ["mass", "e_el", "e_chem", "e_grad", "e_tot"]:
        assert abs(st[k] - ref[k]) <= 1e-10 * max(1.0, abs(ref[k])), k
    b.close()


@pytest.mark.parametrize("dtype", [F32, F64])
def test_batch_graph_replay_matches_direct(gb, dtype):
    """Direct launches, graph replay, groups on concurrent branches or one
    after another: the same bits."""
    ps = mixed_params(gb, dtype)
    etas = [gb.initial_eta(p, 40 + i, 0.4) for i, p in enumerate(ps)]
    outs = []
    for graph, conc in ((False, False), (True, True), (False, True), (True, False)):
        b = gb.Batch(ps)
        b.set_concurrent(conc)
        b.use_graph(graph)
        for i, e in enumerate(etas):
            b.set_eta(i, e)
        b.step(7)
        b.step(4)
        outs.append([b.eta(i) for i in range(len(ps))])
        b.close()
    for other in outs[1:]:
        for a, c in zip(outs[0], other):
            assert np.array_equal(a, c)


def test_ensemble_builder_shapes(gb):
    ps = gb.ensemble_params()
    assert len(ps) == 64
    shapes = [(p.nx, p.ny, p.nz, p.nvariants) for p in ps]
    assert shapes.count((128, 128, 1, 2)) == 32 and shapes.count((256, 256, 1, 2)) == 16
    assert shapes.count((64, 64, 64, 3)) == 12 and shapes.count((128, 128, 128, 3)) == 4
    assert sorted(p.seed for p in ps) == list(range(100, 164))
    b = gb.Batch(ps)
    assert b.groups() == 4
    b.step(2)
    assert np.isfinite(b.eta(63)).all()
    b.close()


def test_sharded_ensemble_equals_single_runs(gb):
    """Two ranks' shares, run one after the other on this GPU without a
    process group, give the same statistics as each simulation alone."""
    import gs_dist

    ps = gb.ensemble_params(gb.GS_DTYPE_F64, counts=(3, 1, 2, 0))
    for p in ps:
        p.nx, p.ny = min(p.nx, 32), min(p.ny, 32)
        if p.nz > 1:
            p.nz = 16
    eta0 = [gb.initial_eta(p, 40 + i, 0.3) for i, p in enumerate(ps)]
    got = {}
    for rank in range(2):
        got.update(gs_dist.run_ensemble_shard(ps, eta0, rank, 2, 3, use_graph=False, gather=False))
    assert sorted(got) == list(range(len(ps)))
    for i, p in enumerate(ps):
        s = gb.Sim(p)
        try:
            s.set_field("eta", eta0[i])
            s.step(3)
            ref = s.stats()
        finally:
            s.close()
        for k in ("mass", "e_el", "e_tot"):
            assert abs(got[i][k] - ref[k]) <= 1e-10 * abs(ref[k]) + 1e-14, (i, k)
