"""The hand-written adjoint of the precipitate run (gs_precip_adjoint_*,
through the C ABI) against the FP64 oracle adjoint and central differences.

Tolerances: FP64 gradients agree with the oracle adjoint to 1e-9 relative
(different FFT algorithms; an entry far below the largest is held to 1e-12 of
the largest); FP32 gradients to 1e-3 relative; central differences of the
FP64 GPU forward with h = 1e-6 to 1e-5 relative."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

F64, F32 = 1, 0


def setup(gb, shape, V=4, dtype=F64, noise=0.0, c_elastic=1, seed=2):
    p = gb.precip3d_params(8, dtype=dtype)
    p.nx, p.ny, p.nz = shape
    p.nvariants = V
    p.noise_amp = noise
    p.c_elastic = c_elastic
    c0 = gb.initial_c(p, seed)
    e0 = gb.initial_eta(p, seed + 1, 0.4)
    rng = np.random.default_rng(seed)
    return p, c0, e0, rng.standard_normal(c0.shape), rng.standard_normal(e0.shape)


def gpu_adjoint(gb, p, c0, e0, ns, sc, se, K=1):
    a = gb.PrecipAdjoint(p, ns, K)
    try:
        cT, eT = a.forward(c0, e0)
        g, gc, ge = a.backward(sc, se)
        return g, gc, ge, cT, eT
    finally:
        a.close()


def close_vec(g, og, rtol):
    g, og = np.asarray(g), np.asarray(og)
    return np.all(np.abs(g - og) <= rtol * np.abs(og) + 1e-12 * np.abs(og).max())


@pytest.mark.parametrize("shape,V,ns,noise,ce,K", [
    ((6, 8, 4), 4, 3, 0.0, 1, 1),
    ((8, 8, 12), 3, 4, 1e-3, 1, 3),
    ((8, 12, 2), 2, 5, 0.0, 0, 2),
    ((1, 16, 24), 2, 4, 1e-3, 1, 4),
    ((8, 8, 8), 4, 7, 1e-3, 1, 3),
])
def test_precip_adjoint_f64_matches_oracle(gb, orc, shape, V, ns, noise, ce, K):
    """K: a checkpoint every K steps, the other states recomputed."""
    p, c0, e0, sc, se = setup(gb, shape, V, F64, noise, ce)
    g, gc, ge, cT, eT = gpu_adjoint(gb, p, c0, e0, ns, sc, se, K)
    og, ogc, oge = orc.precip_adjoint(p, c0, e0, ns, sc, se)
    oc, oe = orc.precip_run(p, c0, e0, ns)
    assert rel_l2(cT, oc) < 1e-11 and rel_l2(eT, oe) < 1e-11
    assert close_vec(g, og, 1e-9), (g, og)
    assert rel_l2(gc, ogc) < 1e-10
    assert rel_l2(ge, oge) < 1e-10


def test_precip_adjoint_f64_matches_central_differences(gb):
    """Directional derivatives of the GPU forward run against the GPU
    adjoint: independent of the oracle."""
    p, c0, e0, sc, se = setup(gb, (8, 8, 8), 3, F64, 0.0, 1, seed=7)
    ns, h = 4, 1e-6
    g, gc, ge, _, _ = gpu_adjoint(gb, p, c0, e0, ns, sc, se)

    def J(q, c=c0, e=e0):
        a = gb.PrecipAdjoint(q, ns)
        try:
            cc, ee = a.forward(c, e)
        finally:
            a.close()
        return (sc * cc).sum() + (se * ee).sum()

    for k in (0, 1, 2, 3, 4):
        q1, q2 = p.copy(), p.copy()
        if k == 0:
            q1.kappa_c += h
            q2.kappa_c -= h
        elif k == 1:
            q1.kappa_eta += h
            q2.kappa_eta -= h
        else:
            q1.coef[k - 1] += h
            q2.coef[k - 1] -= h
        fd = (J(q1) - J(q2)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-5 * abs(fd) + 1e-10, (k, g[k], fd)
    rng = np.random.default_rng(3)
    d = rng.standard_normal(c0.shape)
    fd = (J(p, c0 + h * d) - J(p, c0 - h * d)) / (2 * h)
    assert abs((gc * d).sum() - fd) <= 1e-6 * abs(fd)
    d = rng.standard_normal(e0.shape)
    fd = (J(p, c0, e0 + h * d) - J(p, c0, e0 - h * d)) / (2 * h)
    assert abs((ge * d).sum() - fd) <= 1e-6 * abs(fd)


def test_precip_adjoint_f32(gb, orc):
    p, c0, e0, sc, se = setup(gb, (16, 16, 16), 4, F32, 0.0, 1, seed=11)
    g, gc, ge, _, _ = gpu_adjoint(gb, p, c0, e0, 3, sc, se)
    q = p.copy()
    q.dtype = F64
    og, ogc, oge = orc.precip_adjoint(q, c0, e0, 3, sc, se)
    big = np.abs(og) > 1e-3 * np.abs(og).max()
    assert np.all(np.abs(g - og)[big] <= 1e-3 * np.abs(og)[big]), (g, og)
    assert rel_l2(gc, ogc) < 1e-4
    assert rel_l2(ge, oge) < 1e-4


def test_precip_adjoint_rejects(gb):
    p = gb.mart3d_params(8, dtype=F64)
    with pytest.raises(RuntimeError):
        gb.PrecipAdjoint(p, 2)
    q = gb.precip3d_params(8, dtype=F64)
    with pytest.raises(RuntimeError):
        gb.PrecipAdjoint(q, 0)
    with pytest.raises(RuntimeError):
        gb.PrecipAdjoint(q, 3, 4)  # a checkpoint spacing beyond the run
    with pytest.raises(RuntimeError):
        gb.PrecipAdjoint(q, 3, 0)
    a = gb.PrecipAdjoint(q, 2)
    try:
        c0 = np.zeros((8, 8, 8))
        with pytest.raises(RuntimeError):
            a.backward(c0, np.zeros((4, 8, 8, 8)))
        assert a.device_bytes() >= 8 * 512 * 5 * 3
    finally:
        a.close()


def test_precip_adjoint_replay(gb):
    """A second forward from the kept initial state and a second backward
    with the kept seeds reproduce the first results bit for bit."""
    p, c0, e0, sc, se = setup(gb, (8, 8, 12), 3, F32, 1e-3, 1, seed=5)
    a = gb.PrecipAdjoint(p, 4)
    try:
        cT, eT = a.forward(c0, e0)
        g, gc, ge = a.backward(sc, se)
        assert a.forward(outputs=False) is None
        g2, gc2, ge2 = a.backward()
        cT2, eT2 = a.forward()
        g3, _, _ = a.backward(outputs=False)
    finally:
        a.close()
    assert np.array_equal(cT, cT2) and np.array_equal(eT, eT2)
    assert np.array_equal(g, g2) and np.array_equal(g, g3)
    assert np.array_equal(gc, gc2) and np.array_equal(ge, ge2)


@pytest.mark.parametrize("dtype", [F32, F64])
def test_precip_adjoint_checkpoints_and_graph_give_the_same_bits(gb, dtype):
    """Every checkpoint spacing recomputes the same states (the forward's
    step counters, noise on), so the gradients equal those of the run that
    keeps every state bit for bit; the captured reverse sweep equals the
    direct one; repeated sweeps (the last segment recomputed first) too."""
    p, c0, e0, sc, se = setup(gb, (8, 8, 12), 3, dtype, 1e-3, 1, seed=9)
    ns = 7
    ref = None
    for K in (1, 2, 3, 7):
        for graph in (False, True):
            a = gb.PrecipAdjoint(p, ns, K)
            try:
                a.use_graph(graph)
                a.forward(c0, e0)
                outs = [a.backward(sc, se) for _ in range(3)]  # the third replays the captured graph
                nbytes = a.device_bytes()
            finally:
                a.close()
            for g, gc, ge in outs:
                assert np.isfinite(g).all()
                if ref is None:
                    ref = (g, gc, ge, nbytes)
                assert np.array_equal(g, ref[0]) and np.array_equal(gc, ref[1]) and np.array_equal(ge, ref[2]), (K, graph)
            if K in (2, 3):  # (ceil(7 / K) + 1) + (K - 1) kept states against 8
                assert nbytes < ref[3]


def test_precip_adjoint_graph_recaptured_for_a_new_initial_mass(gb, orc):
    """A forward from a new initial concentration changes the mass projection
    offset baked into the captured sweep: the sweep is captured again and the
    gradients follow the new run."""
    p, c0, e0, sc, se = setup(gb, (8, 8, 8), 3, F64, 0.0, 1, seed=13)
    ns = 4
    c1 = c0 + 0.01
    a = gb.PrecipAdjoint(p, ns, 2)
    try:
        a.forward(c0, e0)
        for _ in range(2):
            a.backward(sc, se)
        a.forward(c1, e0)
        g, gc, ge = a.backward(sc, se)
    finally:
        a.close()
    og, ogc, oge = orc.precip_adjoint(p, c1, e0, ns, sc, se)
    assert close_vec(g, og, 1e-9), (g, og)
    assert rel_l2(gc, ogc) < 1e-10 and rel_l2(ge, oge) < 1e-10
