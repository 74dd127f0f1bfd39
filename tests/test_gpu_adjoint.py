"""The hand-written adjoint of the martensite run (gs_adjoint_*, through the
C ABI) against the FP64 oracle adjoint and against central differences.

Tolerances: FP64 gradients agree with the oracle adjoint to 1e-9 relative
(different FFT algorithms); FP32 gradients to 1e-3 relative (the bar for
gradients); central differences of the FP64 GPU forward with h = 1e-6 to
1e-5 relative."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

F64, F32 = 1, 0


def setup(gb, shape, V=3, dtype=F64, noise=0.0, wel=200.0):
    p = gb.mart3d_params(16, dtype=dtype, noise=noise)
    p.nx, p.ny, p.nz = shape
    if V != 3:
        p.nvariants = V
        p.set_eigenstrain(gb.tetragonal_eigenstrains(V, 0.02, -0.01))
    p.weight_elastic = wel
    eta0 = gb.initial_eta(p, 4, 0.3)
    tgt = gb.initial_eta(p, 5, 0.3)
    return p, eta0, tgt


def gpu_adjoint(gb, p, eta0, tgt, ns, K, lam_el=0.1, et=0.0):
    a = gb.Adjoint(p, ns, K)
    try:
        a.set_loss(tgt, lam_el, et)
        eT, eel = a.forward(eta0)
        lo, g, ge = a.backward()
        return lo, g, ge, eT, eel
    finally:
        a.close()


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(np.asarray(b)), 1e-300)


@pytest.mark.parametrize("shape,V,ns,K,noise", [
    ((8, 8, 12), 3, 6, 4, 0.0),
    ((8, 8, 12), 3, 5, 5, 1e-3),
    ((1, 16, 24), 2, 7, 3, 0.0),
    ((6, 8, 4), 4, 4, 1, 1e-3),
])
def test_adjoint_f64_matches_oracle(gb, orc, shape, V, ns, K, noise):
    p, eta0, tgt = setup(gb, shape, V, F64, noise)
    lo, g, ge, eT, eel = gpu_adjoint(gb, p, eta0, tgt, ns, K)
    olo, og, oge = orc.mart_adjoint(p, eta0, ns, tgt, 0.1, 0.0)
    assert np.all(rel(lo, olo) < 1e-10), (lo, olo)
    assert np.all(rel(g, og) < 1e-9), (g, og)
    assert rel_l2(ge, oge) < 1e-10
    assert rel_l2(eT, orc.mart_run(p, eta0, ns)) < 1e-11


def test_adjoint_f32_matches_oracle(gb, orc):
    p, eta0, tgt = setup(gb, (16, 16, 16), 3, F32, 0.0)
    ns = 12
    lo, g, ge, _, _ = gpu_adjoint(gb, p, eta0, tgt, ns, 4)
    p64 = p.copy()
    p64.dtype = F64
    e32 = eta0.astype(np.float32).astype(np.float64)
    t32 = tgt.astype(np.float32).astype(np.float64)
    olo, og, oge = orc.mart_adjoint(p64, e32, ns, t32, 0.1, 0.0)
    assert np.all(rel(g, og) < 1e-3), (g, og)
    assert rel_l2(ge, oge) < 1e-4
    assert rel(lo[0], olo[0]) < 1e-5


def test_checkpoint_interval_does_not_change_result(gb):
    p, eta0, tgt = setup(gb, (8, 8, 12), 3, F64, 1e-3)
    ref = gpu_adjoint(gb, p, eta0, tgt, 9, 9)
    for K in (1, 2, 4):
        out = gpu_adjoint(gb, p, eta0, tgt, 9, K)
        assert np.array_equal(out[1], ref[1])
        assert np.array_equal(out[2], ref[2])


def test_seed_mode_equals_loss_mode(gb):
    p, eta0, tgt = setup(gb, (8, 8, 12), 3, F64, 0.0)
    ns, lam_el, et = 5, 0.1, 0.003
    a = gb.Adjoint(p, ns, 2)
    try:
        a.set_loss(tgt, lam_el, et)
        eT, eel = a.forward(eta0)
        lo, g, ge = a.backward()
        # the same J as a vector-Jacobian product: seed = dJ/deta_T, seed_e = dJ/dE_el
        lo2, g2, ge2 = a.backward(seed=2 * (eT - tgt), seed_e=2 * lam_el * (eel - et))
        assert np.allclose(g2, g, rtol=1e-12, atol=0)
        assert rel_l2(ge2, ge) < 1e-13
        # a second backward after the first (segments recomputed again)
        lo3, g3, ge3 = a.backward()
        assert np.array_equal(g3, g) and np.array_equal(ge3, ge)
    finally:
        a.close()


def test_adjoint_matches_central_differences_on_gpu(gb):
    """Central differences of the GPU FP64 forward loss (h = 1e-6)."""
    p, eta0, tgt = setup(gb, (8, 8, 12), 3, F64, 0.0)
    ns, K, lam_el, et, h = 6, 2, 0.1, 0.0, 1e-6
    lo, g, ge, _, _ = gpu_adjoint(gb, p, eta0, tgt, ns, K, lam_el, et)

    def loss(q, e0=eta0):
        a = gb.Adjoint(q, ns, K)
        try:
            eT, eel = a.forward(e0)
        finally:
            a.close()
        return ((eT - tgt) ** 2).sum() + lam_el * (eel - et) ** 2

    def with_param(k, scale):
        q = p.copy()
        if k == 0:
            q.kappa = p.kappa + scale
        elif k <= 4:
            q.landau[k - 1] = p.landau[k - 1] + scale
        else:
            q.set_eigenstrain(p.get_eigenstrain() * (1 + scale))
        return q

    for k in range(6):
        fd = (loss(with_param(k, h)) - loss(with_param(k, -h))) / (2 * h)
        assert abs(g[k] - fd) <= 1e-5 * abs(fd) + 1e-9, (k, g[k], fd)
    d = np.random.default_rng(2).standard_normal(eta0.shape)
    fd = (loss(p, eta0 + h * d) - loss(p, eta0 - h * d)) / (2 * h)
    assert abs((ge * d).sum() - fd) <= 1e-6 * abs(fd)


def test_adjoint_rejects_refcompat_and_bad_use(gb):
    p, eta0, tgt = setup(gb, (8, 8, 12), 3, F64, 0.0)
    q = p.copy()
    q.mode = gb.GS_MODE_REFCOMPAT
    with pytest.raises(gb.GsError):
        gb.Adjoint(q, 4, 2)
    a = gb.Adjoint(p, 4, 2)
    try:
        with pytest.raises(gb.GsError):
            a.backward()  # no forward yet
        a.forward(eta0)
        with pytest.raises(gb.GsError):
            a.backward()  # no loss and no seed
        assert a.device_bytes() > 0
    finally:
        a.close()


@pytest.mark.parametrize("dtype", [F64, F32])
def test_graph_replay_equals_direct_launches(gb, dtype):
    """Forward and backward replayed as captured graphs (after the first
    direct run) give the same bits as direct launches, across repeated
    runs, a second backward without a forward and new parameters."""
    p, eta0, tgt = setup(gb, (8, 8, 12), 3, dtype, 1e-3)
    eta1 = gb.initial_eta(p, 9, 0.3)

    def run(graph):
        a = gb.Adjoint(p, 7, 3)
        out = []
        try:
            a.use_graph(graph)
            a.set_loss(tgt, 0.1, 0.0)
            for e in (eta0, eta1, eta0):
                a.forward(e)
                out.append(a.backward())
            out.append(a.backward())  # no forward in between
            q = p.copy()
            q.kappa = 0.7
            a.set_params(q)
            for _ in range(2):
                a.forward(eta1)
                out.append(a.backward())
        finally:
            a.close()
        return out

    direct, graph = run(False), run(True)
    for (l0, g0, e0), (l1, g1, e1) in zip(direct, graph):
        assert np.array_equal(l0, l1) and np.array_equal(g0, g1) and np.array_equal(e0, e1)
