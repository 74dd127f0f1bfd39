"""The schedule autotuner: tuning leaves the state untouched; every tile
schedule gives the same bits (lines, columns and rows are independent); the
alternative radix split of the y lines rounds differently but meets the
oracle's tolerances (FP64 1e-11, FP32 1e-6 per step); tuned batches match
their untuned results within those tolerances."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

F64, F32 = 1, 0


def _params(gb, shape, dtype=F32, V=3):
    p = gb.mart3d_params(16, dtype=dtype, noise=1e-3)
    p.nx, p.ny, p.nz = shape
    if V != 3:
        p.nvariants = V
        p.set_eigenstrain(gb.tetragonal_eigenstrains(V, 0.02, -0.01))
    return p


def _run(gb, p, eta0, steps, tune=False, sched=None):
    s = gb.Sim(p)
    try:
        s.set_field("eta", eta0)
        chosen = None
        if tune:
            chosen = s.autotune(reps=2)
        if sched:
            s.set_schedule(**sched)
        s.step(steps)
        return s.eta(np.float64), chosen
    finally:
        s.close()


@pytest.mark.parametrize("shape", [(32, 32, 32), (1, 48, 64), (16, 24, 96)])
def test_autotune_keeps_state_and_bits(gb, shape):
    p = _params(gb, shape)
    eta0 = gb.initial_eta(p, 3, 0.2)
    ref, _ = _run(gb, p, eta0, 3)
    got, chosen = _run(gb, p, eta0, 3, tune=True)
    assert set(chosen) == {"z_lines", "y_cols", "x_cols", "update_rows", "y_radix"}
    assert all(v >= 0 for v in chosen.values())
    # tuning left the state as it was: the same bits as the chosen schedule set directly
    again, _ = _run(gb, p, eta0, 3, sched=chosen)
    assert np.array_equal(got, again)
    if chosen["y_radix"] == 0:
        assert np.array_equal(got, ref)
    else:
        assert rel_l2(got, ref) < 3e-6


@pytest.mark.parametrize("sched", [dict(z_lines=1, y_cols=1, x_cols=1, update_rows=1),
                                   dict(z_lines=64, y_cols=32, x_cols=32, update_rows=64),
                                   dict(z_lines=3, y_cols=3, x_cols=6, update_rows=5)])
def test_any_schedule_gives_the_same_bits(gb, sched):
    p = _params(gb, (16, 32, 64), dtype=F64, V=4)
    eta0 = gb.initial_eta(p, 4, 0.3)
    ref, _ = _run(gb, p, eta0, 2)
    got, _ = _run(gb, p, eta0, 2, sched=sched)
    assert np.array_equal(got, ref)


def test_batch_autotune_matches_untuned(gb):
    ps = gb.ensemble_params(gb.GS_DTYPE_F32, counts=(3, 2, 2, 1))
    eta0 = [gb.initial_eta(p, 60 + i).astype(np.float32) for i, p in enumerate(ps)]

    def run(tune):
        b = gb.Batch(ps)
        try:
            for i in range(len(ps)):
                b.set_eta(i, eta0[i])
            b.use_graph(True)
            b.step(2)
            scheds = b.autotune(reps=2) if tune else None
            b.step(4)
            return [b.eta(i) for i in range(len(ps))], scheds
        finally:
            b.close()

    ref, _ = run(False)
    got, scheds = run(True)
    assert len(scheds) == 4
    for a, r, sc in zip(got, ref, [None] * len(ref)):
        assert rel_l2(a, r) < 6e-6  # six FP32 steps; bit-equal unless a group chose the other y radix
    if all(sc["y_radix"] == 0 for sc in scheds):
        for a, r in zip(got, ref):
            assert np.array_equal(a, r)


@pytest.mark.parametrize("shape", [(8, 64, 16), (4, 128, 32), (2, 256, 8), (16, 256, 64)])
@pytest.mark.parametrize("dtype,tol", [(F64, 1e-11), (F32, 1e-6)])
def test_alternative_y_radix_matches_oracle(gb, orc, shape, dtype, tol):
    p = _params(gb, shape, dtype=dtype)
    eta0 = gb.initial_eta(p, 5, 0.4)
    if dtype == F32:
        eta0 = eta0.astype(np.float32).astype(np.float64)
    alt = {64: 16, 128: 32, 256: 32}[shape[1]]
    got, _ = _run(gb, p, eta0, 1, sched=dict(y_radix=alt))
    assert rel_l2(got, orc.mart_run(p, eta0, 1)) < tol


def test_bad_y_radix_rejected(gb):
    p = _params(gb, (8, 64, 16))
    s = gb.Sim(p)
    try:
        with pytest.raises(RuntimeError):
            s.set_schedule(y_radix=8)
    finally:
        s.close()


def test_precipitate_autotune_keeps_state_and_bits(gb):
    """Tuning a precipitate simulation runs trial steps on a copy of its
    state; the steps after it match an untuned run bit for bit."""
    p = gb.precip3d_params(32, dtype=F32)
    c0 = gb.initial_c(p, 2)
    e0 = gb.initial_eta(p, 3, 0.3)
    out = []
    for tune in (False, True):
        s = gb.Sim(p)
        try:
            s.set_field("concentration", c0)
            s.set_field("eta", e0)
            s.step(2)
            if tune:
                chosen = s.autotune(reps=2)
                assert all(v >= 0 for v in chosen.values())
            s.step(3)
            out.append((s.concentration(np.float32), s.eta(np.float32)))
        finally:
            s.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
