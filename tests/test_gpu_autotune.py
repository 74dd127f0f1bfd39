"""The tile-schedule autotuner: tuning leaves the state untouched, every
schedule gives the same bits (lines, columns and rows are independent), and
tuned batches still match their untuned results."""
import numpy as np
import pytest

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
    assert set(chosen) == {"z_lines", "y_cols", "x_cols", "update_rows"}
    assert all(v >= 0 for v in chosen.values())
    assert np.array_equal(got, ref)


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
    for a, r in zip(got, ref):
        assert np.array_equal(a, r)


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
