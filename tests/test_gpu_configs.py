"""The five workloads of the step checked at their stated lengths and sizes,
through the C ABI, against the FP64 oracle:

* the 2D FP64 square-to-rectangle martensite (128^2, 2 variants) for all
  1000 steps, fields and statistics compared every 100 steps;
* members of the 64-simulation FP32 ensemble at their real sizes (128^2,
  256^2, 64^3, 128^3), advanced inside the whole batch with the tuned
  schedule, graph replay and noise on: 1e-6 relative L2 for every step
  (each step restarted in the oracle from the device's state) and for the
  accumulated run, statistics within 1e-3;
* the Philox4x32-10 stream: the words the kernels draw equal the oracle's
  bit for bit (counters near 2^32, 64-bit seeds), and a noise-only step
  writes exactly those normals;
* the 256^3 precipitate for 10000 steps: relative mass drift at most 1e-10;
* the headline martensite's own coefficients at 64^3, noise off, 1000 FP32
  steps within 1e-4 relative L2 of the FP64 oracle.

Tolerances are those of the accuracy bar of the step: FP32 fields 1e-6
relative L2 per step and 1e-4 after 1000 steps, statistics 1e-3; FP64
against FP64 agrees to round-off (1e-10 after 1000 steps)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
F64, F32 = 1, 0


def _as_f64(p):
    q = p.copy()
    q.dtype = F64
    return q


def test_config1_2d_fp64_full_length_with_statistics(gb, orc):
    """2D 128^2, 2 variants, FP64, 1000 explicit steps, noise off; the field
    and the statistics (volume fractions, elastic and total energy) every
    100 steps."""
    p = gb.mart2d_params(128, dtype=F64)
    eta0 = gb.initial_eta(p, 0, 0.01)
    sim = gb.Sim(p)
    ref = eta0.copy()
    try:
        sim.set_field("eta", eta0)
        for k in range(10):
            sim.step(100)
            got = sim.eta(np.float64)
            st = sim.stats()
            ref = orc.mart_run(p, ref, 100, step0=100 * k)
            rs = orc.mart_stats(p, ref)
            assert rel_l2(got, ref) < 1e-10, (k, rel_l2(got, ref))
            for key in ("e_el", "e_chem", "e_grad", "e_tot", "mass"):
                assert abs(st[key] - rs[key]) <= 1e-9 * abs(rs[key]) + 1e-18, (k, key, st[key], rs[key])
            assert st["vf"] == rs["vf"], k
            assert np.allclose(st["eta2"], rs["eta2"], rtol=1e-9, atol=0), k
    finally:
        sim.close()
    assert rel_l2(ref, eta0) > 0.1  # the run moved the field


ENSEMBLE_PICKS = (0, 32, 48, 60)  # one simulation of each shape: 128^2, 256^2, 64^3, 128^3


def test_config4_ensemble_members_fp32_match_oracle(gb, orc):
    ps = gb.ensemble_params(gb.GS_DTYPE_F32)
    b = gb.Batch(ps)
    try:
        etas = [gb.initial_eta(p, 200 + i).astype(np.float32) for i, p in enumerate(ps)]
        for i, e in enumerate(etas):
            b.set_eta(i, e)
        b.autotune(reps=2)
        b.use_graph(True)
        prev = {i: etas[i].astype(np.float64) for i in ENSEMBLE_PICKS}
        acc = dict(prev)
        steps = 3
        for k in range(steps):
            b.step(1)
            for i in ENSEMBLE_PICKS:
                q = _as_f64(ps[i])
                got = b.eta(i)
                one = orc.mart_run(q, prev[i], 1, step0=k)
                acc[i] = orc.mart_run(q, acc[i], 1, step0=k)
                assert rel_l2(got, one) < 1e-6, (i, k, rel_l2(got, one))
                assert rel_l2(got, acc[i]) < 1e-6, (i, k, rel_l2(got, acc[i]))
                prev[i] = got
        for i in ENSEMBLE_PICKS:
            st = b.stats(i)
            rs = orc.mart_stats(_as_f64(ps[i]), acc[i])
            for key in ("e_el", "e_chem", "e_grad", "e_tot"):
                assert abs(st[key] - rs[key]) <= 1e-3 * abs(rs[key]) + 1e-12, (i, key, st[key], rs[key])
            assert np.allclose(st["eta2"], rs["eta2"], rtol=1e-3, atol=0), i
            assert np.allclose(st["vf"], rs["vf"], atol=1e-3), i
    finally:
        b.close()


# ---------------------------------------------------------------------------
# the noise stream
# ---------------------------------------------------------------------------
def _noise_block(gb, seed, step, sim, slot, quad0, nq, dtype):
    words = np.zeros(4 * nq, dtype=np.uint32)
    normals = np.zeros(4 * nq, dtype=np.float64 if dtype == F64 else np.float32)
    rc = gb.lib().gs_noise_block(seed, step, sim, slot, quad0, nq, dtype, words.ctypes.data, normals.ctypes.data)
    assert rc == gb.GS_OK, gb.last_error()
    return words.reshape(nq, 4), normals.reshape(nq, 4)


NOISE_CASES = [  # (seed, step, sim, slot, first quad)
    (1, 0, 0, 0, 0),
    (0x123456789ABC, 7, 3, 2, 1000),
    (0xFFFFFFFFFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 8, 0xFFFFFFFF - 300),  # the quad word wraps past 2^32
    (163, 1999, 63, 1, (1 << 32) - 64),
    (2 ** 40 + 5, 123456789, 17, 4, 0x80000000),
]


@pytest.mark.parametrize("case", NOISE_CASES)
def test_philox_words_bit_exact_with_oracle(gb, orc, case):
    seed, step, sim, slot, quad0 = case
    nq = 600
    words, n64 = _noise_block(gb, seed, step, sim, slot, quad0, nq, F64)
    key = (seed & 0xFFFFFFFF, seed >> 32)
    ref = np.array([orc.philox(((quad0 + q) & 0xFFFFFFFF, step, sim, slot), key) for q in range(nq)], dtype=np.uint32)
    assert np.array_equal(words, ref)
    # the normals: the oracle's Box-Muller in FP64 (libm), the device's FP64
    # within round-off, FP32 within the error of its hardware sine/cosine
    zref = np.array([orc.normals4(seed, (quad0 + q) & 0xFFFFFFFF, step, sim, slot) for q in range(nq)])
    assert np.max(np.abs(n64 - zref)) < 1e-13
    _, n32 = _noise_block(gb, seed, step, sim, slot, quad0, nq, F32)
    assert np.max(np.abs(n32.astype(np.float64) - zref)) < 2e-5


def test_philox_known_answers_on_device(gb):
    """Random123's published known-answer vectors of Philox4x32-10, evaluated
    by the device function the kernels inline (counter = (quad, step, sim,
    slot), key = (seed lo, seed hi))."""
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        seed = key[0] | (key[1] << 32)
        w, _ = _noise_block(gb, seed, ctr[1], ctr[2], ctr[3], ctr[0], 1, F64)
        assert tuple(int(x) for x in w[0]) == want


@pytest.mark.parametrize("dtype", [F64, F32])
def test_noise_only_step_writes_the_checked_stream(gb, dtype):
    """From eta = 0 every deterministic term of the step vanishes (each is a
    multiple of eta), so one step with noise amplitude 1 writes the normals
    themselves: they must equal gs_noise_block's bit for bit, which ties the
    stream checked above to the one the update kernel draws."""
    p = gb.mart3d_params(16, dtype=dtype, noise=1.0)
    p.nx, p.ny, p.nz = 8, 12, 16
    p.seed = 0xDEADBEEF12345
    p.sim_id = 5
    V, N = p.nvariants, p.ncells
    s = gb.Sim(p)
    try:
        s.set_field("eta", np.zeros((V, p.nx, p.ny, p.nz)))
        s.set_scalar("step", 41)
        s.step(1)
        got = s.eta(np.float64 if dtype == F64 else np.float32).reshape(V, N)
    finally:
        s.close()
    for v in range(V):
        _, z = _noise_block(gb, p.seed, 41, 5, v, 0, N // 4, dtype)
        assert np.array_equal(got[v], z.reshape(N)), v


# ---------------------------------------------------------------------------
# long runs
# ---------------------------------------------------------------------------
def test_config3_precipitate_256_mass_drift_10000_steps(gb):
    """The precipitate workload at its size and length: 256^3, concentration
    + 4 variants, FP32, 10000 semi-implicit steps; the FP64 sum of the
    stored concentration stays within 1e-10 relative of its initial value."""
    p = gb.precip3d_params(256, dtype=F32)
    c0 = gb.initial_c(p, 2).astype(np.float32)
    e0 = gb.initial_eta(p, 3, 0.01).astype(np.float32)
    m0 = c0.astype(np.float64).sum()
    sim = gb.Sim(p)
    drifts = []
    try:
        sim.set_field("concentration", c0)
        sim.set_field("eta", e0)
        for _ in range(10):
            sim.step(1000)
            drifts.append(abs(sim.stats()["mass"] - m0) / abs(m0))
        c = sim.concentration(np.float64)
        e = sim.eta(np.float64)
    finally:
        sim.close()
    assert np.isfinite(c).all() and np.isfinite(e).all()
    assert rel_l2(c, c0.astype(np.float64)) > 1e-3  # the concentration moved
    assert max(drifts) <= 1e-10, drifts


def test_headline_coefficients_fp32_1000_steps_within_1e4(gb, orc):
    """The headline martensite's own coefficients (A2=0.2, A4=3, A6=2, A_c=1,
    kappa=0.5, tetragonal eigenstrains 0.02/-0.01, C11/C12/C44 =
    1.4/0.84/0.56, sigma_zz=0.005, dt=0.005) at 64^3, noise off, 1000 FP32
    steps against the FP64 oracle."""
    p = gb.mart3d_params(64, dtype=F32, noise=0.0)
    eta0 = gb.initial_eta(p, 1).astype(np.float32).astype(np.float64)
    ref = orc.mart_run(_as_f64(p), eta0, 1000)
    sim = gb.Sim(p)
    try:
        sim.set_field("eta", eta0.astype(np.float32))
        sim.step(1000)
        got = sim.eta(np.float64)
    finally:
        sim.close()
    assert rel_l2(ref, eta0) > 1e-2  # the run moved the field
    assert rel_l2(got, ref) < 1e-4, rel_l2(got, ref)
