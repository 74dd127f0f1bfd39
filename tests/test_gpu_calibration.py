"""Calibration through the torch.autograd bridge (gs_torch) over the
hand-written adjoint: autograd gradients equal the adjoint's, a few
optimiser steps lower the loss, and on the full calibration workload (96^3,
3 variants, 200 steps, checkpoint every 20, noise off) the FP64 gradients
match FP64 central differences (h = 1e-6, relative error <= 1e-3) and the
FP32 gradients match the FP64 ones to 1e-3."""
import numpy as np
import pytest
import torch

import gs_torch as gt

pytestmark = pytest.mark.gpu

F64, F32 = 1, 0
LAM = 0.1


def _loss(run, theta, eta0, target, e_target):
    eT, e = gt.martensite_run(eta0, theta, run)
    return gt.calibration_loss(eT, e, torch.as_tensor(target), e_target, LAM)


def test_autograd_equals_adjoint(gb):
    run, th0, eta0, target, et = gt.calibration_setup(n=16, nsteps=10, dtype=F64, checkpoint_every=4)
    try:
        theta = th0.clone().requires_grad_(True)
        e0 = torch.from_numpy(eta0).requires_grad_(True)
        loss = _loss(run, theta, e0, target, et)
        loss.backward()
        a = run.adj
        a.set_params(run.params_for(th0))
        a.set_loss(target, LAM, et)
        a.forward(eta0)
        lo, g, ge = a.backward()
        assert abs(loss.item() - lo[0]) <= 1e-12 * abs(lo[0])
        gm = g.copy()
        gm[5] /= float(th0[5])
        assert np.allclose(theta.grad.numpy(), gm, rtol=1e-10, atol=0)
        assert np.allclose(e0.grad.numpy(), ge, rtol=1e-10, atol=1e-300)
    finally:
        run.close()


def test_calibration_lowers_loss(gb):
    run, th0, eta0, target, et = gt.calibration_setup(n=16, nsteps=20, dtype=F32, checkpoint_every=5)
    try:
        theta = th0.clone().requires_grad_(True)
        e0 = torch.from_numpy(eta0)
        opt = torch.optim.Adam([theta], lr=0.01)
        losses = []
        for _ in range(6):
            opt.zero_grad()
            loss = _loss(run, theta, e0, target, et)
            loss.backward()
            opt.step()
            losses.append(loss.item())
        assert losses[-1] < losses[0]
    finally:
        run.close()


@pytest.fixture(scope="module")
def full64():
    run, th0, eta0, target, et = gt.calibration_setup(n=96, nsteps=200, dtype=F64, checkpoint_every=20)
    yield run, th0, eta0, target, et
    run.close()


def _adjoint_grads(run, th, eta0, target, et):
    a = run.adj
    a.set_params(run.params_for(th))
    a.set_loss(target, LAM, et)
    a.forward(eta0)
    lo, g, ge = a.backward()
    gm = g.copy()
    gm[5] /= float(th[5])
    return lo, gm, ge


def _fwd(run, th, eta0):
    run.adj.set_params(run.params_for(th))
    return run.adj.forward(eta0)


def _central_difference(run, plus, minus, target, et, h):
    """(J(+h) - J(-h)) / 2h, with the difference of the two losses formed
    per cell as (a - b)(a + b - 2 target): J is a sum of ~10^6 terms whose
    total dwarfs the change, so subtracting two rounded totals would lose
    the small gradients (A6, Ac) to cancellation."""
    (a, ea), (b, eb) = plus, minus
    d = ((a - b) * (a + b - 2 * target)).sum() + LAM * (ea - eb) * (ea + eb - 2 * et)
    return d / (2 * h)


def test_full_workload_f64_gradients_match_central_differences(full64):
    run, th0, eta0, target, et = full64
    lo, g, ge = _adjoint_grads(run, th0, eta0, target, et)
    h = 1e-6
    for k in range(6):
        tp, tm = th0.clone(), th0.clone()
        tp[k] += h
        tm[k] -= h
        fd = _central_difference(run, _fwd(run, tp, eta0), _fwd(run, tm, eta0), target, et, h)
        assert abs(g[k] - fd) <= 1e-3 * abs(fd), (k, g[k], fd)
    d = np.random.default_rng(7).standard_normal(eta0.shape)
    fd = _central_difference(run, _fwd(run, th0, eta0 + h * d), _fwd(run, th0, eta0 - h * d), target, et, h)
    assert abs((ge * d).sum() - fd) <= 1e-3 * abs(fd)


def test_full_workload_f32_gradients_match_f64(full64):
    run64, th0, eta0, target, et = full64
    _, g64, ge64 = _adjoint_grads(run64, th0, eta0, target, et)
    run32, _, _, _, _ = gt.calibration_setup(n=96, nsteps=200, dtype=F32, checkpoint_every=20)
    try:
        _, g32, ge32 = _adjoint_grads(run32, th0, eta0, target, et)
    finally:
        run32.close()
    assert np.all(np.abs(g32 - g64) <= 1e-3 * np.abs(g64)), (g32, g64)
    assert np.linalg.norm(ge32 - ge64) <= 1e-3 * np.linalg.norm(ge64)
