"""A thin torch.autograd.Function over the C ABI's objective and adjoint, used only by the
gradient tests: torch's autograd sees J(c0, g_y, sigma, M) as one node whose backward is
clipb_adjoint.  Checked against the tangent-linear model along a random direction."""
import numpy as np
import pytest
import torch

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu

STEPS = 120


class CentroidObjective(torch.autograd.Function):
    """J = |centroid(c_N) - target|^2 of the FP64 forward from c0 with parameters
    theta = (g_y, sigma, M); backward by the hand-written adjoint."""

    @staticmethod
    def forward(ctx, c0, theta, solver, target):
        th = theta.detach().cpu().numpy()
        solver.set_params(*th)
        J, g0, gp = solver.adjoint(STEPS, target, c0.detach().cpu().numpy(), checkpoint_every=40)
        ctx.save_for_backward(torch.from_numpy(g0), torch.from_numpy(gp))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        g0, gp = ctx.saved_tensors
        return grad_out * g0, grad_out * gp, None, None


def test_autograd_gradient_matches_tangent_linear():
    s = cb.Solver(golden_config("drop2d_small"), "fp64")
    c0 = s.initial_condition()
    p = s.params()
    theta0 = np.array([p["gy"], p["sigma"], p["mobility"]])
    target = np.array([14.0, 20.0])
    c0_t = torch.tensor(c0, requires_grad=True)
    th_t = torch.tensor(theta0, requires_grad=True)
    J = CentroidObjective.apply(c0_t, th_t, s, target)
    J.backward()
    rng = np.random.default_rng(5)
    d = rng.standard_normal(c0.shape)
    for _ in range(3):
        d = (d + np.roll(d, 1, 0) + np.roll(d, -1, 0) + np.roll(d, 1, 1) + np.roll(d, -1, 1)) / 5.0
    d *= 1e-2 / np.abs(d).max()
    dp = np.array([0.1, -0.3, 0.2]) * theta0
    s.set_params(*theta0)
    Jt, dJ = s.tangent(STEPS, target, c0, d, dp)
    assert Jt == J.item()
    via_autograd = float((c0_t.grad.numpy() * d).sum() + th_t.grad.numpy() @ dp)
    assert abs(via_autograd - dJ) <= 1e-9 * abs(dJ)
    s.close()
