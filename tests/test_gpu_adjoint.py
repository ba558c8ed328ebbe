"""Tangent-linear model and adjoint of the FP64 2D step.

Objective J = |centroid(c_N) - target|^2.  Checks: the tangent-linear value and the
adjoint's forward equal the FP64 forward exactly; the adjoint gradient (initial c field and
(g_y, sigma, M)) against the tangent-linear directional derivative (1e-9 relative on the
drop, 1e-8 on the closed-box bubble) and against central finite differences of the FP64
forward.  The finite differences are limited by the forward's rounding: with eps = 1e-6
relative the quotient carries about 1e-4 relative noise for sigma and M on this small
case (it shrinks as 1/eps: 5e-7 at eps = 1e-4), so the parameter check uses eps = 1e-4
relative and the initial-field check eps = 1e-6 on a 1e-2 perturbation; both at the 1e-6
relative bar (1e-5 for the field).

The bubble is placed off the node lattice's symmetry points: where grad c vanishes
exactly the interface normal grad c / (|grad c| + 1e-32) of the reference's formulation
is not differentiable."""
import re

import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu

CASES = {"drop2d_small": 230, "bubble2d_walls": 150}
CENTERS = {"bubble2d_walls": (10.3, 12.6)}


def _config(name):
    text = open(golden_config(name)).read()
    if name in CENTERS:
        cx, cy = CENTERS[name]
        text = re.sub(r"center = \[[^\]]*\]", f"center = [{cx}, {cy}, 0]", text)
    import tempfile
    f = tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False)
    f.write(text)
    f.close()
    return f.name


def _setup(name):
    s = cb.Solver(_config(name), "fp64")
    c0 = s.initial_condition()
    steps = CASES[name]
    s.objective(steps, np.zeros(2), c0)  # centroid of the unperturbed run
    c = s.interior_field("c")[..., 0, 0]
    x = np.arange(1, c.shape[0] + 1)[:, None]
    y = np.arange(1, c.shape[1] + 1)[None, :]
    X = np.array([(x * c).sum() / c.sum(), (y * c).sum() / c.sum()])
    p = s.params()
    return s, c0, steps, X + np.array([3.0, 5.0]), np.array([p["gy"], p["sigma"], p["mobility"]])


def _smooth_direction(shape, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(shape)
    for _ in range(3):  # a few box-filter passes: a smooth perturbation of the interface
        d = (d + np.roll(d, 1, 0) + np.roll(d, -1, 0) + np.roll(d, 1, 1) + np.roll(d, -1, 1)) / 5.0
    return 1e-2 * d / np.abs(d).max()


@pytest.mark.parametrize("name", list(CASES))
def test_forward_values_agree(name):
    s, c0, steps, target, _ = _setup(name)
    J = s.objective(steps, target, c0)
    Jt, _ = s.tangent(steps, target, c0, np.zeros_like(c0), np.zeros(3))
    fwd = {f: s.field(f) for f in ("c", "p", "vel", "f", "g")}
    Ja, _, _ = s.adjoint(steps, target, c0, checkpoint_every=50)
    assert Jt == J and Ja == J
    # the adjoint leaves the solver at the end of its forward run
    assert s.steps == steps
    for f, v in fwd.items():
        np.testing.assert_array_equal(s.field(f), v, err_msg=f)
    s.close()


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_matches_tangent_linear(name):
    s, c0, steps, target, theta = _setup(name)
    _, gc0, gp = s.adjoint(steps, target, c0, checkpoint_every=50)
    dc0 = _smooth_direction(c0.shape, 1)
    dp = np.array([0.3, -0.2, 0.5]) * theta
    _, dJ_field = s.tangent(steps, target, c0, dc0, None)
    _, dJ_par = s.tangent(steps, target, c0, None, dp)
    tol = 1e-9 if name == "drop2d_small" else 1e-8
    assert abs(np.sum(gc0 * dc0) - dJ_field) <= tol * abs(dJ_field)
    assert abs(np.dot(gp, dp) - dJ_par) <= tol * abs(dJ_par)
    # each parameter on its own
    for i in range(3):
        e = np.zeros(3)
        e[i] = theta[i]
        _, dJ = s.tangent(steps, target, c0, None, e)
        assert abs(gp[i] * theta[i] - dJ) <= tol * abs(dJ) + 1e-300, i
    s.close()


def test_gradient_matches_central_differences():
    s, c0, steps, target, theta = _setup("drop2d_small")
    _, gc0, gp = s.adjoint(steps, target, c0, checkpoint_every=100)
    eps = 1e-4
    for i in range(3):
        h = eps * abs(theta[i])
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        s.set_params(*tp)
        Jp = s.objective(steps, target, c0)
        s.set_params(*tm)
        Jm = s.objective(steps, target, c0)
        s.set_params(*theta)
        fd = (Jp - Jm) / (2 * h)
        assert abs(gp[i] - fd) <= 1e-6 * abs(fd), (i, gp[i], fd)
    d = _smooth_direction(c0.shape, 2)
    eps = 1e-6
    Jp = s.objective(steps, target, c0 + eps * d)
    Jm = s.objective(steps, target, c0 - eps * d)
    fd = (Jp - Jm) / (2 * eps)
    assert abs(np.sum(gc0 * d) - fd) <= 1e-5 * abs(fd)
    s.close()


@pytest.mark.parametrize("every", [2, 7, 8, 230])
def test_checkpoint_interval_does_not_change_the_gradient(every):
    """Odd intervals run every segment with plain launches, even ones replay captured
    graphs for the middle segments (230 steps: 115, 33 and 29 segments); 230 and 1000
    keep the whole run in one tape.  The workspace of a call is reused by the next."""
    s, c0, steps, target, _ = _setup("drop2d_small")
    J1, g1, p1 = s.adjoint(steps, target, c0, checkpoint_every=every)
    J2, g2, p2 = s.adjoint(steps, target, c0, checkpoint_every=1000)
    J3, g3, p3 = s.adjoint(steps, target, c0, checkpoint_every=every)
    assert J1 == J2 == J3
    for a in (g1, g3):
        assert np.allclose(a, g2, rtol=1e-12, atol=1e-12 * np.abs(g2).max())
    for a in (p1, p3):
        assert np.allclose(a, p2, rtol=1e-12)
    s.close()


def test_derivative_paths_reject_other_cases():
    with cb.Solver(golden_config("drop2d_small"), "fp32") as s:
        with pytest.raises(cb.ClipError):
            s.adjoint(10, np.zeros(2))
    with cb.Solver(golden_config("drop3d_small"), "fp64") as s:
        with pytest.raises(cb.ClipError):
            s.tangent(10, np.zeros(2))
    with cb.Solver(golden_config("inlet2d_small"), "fp64") as s:
        with pytest.raises(cb.ClipError):
            s.adjoint(10, np.zeros(2))


def test_adjoint_workload_against_central_differences():
    """The configured adjoint workload (256x256 drop, drop2d_256x256_adjoint.txt) over 200
    steps, with the library's own tape policy (checkpoint_every = 0).  dJ/dg_y agrees with
    central differences (eps = 1e-4 relative) to 1e-6 (measured 3e-8).  For sigma and M the
    differences themselves move between step sizes by more than the adjoint's distance from
    them: their effect passes through the interface normal grad c / (|grad c| + 1e-32), not
    differentiable where grad c vanishes, and the relaxation time clamped at c = 0 and 1.
    The bar there is the differences' own spread over eps = 1e-6 .. 1e-4: the adjoint lies
    within twice that spread of the eps = 1e-5 difference (measured: sigma 0.0015 against a
    spread of 0.0016, M 5e-6 against 4e-5)."""
    import os

    cfg = os.path.join(os.path.dirname(cb.__file__), "workloads", "drop2d_256x256_adjoint.txt")
    s = cb.Solver(cfg, "fp64")
    c0 = s.initial_condition()
    steps = 200
    s.objective(steps, np.zeros(2), c0)
    c = s.interior_field("c")[..., 0, 0]
    x = np.arange(1, c.shape[0] + 1)[:, None]
    y = np.arange(1, c.shape[1] + 1)[None, :]
    target = np.array([(x * c).sum() / c.sum() + 3.0, (y * c).sum() / c.sum() + 5.0])
    p = s.params()
    theta = np.array([p["gy"], p["sigma"], p["mobility"]])
    J, _, gp = s.adjoint(steps, target, c0, checkpoint_every=0)
    Jc, _, gpc = s.adjoint(steps, target, c0, checkpoint_every=50)
    assert J == Jc
    assert np.allclose(gp, gpc, rtol=1e-12)

    def fd(i, eps):
        h = eps * abs(theta[i])
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        s.set_params(*tp)
        Jp = s.objective(steps, target, c0)
        s.set_params(*tm)
        Jm = s.objective(steps, target, c0)
        s.set_params(*theta)
        return (Jp - Jm) / (2 * h)

    g_fd = fd(0, 1e-4)
    assert abs(gp[0] - g_fd) <= 1e-6 * abs(g_fd), (gp[0], g_fd)
    for i in (1, 2):
        vals = [fd(i, eps) for eps in (1e-6, 1e-5, 1e-4)]
        spread = max(vals) - min(vals)
        assert abs(gp[i] - vals[1]) <= 2 * spread, (i, gp[i], vals)
    s.close()
