"""The search methods of ``cubnm_b200.fit`` on closed-form objectives (CPU).

The GPU fit compares Adam on adjoint gradients with CMA-ES and a grid at equal
loss; these tests check that the CMA-ES restatement (Hansen 2016) and the Adam
and grid loops are sound on problems with known minima, so that comparison is
against a working CMA-ES: a shifted sphere, an ill-conditioned rotated
ellipsoid (which needs the covariance adaptation) and a grid whose best point
is known.
"""
import math

import numpy as np
import torch

from cubnm_b200 import fit


class Toy:
    """Stands in for FitProblem: `loss_np` on [B, dim] arrays, `loss` on torch."""

    def __init__(self, dim, f_np, f_torch=None):
        self.dim, self.nodes = dim, dim - 2
        self.f_np, self.f_torch = f_np, f_torch
        self.torch, self.dev = torch, "cpu"

    def loss_np(self, x):
        return self.f_np(np.asarray(x, dtype=float))

    def loss(self, x):
        return self.f_torch(x)


def _monotone(hist):
    best = [b for _, b in hist]
    return all(b1 <= b0 for b0, b1 in zip(best, best[1:]))


def test_cmaes_sphere():
    c = np.linspace(0.2, 0.8, 12)
    toy = Toy(12, lambda x: ((x - c) ** 2).sum(axis=1))
    hist, x = fit.cmaes_fit(toy, popsize=12, generations=400, seed=1)
    assert _monotone(hist)
    assert hist[-1][1] < 1e-12
    np.testing.assert_allclose(x, c, atol=1e-5)


def test_cmaes_rotated_ellipsoid():
    """Condition number 1e4 in a random rotation: plain isotropic steps stall,
    the rank-one / rank-mu updates and the eigendecomposition must learn it."""
    n = 8
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    scale = 10.0 ** (2 * np.arange(n) / (n - 1))  # axis lengths 1 .. 100, condition 1e4
    c = np.full(n, 0.45)

    def f(x):
        y = (x - c) @ Q
        return ((scale * y) ** 2).sum(axis=1)

    hist, x = fit.cmaes_fit(Toy(n, f), popsize=10, generations=1500, seed=2)
    assert _monotone(hist)
    assert hist[-1][1] < 1e-8
    np.testing.assert_allclose(x, c, atol=1e-4)


def test_adam_sphere():
    c = torch.linspace(0.25, 0.75, 6, dtype=torch.float64)
    toy = Toy(6, None, lambda x: ((x - c) ** 2).sum(dim=1))
    hist, x = fit.adam_fit(toy, n_starts=4, iters=800, lr=0.05, seed=0)
    assert _monotone(hist)
    assert hist[-1][1] < 1e-8
    np.testing.assert_allclose(x, c.numpy(), atol=1e-4)


def test_adam_skips_non_finite_candidates():
    """A start whose loss is not finite gets no update and never becomes best."""
    c = 0.5

    def f(x):
        v = ((x - c) ** 2).sum(dim=1)
        return torch.where(torch.arange(x.shape[0]) == 0, torch.full_like(v, math.nan), v)

    hist, x = fit.adam_fit(Toy(4, None, f), n_starts=3, iters=200, lr=0.05, seed=0)
    assert math.isfinite(hist[-1][1]) and hist[-1][1] < 1e-6


def test_grid_finds_its_best_point():
    n = 5  # G, J_N and 3 nodes of w_p
    target = np.array([0.25, 0.75, 0.5, 0.5, 0.5])
    toy = Toy(n, lambda x: ((x - target) ** 2).sum(axis=1))
    hist, x = fit.grid_fit(toy, per_axis=5)
    assert len(hist) == 5
    np.testing.assert_allclose(x, target)
    assert hist[-1][1] == 0.0


def test_time_to():
    hist = [(0.5, 3.0), (1.0, 2.0), (2.0, 1.0)]
    assert fit.time_to(hist, 2.0) == 1.0
    assert fit.time_to(hist, 0.5) is None
