"""The differentiable loss pieces of cubnm_b200.grad (FP64 torch, CPU) against
the numpy FC / FCD of cubnm_b200.utils (the reference's empirical FC/FCD) and
scipy's Wasserstein distance, their gradients against finite differences, and
the argument checks of the adjoint entry points (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest
import scipy.stats
import torch

import cases
from cubnm_b200 import _abi, _lib, utils
from cubnm_b200.grad import (AdjointSizes, _declare, fc_corr_loss, fc_tril, fcd_tril, fcd_wasserstein,
                             rww_fit_loss, window_bounds)


def _bold(N=3, T=40, n=9, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(N, T, n)).cumsum(axis=1)


def test_fc_and_fcd_match_the_numpy_reference():
    bold = _bold()
    remove, ws, step = 6, 8, 3
    fc = fc_tril(torch.tensor(bold), remove).numpy()
    fcd = fcd_tril(torch.tensor(bold), remove, ws, step).numpy()
    for s in range(bold.shape[0]):
        x = bold[s, remove:, :].T  # (nodes, volumes)
        np.testing.assert_allclose(fc[s], utils.calculate_fc(x), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(fcd[s], utils.calculate_fcd(x, ws, step), rtol=1e-10, atol=1e-12)


def test_window_bounds_match_the_library_window_count():
    L = _lib.lib()
    for dur, remove, ws, step in ((60, 30, 10, 2), (300, 30, 30, 5), (40, 10, 8, 3)):
        args = cases.synthetic_args("rWW", N=2, nodes=8, duration_s=dur, bold_remove_s=remove, window_size=ws,
                                    window_step=step)
        p = _abi.Prepared(*args)
        sz = _abi.Sizes()
        assert L.cbnm_query_sizes(C.byref(p.args), C.byref(sz)) == 0
        assert len(window_bounds(dur, remove, ws, step)) == sz.n_windows


def test_wasserstein_matches_scipy():
    rng = np.random.default_rng(1)
    a = rng.normal(size=(4, 50))
    b = rng.normal(0.3, 1.2, size=50)
    w = fcd_wasserstein(torch.tensor(a), torch.tensor(b)).numpy()
    for s in range(4):  # equal sizes: exact
        assert abs(w[s] - scipy.stats.wasserstein_distance(a[s], b)) < 1e-12
    b2 = rng.normal(0.3, 1.2, size=173)  # unequal sizes: midpoint rule on the simulated quantiles
    w2 = fcd_wasserstein(torch.tensor(a), torch.tensor(b2)).numpy()
    for s in range(4):
        assert abs(w2[s] - scipy.stats.wasserstein_distance(a[s], b2)) < 0.05


def test_loss_gradient_matches_finite_differences():
    bold = torch.tensor(_bold(N=2, T=30, n=6, seed=2), requires_grad=True)
    emp = _bold(N=1, T=30, n=6, seed=3)[0].T
    emp_fc = torch.tensor(utils.calculate_fc(emp))
    emp_fcd = torch.tensor(utils.calculate_fcd(emp, 6, 2))
    loss = rww_fit_loss(bold, emp_fc, emp_fcd, 4, 6, 2).sum()
    loss.backward()
    g = bold.grad.numpy()
    rng = np.random.default_rng(4)
    v = rng.normal(size=bold.shape)
    h = 1e-6
    with torch.no_grad():
        lp = rww_fit_loss(bold + h * torch.tensor(v), emp_fc, emp_fcd, 4, 6, 2).sum().item()
        lm = rww_fit_loss(bold - h * torch.tensor(v), emp_fc, emp_fcd, 4, 6, 2).sum().item()
    assert abs((lp - lm) / (2 * h) - (g * v).sum()) < 1e-6 * max(1.0, abs((g * v).sum()))
    assert abs(fc_corr_loss(emp_fc[None], emp_fc).item()) < 1e-12


def test_adjoint_query_sizes_and_rejections():
    L = _declare(_lib.lib())
    N, n, dur = 3, 8, 4
    args = cases.synthetic_args("rWW", N=N, nodes=n, duration_s=dur, bold_remove_s=1, window_size=2, window_step=1)
    p = _abi.Prepared(*args)
    sz = AdjointSizes()
    assert L.cbnm_adjoint_query(C.byref(p.args), 1000, C.byref(sz)) == 0
    n_seg = dur * 1000 // 100
    assert sz.n_segments == n_seg and sz.bold_len == dur
    assert sz.checkpoint_bytes == N * n_seg * n * (2 * 4 + 4 * 8)
    assert sz.scratch_bytes == N * (100 * 4 * n * 8 + 1000 * 3 * n * 4 + 100 * n * 4)
    for model, fic, delay, seg in (("WC", 0, False, 1000), ("rWW", 1, False, 1000), ("rWW", 0, True, 1000),
                                   ("rWW", 0, False, 15)):
        a = list(cases.synthetic_args(model, N=2, nodes=8, duration_s=4, do_fic=fic, bold_remove_s=1,
                                      window_size=2, window_step=1))
        a[11] = delay
        pa = _abi.Prepared(*a)
        assert L.cbnm_adjoint_query(C.byref(pa.args), seg, C.byref(AdjointSizes())) != 0
        assert L.cbnm_last_error()


class _Sphere:
    """Stand-in for FitProblem: a shifted sphere in the unit box (CPU torch)."""

    def __init__(self, dim):
        self.torch, self.dev, self.dim, self.evals = torch, torch.device("cpu"), dim, 0
        self.c = torch.linspace(0.2, 0.8, dim, dtype=torch.float64)

    def loss(self, x):
        self.evals += x.shape[0]
        return ((x - self.c) ** 2).sum(dim=1)

    def loss_np(self, x):
        with torch.no_grad():
            return self.loss(torch.as_tensor(x, dtype=torch.float64)).numpy()


def test_cmaes_and_adam_minimise_a_sphere():
    from cubnm_b200.fit import adam_fit, cmaes_fit, grid_fit, time_to
    hist, x = cmaes_fit(_Sphere(12), popsize=16, generations=120, seed=1)
    assert hist[-1][1] < 1e-6 and all(b1 >= b2 for (_, b1), (_, b2) in zip(hist, hist[1:]))
    np.testing.assert_allclose(x, np.linspace(0.2, 0.8, 12), atol=2e-3)
    hist, x = adam_fit(_Sphere(12), n_starts=4, iters=300, lr=0.05)
    assert hist[-1][1] < 1e-4
    s = _Sphere(3)
    s.nodes = 1
    hist, x = grid_fit(s, 5)
    assert hist[-1][1] <= 0.1 and time_to(hist, 1e9) is not None
