"""The hand-written loss kernels of the gradient fit (cbnm_fit_loss, FP64)
against the torch FP64 restatement with autograd: both loss terms, and
dL/dBOLD, on random BOLD with the reference's window placement.  The
torch.autograd.Function that wraps the kernels (grad.rww_fit_loss on a CUDA
tensor) gives the same gradient as autograd through the restatement."""
import numpy as np
import pytest

import cases
from cubnm_b200 import grad, utils

pytestmark = pytest.mark.gpu


def _bold(N, T, n, seed):
    rng = np.random.default_rng(seed)
    lat = np.cumsum(rng.standard_normal((N, T, 3)), axis=1)
    return lat @ rng.standard_normal((3, n)) * 0.1 + rng.standard_normal((N, T, n))


@pytest.mark.parametrize("N,T,n,remove,ws,step,edges", [(4, 60, 20, 10, 10, 2, True), (3, 80, 33, 5, 8, 3, False),
                                                        (2, 300, 200, 30, 30, 5, True), (3, 30, 12, 2, 40, 2, True)])
def test_kernels_match_torch_autograd(N, T, n, remove, ws, step, edges):
    import torch
    dev = torch.device("cuda:0")
    b = torch.tensor(_bold(N, T, n, N * T), dtype=torch.float64, device=dev)
    emp = cases.synthetic_emp_bold(n, T, 3)
    efc = torch.tensor(utils.calculate_fc(emp), dtype=torch.float64, device=dev)
    efcd = torch.tensor(utils.calculate_fcd(emp, ws, step) if T - remove > ws else np.zeros(3), dtype=torch.float64,
                        device=dev)
    wins = grad.window_bounds(T, remove, ws, step, edges)
    lf, ld, db = grad.fit_loss_terms(b, efc, efcd, remove, ws, step, edges, grad=True)
    x = b.clone().requires_grad_(True)
    ref_fc = grad.fc_corr_loss(grad.fc_tril(x, remove), efc)
    if len(wins) >= 2:
        ref_fcd = grad.fcd_wasserstein(grad.fcd_tril(x, remove, ws, step, edges), efcd)
    else:
        ref_fcd = torch.zeros_like(ref_fc)
    (ref_fc + ref_fcd).sum().backward()
    np.testing.assert_allclose(lf.cpu().numpy(), ref_fc.detach().cpu().numpy(), rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(ld.cpu().numpy(), ref_fcd.detach().cpu().numpy(), rtol=1e-11, atol=1e-13)
    g, gr = db.cpu().numpy(), x.grad.cpu().numpy()
    assert np.abs(g - gr).max() <= 1e-9 * np.abs(gr).max(), np.abs(g - gr).max() / np.abs(gr).max()
    # the autograd wrapper: the same gradient, scaled per simulation by the upstream gradient
    y = b.clone().requires_grad_(True)
    w = torch.arange(1, N + 1, dtype=torch.float64, device=dev)
    (grad.rww_fit_loss(y, efc, efcd, remove, ws, step, edges) * w).sum().backward()
    np.testing.assert_allclose(y.grad.cpu().numpy(), g * w.cpu().numpy()[:, None, None], rtol=1e-12, atol=1e-15)


def test_loss_only_call_and_argument_errors():
    import torch
    b = torch.tensor(_bold(2, 40, 10, 1), dtype=torch.float64, device="cuda:0")
    emp = cases.synthetic_emp_bold(10, 40, 3)
    lf, ld, db = grad.fit_loss_terms(b, utils.calculate_fc(emp), utils.calculate_fcd(emp, 6, 2), 4, 6, 2, True)
    assert db is None and torch.isfinite(lf).all() and torch.isfinite(ld).all()
    with pytest.raises(RuntimeError):
        grad.fit_loss_terms(b, utils.calculate_fc(emp), utils.calculate_fcd(emp, 6, 2), 39, 6, 2, True)
