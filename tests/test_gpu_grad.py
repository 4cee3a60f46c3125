"""Adjoint gradients (cubnm_b200.grad, C ABI cbnm_adjoint_*) on the GPU.

1. The adjoint's forward BOLD is the FP32 per-simulation run's BOLD.
2. Gradients of the fit loss (1 - r(FC)) + W1(FCD) match FP64 central finite
   differences of the FP64 path (directional derivatives along G, tied J_N, and a
   random w_p direction) within 1e-3 relative (the adjoint runs the FP32 state;
   measured agreement 7e-6 .. 9e-5).
3. Gradients of a BOLD loss match torch autograd through an FP64 torch
   restatement of the forward pass (tests/torch_rww.py) at 10 nodes.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

REL_TOL = 2e-2   # torch-autograd comparison
FD_TOL = 1e-3    # finite-difference comparison


def _problem_inputs(N, nodes, duration_s, seed, bold_tr=1000):
    rng = np.random.default_rng(seed)
    sc = cases.synthetic_sc(nodes, 0.4, seed)
    G = rng.uniform(0.5, 3.0, N)
    w_p = rng.uniform(0.8, 1.6, (N, 1)) * np.ones((N, nodes))
    J_N = rng.uniform(0.1, 0.3, (N, 1)) * np.ones((N, nodes))
    wIE = np.ones((N, nodes))
    sigma = np.full((N, nodes), 0.01)
    return sc, G, w_p, J_N, wIE, sigma


def _run_args(sc, G, w_p, J_N, wIE, sigma, duration_s, bold_tr, precision, noise_out=False):
    N, nodes = w_p.shape
    glob = G[None, :].astype(float).copy()
    reg = np.vstack([x.reshape(1, -1) for x in (w_p, J_N, wIE, sigma)]).astype(float)
    cfg = cases.model_config("rWW", 0, window_size=4, window_step=2, bold_remove_s=0, do_fc=False, do_fcd=False)
    cfg["precision"] = precision
    return ["rWW", np.ascontiguousarray(sc.reshape(1, -1)), np.zeros(N, np.intc), np.zeros(nodes * nodes), glob,
            np.ascontiguousarray(reg), np.zeros(N), cfg, True, False, noise_out, False, False, False, N, nodes,
            int(duration_s * 1000), bold_tr, bold_tr, 0, 0.1, 1.0]


def test_adjoint_forward_equals_fp32_run(monkeypatch):
    import torch
    from cubnm_b200 import core
    from cubnm_b200.grad import RWWProblem
    N, nodes, dur = 6, 24, 8
    sc, G, w_p, J_N, wIE, sigma = _problem_inputs(N, nodes, dur, 1)
    prob = RWWProblem(sc, nodes, dur, segment_steps=1000)
    t = lambda x: torch.tensor(x, dtype=torch.float64, device="cuda:0")  # noqa: E731
    bold = prob.bold(t(G), t(w_p), t(J_N), t(wIE), t(sigma)).cpu().numpy()
    monkeypatch.setenv("CBNM_FP32_KERNEL", "simt")
    ref = core.run_simulations(*_run_args(sc, G, w_p, J_N, wIE, sigma, dur, 1000, "fp32"))["sim_bold"]
    np.testing.assert_array_equal(bold.reshape(N, -1), ref)


def _fit_loss_np(bold, emp_fc, emp_fcd, remove, ws, step):
    import torch
    from cubnm_b200.grad import rww_fit_loss
    b = torch.as_tensor(bold, dtype=torch.float64)
    return rww_fit_loss(b, torch.as_tensor(emp_fc), torch.as_tensor(emp_fcd), remove, ws, step).numpy()


def test_gradients_match_fp64_finite_differences():
    import torch
    from cubnm_b200 import core, utils
    from cubnm_b200.grad import RWWProblem, rww_fit_loss
    N, nodes, dur, remove, ws, step = 4, 16, 24, 4, 6, 2
    sc, G, w_p, J_N, wIE, sigma = _problem_inputs(N, nodes, dur, 2)
    emp = cases.synthetic_emp_bold(nodes, dur, 7)
    emp_fc, emp_fcd = utils.calculate_fc(emp), utils.calculate_fcd(emp, ws, step)
    prob = RWWProblem(sc, nodes, dur, segment_steps=1000)
    t = lambda x: torch.tensor(x, dtype=torch.float64, device="cuda:0", requires_grad=True)  # noqa: E731
    tG, tw, tJ, tI, ts = t(G), t(w_p), t(J_N), t(wIE), t(sigma)
    bold = prob.bold(tG, tw, tJ, tI, ts)
    loss = rww_fit_loss(bold, torch.as_tensor(emp_fc, device="cuda:0"), torch.as_tensor(emp_fcd, device="cuda:0"),
                        remove, ws, step)
    loss.sum().backward()
    gG, gw, gJ = tG.grad.cpu().numpy(), tw.grad.cpu().numpy(), tJ.grad.cpu().numpy()

    def fp64_loss(G_, w_, J_):
        out = core.run_simulations(*_run_args(sc, G_, w_, J_, wIE, sigma, dur, 1000, "fp64"))
        return _fit_loss_np(out["sim_bold"].reshape(N, -1, nodes), emp_fc, emp_fcd, remove, ws, step)

    rng = np.random.default_rng(5)
    v = rng.normal(size=(N, nodes))
    checks = []
    h = 1e-5
    d = (fp64_loss(G + h, w_p, J_N) - fp64_loss(G - h, w_p, J_N)) / (2 * h)
    checks.append(("G", d, gG))
    d = (fp64_loss(G, w_p, J_N + h) - fp64_loss(G, w_p, J_N - h)) / (2 * h)
    checks.append(("J_N tied", d, gJ.sum(axis=1)))
    d = (fp64_loss(G, w_p + h * v, J_N) - fp64_loss(G, w_p - h * v, J_N)) / (2 * h)
    checks.append(("w_p along v", d, (gw * v).sum(axis=1)))
    for name, fd, adj in checks:
        scale = np.abs(fd).max()
        assert np.abs(fd - adj).max() <= FD_TOL * scale + 1e-8, (name, fd, adj)


def test_gradients_match_torch_fp64_autograd():
    import torch
    import torch_rww
    from cubnm_b200 import core
    from cubnm_b200.grad import RWWProblem
    N, nodes, dur, tr = 3, 10, 3, 100
    sc, G, w_p, J_N, wIE, sigma = _problem_inputs(N, nodes, dur, 3)
    out = core.run_simulations(*_run_args(sc, G, w_p, J_N, wIE, sigma, dur, tr, "fp64", noise_out=True))
    bw_it = dur * 1000
    nz = torch_rww.noise_steps(out["_noise"], out["_shuffled_nodes"], out["_shuffled_ts"], nodes, bw_it, 10)
    rng = np.random.default_rng(11)
    wgt = rng.normal(size=(N, bw_it // tr, nodes))

    # torch FP64 reference
    c = lambda x: torch.tensor(x, dtype=torch.float64, requires_grad=True)  # noqa: E731
    rG, rw, rJ = c(G), c(w_p), c(J_N)
    b_ref = torch_rww.bold_rww(rG, rw, rJ, torch.tensor(wIE), torch.tensor(sigma), sc, nz, bold_tr_iters=tr)
    np.testing.assert_allclose(b_ref.detach().numpy().reshape(N, -1), out["sim_bold"], rtol=1e-9, atol=1e-12)
    (b_ref * torch.tensor(wgt)).sum().backward()

    # adjoint
    prob = RWWProblem(sc, nodes, dur, bold_tr=tr, segment_steps=1000)
    g = lambda x: torch.tensor(x, dtype=torch.float64, device="cuda:0", requires_grad=True)  # noqa: E731
    aG, aw, aJ = g(G), g(w_p), g(J_N)
    bold = prob.bold(aG, aw, aJ, g(wIE), g(sigma))
    (bold * torch.tensor(wgt, device="cuda:0")).sum().backward()
    for name, ref, adj in (("G", rG.grad, aG.grad), ("w_p", rw.grad, aw.grad), ("J_N", rJ.grad, aJ.grad)):
        ref = ref.numpy()
        adj = adj.cpu().numpy()
        assert np.abs(ref - adj).max() <= REL_TOL * np.abs(ref).max() + 1e-10, (name, ref, adj)


# ---- G gradients by the tangent-linear integrator (cbnm_run_tangent_device)

def _delayed_args(model, N, nodes, duration_s, seed, precision, G):
    args = list(cases.synthetic_args(model, N=N, nodes=nodes, duration_s=duration_s, seed=seed, density=0.3, G=G,
                                     precision=precision, window_size=4, window_step=1, bold_remove_s=1))
    if model == "WC":
        reg = args[5].reshape(8, N, nodes)
        reg[6] = reg[7] = 0.01   # noise as the large-network workload
    args[3] = np.ascontiguousarray(cases.synthetic_lengths(nodes, seed).ravel())
    args[6] = np.full(N, 6.0)
    args[11] = True
    return args


@pytest.mark.parametrize("model,G", [("WC", [0.4, 1.2, 1.8]), ("rWW", [0.5, 1.5, 3.0])])
def test_tangent_dG_matches_fp64_finite_differences(model, G, monkeypatch):
    """dL/dG of L = sum(w * BOLD) (fixed random weights) and of the fit loss, from
    dBOLD/dG of the tangent integrator (FP32 state, delays, 6 m/s), against central
    differences of the FP64 path.  The tangent run's BOLD is the plain FP32 lane
    kernel run's.

    Every G here leaves the trajectory non-chaotic: on this network WC at G = 2.5
    is chaotic (a 1e-9 relative change of G moves the FP64 BOLD by 5e-3 within
    8 s), so its derivative grows exponentially and central differences cannot
    check it."""
    import torch
    from cubnm_b200 import core, grad, utils
    N, nodes, dur = 3, 24, 8
    G = np.array(G)
    bold, dG = grad.bold_and_dG(_delayed_args(model, N, nodes, dur, 11, "fp32", G))
    # the tangent integrates on the lane kernel: its value path is that kernel's plain run
    monkeypatch.setenv("CBNM_FP32_KERNEL", "lanes")
    plain = core.run_simulations(*_delayed_args(model, N, nodes, dur, 11, "fp32", G))["sim_bold"]
    monkeypatch.delenv("CBNM_FP32_KERNEL")
    np.testing.assert_array_equal(bold.cpu().numpy().reshape(N, -1), plain)
    w = np.random.default_rng(2).standard_normal(bold.shape[1:])
    tan = (dG.cpu().numpy() * w).sum(axis=(1, 2))
    emp = cases.synthetic_emp_bold(nodes, dur, 3)
    efc, efcd = utils.calculate_fc(emp), utils.calculate_fcd(emp, 4, 1)
    lf, ld, db = grad.fit_loss_terms(bold, efc, efcd, 1, 4, 1, True, grad=True)
    tan_fit = (db * dG).sum(dim=(1, 2)).cpu().numpy()

    def losses(Gv):
        o = core.run_simulations(*_delayed_args(model, N, nodes, dur, 11, "fp64", Gv))
        b = o["sim_bold"].reshape(N, -1, nodes)
        bt = torch.tensor(b, dtype=torch.float64)
        fit = grad.rww_fit_loss_torch(bt, torch.tensor(efc), torch.tensor(efcd), 1, 4, 1).numpy()
        return (b * w).sum(axis=(1, 2)), fit

    h = 1e-4 * np.maximum(1.0, G)
    (lp, fp), (lm, fm) = losses(G + h), losses(G - h)
    fd, fd_fit = (lp - lm) / (2 * h), (fp - fm) / (2 * h)
    rel = np.abs(tan - fd) / np.abs(fd).max()
    rel_fit = np.abs(tan_fit - fd_fit) / np.abs(fd_fit).max()
    assert rel.max() < 1e-2, (tan, fd, rel)
    assert rel_fit.max() < 2e-2, (tan_fit, fd_fit, rel_fit)
