"""Fitting rWW parameters on the GPU: Adam on adjoint gradients beside the
gradient-free searches the reference offers (grid and CMA-ES,
src/cubnm/optimize.py: GridOptimizer, CMAESOptimizer).

Free parameters per candidate: G, J_N (one value for all nodes) and w_p per node
(2 + nodes in total), searched in the box G in [0.001, 10], J_N in [0.001, 0.5],
w_p in [0, 2] (the reference's default rWW bounds).  The objective is the loss
of :func:`cubnm_b200.grad.rww_fit_loss`, (1 - r(FC)) + W1(FCD), lower is better;
every method evaluates its candidates as one batch of simulations through
:class:`cubnm_b200.grad.RWWProblem` (same kernel, same noise).

* ``adam_fit``: independent starts in one batch; parameters are
  lo + (hi - lo) sigmoid(z) and Adam steps z with the adjoint gradient.
* ``cmaes_fit``: CMA-ES in the unit box (mean 0.5, step 0.3, candidates
  clipped to the box), restated from N. Hansen, "The CMA Evolution Strategy: A
  Tutorial" (2016): weighted recombination, cumulative step-size adaptation,
  rank-one and rank-mu covariance updates.
* ``grid_fit``: a regular grid over (G, J_N, homogeneous w_p).

``python -m cubnm_b200.fit`` runs the three on one synthetic problem and prints
one JSON line with each method's best loss over wall time.
"""
import argparse
import json
import math
import time

import numpy as np

from . import utils
from .grad import RWWProblem, rww_fit_loss
from .synthetic import synthetic_emp_bold, synthetic_sc

BOUNDS = {"G": (0.001, 10.0), "J_N": (0.001, 0.5), "w_p": (0.0, 2.0)}


class FitProblem:
    """One empirical target and the batched loss of candidate parameter sets."""

    def __init__(self, sc, emp_bold, duration_s, *, window_size=30, window_step=5, n_vols_remove=0, wIE=1.0,
                 sigma=0.01, sim_seed=0, segment_steps=1000, device="cuda:0", fast_eval=False):
        import torch
        self.torch = torch
        self.nodes = sc.shape[0]
        self.prob = RWWProblem(sc, self.nodes, duration_s, sim_seed=sim_seed, segment_steps=segment_steps,
                               device=device)
        self.dev = self.prob.dev
        self.emp_fc = torch.as_tensor(utils.calculate_fc(emp_bold), device=self.dev)
        self.emp_fcd = torch.as_tensor(utils.calculate_fcd(emp_bold, window_size, window_step), device=self.dev)
        self.ws, self.step, self.remove = window_size, window_step, n_vols_remove
        self.wIE, self.sigma = wIE, sigma
        self.dim = 2 + self.nodes
        self.evals = 0
        self.fast_eval = fast_eval

    def params_from_unit(self, x):
        """x [B, 2 + nodes] in [0, 1] -> G [B], w_p [B, nodes], J_N [B, nodes]."""
        (g0, g1), (j0, j1), (w0, w1) = BOUNDS["G"], BOUNDS["J_N"], BOUNDS["w_p"]
        G = g0 + (g1 - g0) * x[:, 0]
        J = j0 + (j1 - j0) * x[:, 1]
        w_p = w0 + (w1 - w0) * x[:, 2:]
        return G, w_p, J[:, None].expand(-1, self.nodes)

    def loss(self, x):
        """Per-candidate loss of x [B, dim] (torch, in [0, 1]); differentiable."""
        torch = self.torch
        G, w_p, J_N = self.params_from_unit(x)
        B = x.shape[0]
        wIE = torch.full((B, self.nodes), self.wIE, dtype=torch.float64, device=self.dev)
        sig = torch.full((B, self.nodes), self.sigma, dtype=torch.float64, device=self.dev)
        bold = self.prob.bold(G, w_p, J_N, wIE, sig)
        self.evals += B
        return rww_fit_loss(bold, self.emp_fc, self.emp_fcd, self.remove, self.ws, self.step)

    def loss_np(self, x):
        """Loss of candidates without gradients (grid, CMA-ES): with ``fast_eval`` on the
        fastest FP32 forward kernel for the shape (cbnm_run_simulations_device) and the
        loss kernels, else through the adjoint's forward pass."""
        torch = self.torch
        with torch.no_grad():
            xt = torch.as_tensor(x, dtype=torch.float64, device=self.dev)
            v = self._fast_loss(xt) if self.fast_eval else self.loss(xt)
        v = v.cpu().numpy()
        return np.where(np.isfinite(v), v, np.inf)

    def _fast_loss(self, x):
        from .grad import fit_loss_terms, run_device
        G, w_p, J_N = self.params_from_unit(x)
        B, n = x.shape[0], self.nodes
        cfg = dict(self.prob.config)
        cfg["precision"] = "fp32"
        reg = np.stack([w_p.cpu().numpy().reshape(-1), J_N.cpu().numpy().reshape(-1), np.full(B * n, self.wIE),
                        np.full(B * n, self.sigma)])
        args = ["rWW", self.prob.sc.cpu().numpy(), np.zeros(B, np.int32), np.zeros(n * n),
                G.cpu().numpy().reshape(1, B).astype(float), reg, np.zeros(B), cfg, False, False, False, False, False,
                False, B, n, self.prob.duration_ms, self.prob.bold_tr, self.prob.bold_tr, self.prob.sim_seed,
                self.prob.dt, self.prob.bw_dt]
        bold = run_device(args, device=self.dev)
        lf, ld, _ = fit_loss_terms(bold, self.emp_fc, self.emp_fcd, self.remove, self.ws, self.step)
        self.evals += B
        return lf + ld


def adam_fit(fp, n_starts, iters, lr=0.6, seed=0):
    """Adam from n_starts random starts (one batch); returns the history
    [(seconds, best loss so far)] and the best unit-box point."""
    torch = fp.torch
    g = torch.Generator().manual_seed(seed)
    x0 = torch.rand((n_starts, fp.dim), generator=g, dtype=torch.float64) * 0.8 + 0.1
    z = torch.logit(x0).to(fp.dev).requires_grad_(True)
    opt = torch.optim.Adam([z], lr=lr)
    hist, best, best_x = [], math.inf, None
    t0 = time.perf_counter()
    for _ in range(iters):
        opt.zero_grad()
        x = torch.sigmoid(z)
        loss = fp.loss(x)
        finite = torch.isfinite(loss)
        torch.where(finite, loss, torch.zeros_like(loss)).sum().backward()
        with torch.no_grad():
            z.grad[~finite] = 0
        opt.step()
        lv = loss.detach().cpu().numpy()
        if np.isfinite(lv).any():
            i = int(np.nanargmin(np.where(np.isfinite(lv), lv, np.nan)))
            if lv[i] < best:
                best, best_x = float(lv[i]), x.detach()[i].cpu().numpy()
        hist.append((time.perf_counter() - t0, best))
    return hist, best_x


def cmaes_fit(fp, popsize, generations, sigma0=0.3, seed=0):
    """CMA-ES (Hansen 2016) in the unit box; returns history and best point."""
    rng = np.random.default_rng(seed)
    n = fp.dim
    lam = popsize
    mu = lam // 2
    w = np.log(mu + 0.5) - np.log(np.arange(1, mu + 1))
    w /= w.sum()
    mueff = 1.0 / np.sum(w ** 2)
    cc = (4 + mueff / n) / (n + 4 + 2 * mueff / n)
    cs = (mueff + 2) / (n + mueff + 5)
    c1 = 2 / ((n + 1.3) ** 2 + mueff)
    cmu = min(1 - c1, 2 * (mueff - 2 + 1 / mueff) / ((n + 2) ** 2 + mueff))
    damps = 1 + 2 * max(0.0, math.sqrt((mueff - 1) / (n + 1)) - 1) + cs
    chin = math.sqrt(n) * (1 - 1 / (4 * n) + 1 / (21 * n * n))
    m = np.full(n, 0.5)
    sigma = sigma0
    pc, ps = np.zeros(n), np.zeros(n)
    B, D, C = np.eye(n), np.ones(n), np.eye(n)
    invsqrtC = np.eye(n)
    eigen_gen = 0
    hist, best, best_x = [], math.inf, None
    t0 = time.perf_counter()
    for gen in range(generations):
        zs = rng.standard_normal((lam, n))
        ys = (zs * D) @ B.T
        xs = np.clip(m + sigma * ys, 0.0, 1.0)
        f = fp.loss_np(xs)
        order = np.argsort(f)
        if f[order[0]] < best:
            best, best_x = float(f[order[0]]), xs[order[0]].copy()
        hist.append((time.perf_counter() - t0, best))
        ysel = (xs[order[:mu]] - m) / sigma  # the steps actually taken (after clipping)
        m_old = m
        m = m + sigma * (w @ ysel)
        ps = (1 - cs) * ps + math.sqrt(cs * (2 - cs) * mueff) * (invsqrtC @ (m - m_old)) / sigma
        hsig = np.linalg.norm(ps) / math.sqrt(1 - (1 - cs) ** (2 * (gen + 1))) / chin < 1.4 + 2 / (n + 1)
        pc = (1 - cc) * pc + hsig * math.sqrt(cc * (2 - cc) * mueff) * (m - m_old) / sigma
        C = ((1 - c1 - cmu) * C + c1 * (np.outer(pc, pc) + (1 - hsig) * cc * (2 - cc) * C)
             + cmu * (ysel.T * w) @ ysel)
        sigma *= math.exp((cs / damps) * (np.linalg.norm(ps) / chin - 1))
        if gen - eigen_gen > lam / (c1 + cmu) / n / 10:
            eigen_gen = gen
            C = np.triu(C) + np.triu(C, 1).T
            D2, B = np.linalg.eigh(C)
            D = np.sqrt(np.maximum(D2, 1e-20))
            invsqrtC = B @ np.diag(1 / D) @ B.T
    return hist, best_x


def grid_fit(fp, per_axis):
    """Grid over G x J_N x homogeneous w_p (per_axis points each) in batches of
    per_axis**2 candidates."""
    axis = np.linspace(0.0, 1.0, per_axis)
    pts = np.array([[g, j, wp] for g in axis for j in axis for wp in axis])
    x = np.concatenate([pts[:, :2], np.repeat(pts[:, 2:3], fp.nodes, axis=1)], axis=1)
    hist, best, best_x = [], math.inf, None
    t0 = time.perf_counter()
    bs = per_axis * per_axis
    for s in range(0, len(x), bs):
        f = fp.loss_np(x[s:s + bs])
        i = int(np.argmin(f))
        if f[i] < best:
            best, best_x = float(f[i]), x[s + i].copy()
        hist.append((time.perf_counter() - t0, best))
    return hist, best_x


def time_to(hist, target):
    """First time in a [(seconds, best)] history at which best <= target (None if never)."""
    for t, b in hist:
        if b <= target:
            return t
    return None


def main(argv=None):
    ap = argparse.ArgumentParser(description="Adam (adjoint gradients) vs CMA-ES vs grid on one synthetic rWW fit")
    ap.add_argument("--nodes", type=int, default=200)
    ap.add_argument("--duration", type=int, default=60)
    ap.add_argument("--window", type=int, default=30)
    ap.add_argument("--step", type=int, default=5)
    ap.add_argument("--popsize", type=int, default=128)
    ap.add_argument("--generations", type=int, default=40)
    ap.add_argument("--adam-iters", type=int, default=14)
    ap.add_argument("--lr", type=float, default=0.6)
    ap.add_argument("--grid", type=int, default=6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--methods", default="grid,cmaes,adam", help="comma-separated subset of grid,cmaes,adam")
    ap.add_argument("--target", type=float, default=None, help="loss to time against (default: CMA-ES's best)")
    ap.add_argument("--fast-eval", action="store_true",
                    help="grid / CMA-ES evaluate on the fastest FP32 forward kernel instead of the adjoint's forward")
    o = ap.parse_args(argv)
    sc = synthetic_sc(o.nodes, 0.25, o.seed)
    emp = synthetic_emp_bold(o.nodes, o.duration, o.seed + 7)
    fp = FitProblem(sc, emp, o.duration, window_size=o.window, window_step=o.step, fast_eval=o.fast_eval)
    fp.loss_np(np.full((2, fp.dim), 0.5))  # warm-up: noise generation, allocations
    res = {}
    methods = o.methods.split(",")
    for name, fn in (("grid", lambda: grid_fit(fp, o.grid)),
                     ("cmaes", lambda: cmaes_fit(fp, o.popsize, o.generations, seed=o.seed)),
                     ("adam", lambda: adam_fit(fp, o.popsize, o.adam_iters, lr=o.lr, seed=o.seed))):
        if name not in methods:
            continue
        fp.evals = 0
        hist, _ = fn()
        res[name] = {"best": hist[-1][1], "seconds": hist[-1][0], "simulations": fp.evals,
                     "history": [[round(t, 3), b] for t, b in hist]}
    target = o.target if o.target is not None else res["cmaes"]["best"]
    res["target"] = target
    res["seconds_to_target"] = {k: time_to([tuple(h) for h in res[k]["history"]], target) for k in res
                                if k in ("grid", "cmaes", "adam")}
    res["config"] = vars(o)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
