"""Gradients of a BOLD-based loss with respect to rWW parameters.

The reference fits parameters with grid search and gradient-free optimisers
(src/cubnm/optimize.py: grid, CMA-ES, NSGA-II over SimGroup.run).  This module
makes the same simulation differentiable: :class:`RWWProblem` runs a batch of
rWW simulations through the adjoint entry points of the C ABI
(``cbnm_adjoint_forward`` / ``cbnm_adjoint_backward``), and
``RWWProblem.bold(G, w_p, J_N, wIE, sigma)`` returns BOLD as a torch tensor with
a backward pass, so any torch loss on BOLD yields pathwise gradients (noise held
fixed) for G per simulation and w_p, J_N, wIE, sigma per node.

The forward is the FP32 per-simulation rWW integrator (FP64 Balloon-Windkessel),
checkpointed every ``segment_steps`` integration steps; the backward recomputes
each segment from its checkpoint and runs it in reverse on the GPU.

Loss: :func:`rww_fit_loss` = (1 - Pearson r of FC lower triangles) + the 1-D
Wasserstein distance of FCD value distributions from sorted values.  On the
GPU it runs the library's hand-written FP64 kernels for the loss and its
gradient (``cbnm_fit_loss``); :func:`rww_fit_loss_torch` (built from
:func:`fc_tril`, :func:`fcd_tril`, :func:`fc_corr_loss`,
:func:`fcd_wasserstein`) is the torch restatement used on the CPU and as the
check.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import check, lib


class AdjointSizes(C.Structure):
    _fields_ = [("n_segments", C.c_int64), ("checkpoint_bytes", C.c_int64), ("scratch_bytes", C.c_int64),
                ("bold_len", C.c_int64), ("sims_per_backward_launch", C.c_int64)]


def _declare(L):
    if getattr(L, "_adjoint_declared", False):
        return L
    vp, ap = C.c_void_p, C.POINTER(_abi.RunArgs)
    L.cbnm_adjoint_query.argtypes = [ap, C.c_int, C.POINTER(AdjointSizes)]
    L.cbnm_adjoint_query.restype = C.c_int
    L.cbnm_adjoint_forward.argtypes = [ap, C.c_int, vp, vp]
    L.cbnm_adjoint_forward.restype = C.c_int
    L.cbnm_adjoint_backward.argtypes = [ap, C.c_int, vp, vp, vp, vp, vp]
    L.cbnm_adjoint_backward.restype = C.c_int
    L.cbnm_fit_loss.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int,
                                vp, vp, vp]
    L.cbnm_fit_loss.restype = C.c_int
    L._adjoint_declared = True
    return L


def window_bounds(bold_len, n_vols_remove, window_size, window_step, drop_edges=True):
    """Inclusive volume ranges of the dynamic-FC windows (src/ext/utils.cpp:21-52)."""
    corr_len = bold_len - n_vols_remove
    half = window_size // 2
    first = (half if drop_edges else 0) + n_vols_remove
    last = (corr_len - 1 - half if drop_edges else corr_len - 1) + n_vols_remove
    return [(max(0, c - half), min(bold_len - 1, c + half)) for c in range(first, last + 1, window_step)]


def _corr_tril(x):
    """Pearson r of the columns of x [..., T, n], lower triangle in np.tril_indices(n, -1) order."""
    import torch
    xc = x - x.mean(dim=-2, keepdim=True)
    cov = xc.transpose(-1, -2) @ xc
    sd = torch.sqrt(torch.diagonal(cov, dim1=-2, dim2=-1))
    r = cov / (sd.unsqueeze(-1) * sd.unsqueeze(-2))
    i, j = np.tril_indices(x.shape[-1], -1)
    return r[..., i, j]


def fc_tril(bold, n_vols_remove):
    """Static FC of BOLD [N, T, n] over volumes [n_vols_remove, T): [N, n_pairs]."""
    return _corr_tril(bold[:, n_vols_remove:, :])


def fcd_tril(bold, n_vols_remove, window_size, window_step, drop_edges=True):
    """FCD lower triangle of BOLD [N, T, n]: Pearson r between window-FC vectors."""
    import torch
    wins = window_bounds(bold.shape[1], n_vols_remove, window_size, window_step, drop_edges)
    wfc = torch.stack([_corr_tril(bold[:, s:e + 1, :]) for s, e in wins], dim=1)  # [N, W, P]
    return _corr_tril(wfc.transpose(1, 2))


def fc_corr_loss(sim_fc, emp_fc):
    """1 - Pearson r between each row of sim_fc [N, P] and emp_fc [P]."""
    import torch
    s = sim_fc - sim_fc.mean(dim=1, keepdim=True)
    e = emp_fc - emp_fc.mean()
    r = (s * e).sum(dim=1) / (torch.sqrt((s * s).sum(dim=1)) * torch.sqrt((e * e).sum()))
    return 1.0 - r


def fcd_wasserstein(sim_fcd, emp_fcd):
    """1-D Wasserstein distance W1 = int_0^1 |Q_sim(p) - Q_emp(p)| dp between the value
    distribution of each row of sim_fcd [N, m] and emp_fcd [m2], by the midpoint
    rule on the simulated quantiles: mean_i |sorted_sim[i] - Q_emp((i + 1/2)/m)|
    with Q_emp the empirical quantile function (sorted_emp[floor(p m2)]).  Exact
    when m == m2; the gradient flows through the sorted simulated values.  The
    index floor((i + 1/2) m2 / m) = ((2i + 1) m2) // (2m) is taken in integers:
    in floating point it can fall one short where the quotient is a whole number."""
    import torch
    m, m2 = sim_fcd.shape[1], emp_fcd.numel()
    emp_sorted = torch.sort(emp_fcd.reshape(-1)).values
    i = torch.arange(m, dtype=torch.int64, device=sim_fcd.device)
    q = emp_sorted[((2 * i + 1) * m2 // (2 * m)).clamp(max=m2 - 1)]
    return (torch.sort(sim_fcd, dim=1).values - q).abs().mean(dim=1)


def rww_fit_loss_torch(bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges=True):
    """Per-simulation loss (1 - r(FC)) + W1(FCD) on BOLD [N, T, n], in torch (FP64
    autograd): the reference the hand-written kernels are checked against."""
    return (fc_corr_loss(fc_tril(bold, n_vols_remove), emp_fc) +
            fcd_wasserstein(fcd_tril(bold, n_vols_remove, window_size, window_step, drop_edges), emp_fcd))


def rww_fit_loss(bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges=True):
    """Per-simulation loss (1 - r(FC)) + W1(FCD) on BOLD [N, T, n] (float64).

    On a CUDA tensor the loss and its gradient come from the library's
    hand-written kernels (``cbnm_fit_loss``: FC, window FCs, FCD, sort, W1 and the
    chain rule back to BOLD in one pass); elsewhere from the torch restatement."""
    if not bold.is_cuda:
        return rww_fit_loss_torch(bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges)
    return _LOSS.apply(bold, emp_fc, emp_fcd, int(n_vols_remove), int(window_size), int(window_step), bool(drop_edges))


def fit_loss_terms(bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges=True, grad=False):
    """The two loss terms (1 - r(FC), W1(FCD)) of BOLD [N, T, n] on the device, and
    d(sum of both)/dBOLD when ``grad``: (loss_fc [N], loss_fcd [N], dbold or None)."""
    import torch
    L = _declare(lib())
    bold = bold.detach().to(torch.float64).contiguous()
    N, T, n = bold.shape
    efc = np.ascontiguousarray(np.asarray(emp_fc.detach().cpu() if hasattr(emp_fc, "detach") else emp_fc,
                                          dtype=np.float64))
    efcd = np.ascontiguousarray(np.asarray(emp_fcd.detach().cpu() if hasattr(emp_fcd, "detach") else emp_fcd,
                                           dtype=np.float64))
    lf = torch.empty(N, dtype=torch.float64, device=bold.device)
    ld = torch.empty(N, dtype=torch.float64, device=bold.device)
    db = torch.empty_like(bold) if grad else None
    torch.cuda.synchronize(bold.device)  # the library works on its own stream
    dp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    check(L.cbnm_fit_loss(_ptr(bold), N, T, n, int(n_vols_remove), int(window_size), int(window_step),
                          int(bool(drop_edges)), dp(efc), dp(efcd), int(efcd.size), _ptr(lf), _ptr(ld),
                          _ptr(db) if db is not None else None))
    return lf, ld, db


class RWWProblem:
    """A differentiable batch of rWW simulations on one GPU.

    sc: [n_scs, nodes*nodes] or [nodes, nodes] (row = source); sc_indices [N] picks
    each simulation's SC (all 0 by default).  The noise follows the reference's
    generator for (sim_seed, nodes, duration, noise segment), exactly as
    cbnm_run_simulations does, so BOLD equals that of a "fp32" run with the same
    inputs (per-simulation kernel).
    """

    def __init__(self, sc, nodes, duration_s, *, sc_indices=None, sim_seed=0, dt=0.1, bw_dt=1.0, bold_tr=1000,
                 noise_segment_s=30, segment_steps=1000, device="cuda:0"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.nodes = int(nodes)
        sc = np.asarray(sc, dtype=np.float64).reshape(-1, self.nodes * self.nodes)
        self.sc = torch.from_numpy(np.ascontiguousarray(sc)).to(self.dev)
        self.sc_indices = None if sc_indices is None else np.asarray(sc_indices, dtype=np.int32)
        self.duration_ms = int(round(duration_s * 1000))
        self.sim_seed, self.dt, self.bw_dt, self.bold_tr = int(sim_seed), float(dt), float(bw_dt), int(bold_tr)
        self.segment_steps = int(segment_steps)
        self.config = {"do_fc": "0", "do_fcd": "0", "bold_remove_s": "0", "exc_interhemispheric": "0",
                       "window_size": "10", "window_step": "2", "drop_edges": "1",
                       "noise_time_steps": str(int(noise_segment_s * 1000)), "verbose": "0",
                       "progress_interval": "500", "do_fic": "0", "max_fic_trials": "0",
                       "precision": "fp32"}
        self.L = _declare(lib())
        self.last_forward_ms = self.last_backward_ms = 0.0

    def _args(self, N, g, r):
        """cbnm_run_args for N simulations with device parameter arrays g [1, N], r [4, N*n]."""
        torch = self.torch
        n = self.nodes
        sc_idx = np.zeros(N, np.int32) if self.sc_indices is None else self.sc_indices
        host = ["rWW", self.sc.cpu().numpy(), sc_idx, np.zeros(n * n), np.zeros((1, N)), np.zeros((4, N * n)),
                np.zeros(N), self.config, False, False, False, False, False, False, N, n, self.duration_ms,
                self.bold_tr, self.bold_tr, self.sim_seed, self.dt, self.bw_dt]
        prep = _abi.Prepared(*host)
        keep = {"sc_idx": torch.from_numpy(sc_idx).to(self.dev), "dist": torch.zeros(n * n, dtype=torch.float64,
                                                                                     device=self.dev),
                "v": torch.zeros(N, dtype=torch.float64, device=self.dev), "g": g, "r": r}
        dp = lambda x: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_double))  # noqa: E731
        a = prep.args
        a.sc = dp(self.sc)
        a.n_scs = int(self.sc.shape[0])
        a.sc_indices = C.cast(C.c_void_p(keep["sc_idx"].data_ptr()), C.POINTER(C.c_int32))
        a.sc_dist = dp(keep["dist"])
        a.global_params = dp(g)
        a.regional_params = dp(r)
        a.v_list = dp(keep["v"])
        return prep, keep

    def sizes(self, N):
        torch = self.torch
        g = torch.zeros((1, N), dtype=torch.float64, device=self.dev)
        r = torch.zeros((4, N * self.nodes), dtype=torch.float64, device=self.dev)
        prep, _ = self._args(N, g, r)
        sz = AdjointSizes()
        check(self.L.cbnm_adjoint_query(C.byref(prep.args), self.segment_steps, C.byref(sz)))
        return sz

    def bold(self, G, w_p, J_N, wIE, sigma):
        """BOLD [N, bold_len, nodes] (float64, on the device) of simulations with G [N]
        and w_p, J_N, wIE, sigma [N, nodes]; differentiable in all five."""
        return _BOLD.apply(self, G, w_p, J_N, wIE, sigma)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _load_timing(L):
    t = _abi.Timing()
    L.cbnm_last_timing(C.byref(t))
    return float(t.integrate_ms)


def _autograd_function():
    import torch

    class BOLD(torch.autograd.Function):
        @staticmethod
        def forward(ctx, prob, G, w_p, J_N, wIE, sigma):
            N, n = G.shape[0], prob.nodes
            g = G.detach().to(prob.dev, torch.float64).reshape(1, N).contiguous()
            r = torch.stack([x.detach().to(prob.dev, torch.float64).reshape(N, n) for x in (w_p, J_N, wIE, sigma)])
            r = r.reshape(4, N * n).contiguous()
            prep, keep = prob._args(N, g, r)
            sz = AdjointSizes()
            check(prob.L.cbnm_adjoint_query(C.byref(prep.args), prob.segment_steps, C.byref(sz)))
            bold = torch.empty((N, int(sz.bold_len), n), dtype=torch.float64, device=prob.dev)
            ckpt = torch.empty(int(sz.checkpoint_bytes), dtype=torch.uint8, device=prob.dev)
            torch.cuda.synchronize(prob.dev)  # the library runs on its own stream
            check(prob.L.cbnm_adjoint_forward(C.byref(prep.args), prob.segment_steps, _ptr(bold), _ptr(ckpt)))
            prob.last_forward_ms = _load_timing(prob.L)
            ctx.prob, ctx.sz = prob, sz
            ctx.save_for_backward(g, r, ckpt)
            return bold

        @staticmethod
        def backward(ctx, gbold):
            prob, sz = ctx.prob, ctx.sz
            g, r, ckpt = ctx.saved_tensors
            N, n = g.shape[1], prob.nodes
            gbold = gbold.to(torch.float64).contiguous()
            scratch = torch.empty(int(sz.scratch_bytes), dtype=torch.uint8, device=prob.dev)
            gg = torch.empty((1, N), dtype=torch.float64, device=prob.dev)
            gr = torch.empty((4, N * n), dtype=torch.float64, device=prob.dev)
            prep, keep = prob._args(N, g, r)
            torch.cuda.synchronize(prob.dev)
            check(prob.L.cbnm_adjoint_backward(C.byref(prep.args), prob.segment_steps, _ptr(gbold), _ptr(ckpt),
                                               _ptr(scratch), _ptr(gg), _ptr(gr)))
            prob.last_backward_ms = _load_timing(prob.L)
            gr = gr.reshape(4, N, n)
            return None, gg[0], gr[0], gr[1], gr[2], gr[3]

    return BOLD


class _Lazy:
    fn = None
    make = staticmethod(_autograd_function)

    @classmethod
    def apply(cls, *args):
        if cls.fn is None:
            cls.fn = cls.make()
        return cls.fn.apply(*args)


def _loss_function():
    import torch

    class Loss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges):
            lf, ld, db = fit_loss_terms(bold, emp_fc, emp_fcd, n_vols_remove, window_size, window_step, drop_edges,
                                        grad=ctx.needs_input_grad[0])
            ctx.save_for_backward(db if db is not None else torch.empty(0))
            return (lf + ld).to(bold.dtype)

        @staticmethod
        def backward(ctx, go):
            (db,) = ctx.saved_tensors
            return (go.to(db.dtype)[:, None, None] * db), None, None, None, None, None, None

    return Loss


class _LazyBOLD(_Lazy):
    fn = None
    make = staticmethod(_autograd_function)


class _LazyLoss(_Lazy):
    fn = None
    make = staticmethod(_loss_function)


_BOLD = _LazyBOLD
_LOSS = _LazyLoss


def _device_run(args, device, tangent):
    """Runs the reference's 22 arguments (host arrays) with inputs and outputs in
    device memory; returns (bold [N, bold_len, nodes], dBOLD/dG or None)."""
    import torch
    dev = torch.device(device)
    L = lib()
    L.cbnm_run_tangent_device.argtypes = [C.POINTER(_abi.RunArgs), C.POINTER(_abi.Outputs), C.c_void_p]
    L.cbnm_run_tangent_device.restype = C.c_int
    prep = _abi.Prepared(*args)
    sizes = _abi.Sizes()
    check(L.cbnm_query_sizes(C.byref(prep.args), C.byref(sizes)))
    N, n = int(args[14]), int(args[15])
    t = lambda x, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(x)).to(dev, dt)  # noqa: E731
    keep = {"sc": t(args[1]), "sc_idx": t(np.asarray(args[2], np.int32), torch.int32), "dist": t(args[3]),
            "g": t(args[4]), "r": t(args[5]), "v": t(args[6])}
    bold = torch.empty((N, sizes.bold_len, n), dtype=torch.float64, device=dev)
    dG = torch.zeros_like(bold) if tangent else None
    fc = torch.empty((N, max(1, sizes.n_pairs)), dtype=torch.float64, device=dev)
    fcd = torch.empty((N, max(1, sizes.n_window_pairs)), dtype=torch.float64, device=dev)
    states = torch.empty((sizes.n_state_vars, N, n * (sizes.states_len if args[9] else 1)), dtype=torch.float64,
                         device=dev)
    gb = torch.empty((max(1, sizes.n_global_out_bool), N), dtype=torch.uint8, device=dev)
    gi = torch.empty((max(1, sizes.n_global_out_int), N), dtype=torch.int32, device=dev)
    dp = lambda x: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_double))  # noqa: E731
    a = prep.args
    a.sc, a.sc_dist, a.global_params, a.regional_params, a.v_list = (dp(keep[k]) for k in ("sc", "dist", "g", "r", "v"))
    a.sc_indices = C.cast(C.c_void_p(keep["sc_idx"].data_ptr()), C.POINTER(C.c_int32))
    out = _abi.Outputs(dp(bold), dp(fc), dp(fcd), dp(states), C.cast(C.c_void_p(gb.data_ptr()), C.POINTER(C.c_uint8)),
                       C.cast(C.c_void_p(gi.data_ptr()), C.POINTER(C.c_int32)), None, None, None, 0.0, 0.0)
    torch.cuda.synchronize(dev)
    if tangent:
        check(L.cbnm_run_tangent_device(C.byref(a), C.byref(out), _ptr(dG)))
    else:
        check(L.cbnm_run_simulations_device(C.byref(a), C.byref(out)))
    return bold, dG


def run_device(args, device="cuda:0"):
    """BOLD [N, bold_len, nodes] (float64 torch tensor on ``device``) of the batch
    given by the reference's 22 run_simulations arguments, inputs and outputs in
    device memory (cbnm_run_simulations_device)."""
    return _device_run(args, device, tangent=False)[0]


def bold_and_dG(args, device="cuda:0"):
    """BOLD and dBOLD/dG of a batch given by the reference's 22 run_simulations
    arguments (host arrays; precision "fp32", model rWW or WC, delays allowed):
    both [N, bold_len, nodes] float64 torch tensors on ``device``.

    The derivative comes from the tangent-linear integrator (forward mode along
    each simulation's G, noise held fixed), so dL/dG of any loss on BOLD is
    ``(dL/dBOLD * dBOLD/dG).sum((1, 2))``, e.g. with the loss kernels::

        bold, dG = bold_and_dG(args)
        lf, ld, db = fit_loss_terms(bold, emp_fc, emp_fcd, remove, ws, step, grad=True)
        dL_dG = (db * dG).sum((1, 2))
    """
    return _device_run(args, device, tangent=True)
