"""Running one batch of simulations across several GPUs (one process per GPU).

Simulations are independent: nothing is exchanged during the time loop, and
the noise array (segment + shuffles) depends only on the seed, the node count
and the duration, not on which simulations a process runs.  So a batch is cut
into contiguous shards of simulations, each rank runs its shard through the
single-GPU entry point on its own device, and the outputs are gathered.  The
gathered result equals the one-GPU result of the whole batch, simulation by
simulation.  The only collectives are the gather of outputs at the end (to one
rank by default) and a MAX of timings; none sits on the data path.

The reference runs a batch on one GPU (src/cubnm/sim/base.py:673-766 calls
cubnm.core.run_simulations once); this module adds the multi-GPU split behind
the same 22 positional arguments.
"""
import numpy as np

# positions of the reference's run_simulations arguments (src/ext/core.cpp:202-225)
A_MODEL, A_SC, A_SC_IDX, A_SC_DIST, A_GLOBAL, A_REGIONAL, A_V = 0, 1, 2, 3, 4, 5, 6
A_N_SIMS, A_NODES, A_TIME_STEPS = 14, 15, 16


def shard_bounds(n_sims, world, weights=None):
    """Contiguous [begin, end) per rank.  With ``weights`` (e.g. nodes x duration of
    each simulation) the cut balances the summed weight; otherwise the counts
    differ by at most one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if weights is None:
        base, extra = divmod(n_sims, world)
        bounds, b = [], 0
        for r in range(world):
            e = b + base + (1 if r < extra else 0)
            bounds.append((b, e))
            b = e
        return bounds
    w = np.asarray(weights, dtype=float)
    if w.shape != (n_sims,):
        raise ValueError("weights must have one entry per simulation")
    cum = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, cum[-1] * r / world, side="left")))
    cuts.append(n_sims)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, n_sims))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def slice_args(args, begin, end):
    """The 22 run_simulations arguments restricted to simulations [begin, end).
    Array arguments are copied (C-contiguous), scalars and the SC stack are shared."""
    a = list(args)
    n, nodes = int(a[A_N_SIMS]), int(a[A_NODES])
    a[A_SC_IDX] = np.ascontiguousarray(np.asarray(args[A_SC_IDX])[begin:end])
    a[A_GLOBAL] = np.ascontiguousarray(np.asarray(args[A_GLOBAL], dtype=float)[:, begin:end])
    reg = np.asarray(args[A_REGIONAL], dtype=float).reshape(-1, n, nodes)
    a[A_REGIONAL] = np.ascontiguousarray(reg[:, begin:end].reshape(reg.shape[0], -1))
    a[A_V] = np.ascontiguousarray(np.asarray(args[A_V], dtype=float)[begin:end])
    a[A_N_SIMS] = end - begin
    return a


# outputs with a simulation axis, and where it is
_SIM_AXIS = {"sim_bold": 0, "sim_fc_trils": 0, "sim_fcd_trils": 0, "_sim_states": 1, "_global_bools": 1,
             "_global_ints": 1}
_SHARED = ("_noise", "_shuffled_nodes", "_shuffled_ts")


def merge_outputs(parts):
    """Concatenates per-shard output dicts (in rank order) into one batch dict."""
    parts = [p for p in parts if p is not None]
    out = {}
    for k in parts[0]:
        if k in _SIM_AXIS:
            out[k] = np.concatenate([p[k] for p in parts], axis=_SIM_AXIS[k])
        elif k in _SHARED:
            out[k] = parts[0][k]
        elif k in ("init_time", "run_time"):
            out[k] = max(p[k] for p in parts)
        else:
            out[k] = parts[0][k]
    return out


def run_sharded(args, runner=None, group=None, weights=None, dst=0):
    """Runs the batch described by the reference's 22 arguments across the ranks of
    ``group`` (torch.distributed must be initialised; each rank on its own GPU).

    The shards' outputs are gathered on rank ``dst`` only (one pickled message per
    other rank), which returns the merged output dict of the whole batch; the other
    ranks return None.  ``dst=None`` gathers on every rank instead.  Parameters the
    run modifies (rWW FIC writes wIE back, src/ext/core.cpp:437-450) are written
    back into ``regional_params`` on the ranks that receive the outputs.
    ``runner`` defaults to :func:`cubnm_b200.core.run_simulations`; it receives
    the shard's 22 arguments.
    """
    import torch.distributed as dist
    if runner is None:
        from . import core
        runner = core.run_simulations
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n, nodes = int(args[A_N_SIMS]), int(args[A_NODES])
    bounds = shard_bounds(n, world, weights)
    b, e = bounds[rank]
    mine = slice_args(args, b, e)
    out = runner(*mine) if e > b else None
    if out is not None:
        out = dict(out)
        out["_regional_params_shard"] = mine[A_REGIONAL]
    if dst is None:
        parts = [None] * world
        dist.all_gather_object(parts, out, group=group)
    else:
        dst_global = dist.get_global_rank(group, dst) if group is not None else dst
        parts = [None] * world if rank == dst else None
        dist.gather_object(out, parts, dst=dst_global, group=group)
        if rank != dst:
            return None
    reg = args[A_REGIONAL]
    if isinstance(reg, np.ndarray) and reg.dtype == np.float64 and reg.flags.c_contiguous:
        full = reg.reshape(-1, n, nodes)
        for (pb, pe), p in zip(bounds, parts):
            if p is not None:
                full[:, pb:pe] = p["_regional_params_shard"].reshape(full.shape[0], pe - pb, nodes)
    for p in parts:
        if p is not None:
            p.pop("_regional_params_shard", None)
    return merge_outputs(parts)


def max_over_ranks(value, group=None, device=None):
    """MAX of a float over the ranks (timings: the slowest rank sets the job time)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
