"""Multi-GPU host logic (cubnm_b200.shard) on the CPU: shard bounds, argument
slicing and output merging, and a world_size-2 run over torch.distributed
(gloo), with the oracle as each rank's runner.  The merged result must equal
the single-process run of the whole batch, simulation by simulation, and the
FIC write-back must land in the caller's array on every rank."""
import os
import socket
import tempfile

import numpy as np
import pytest

import cases
from cubnm_b200 import shard
from oracle import oracle


def _small_batch(do_fic=1, N=7):
    return list(cases.synthetic_args("rWW", N=N, nodes=12, duration_s=6, seed=3, G=np.linspace(0.2, 3.0, N),
                                     do_fic=do_fic, window_size=2, window_step=1, bold_remove_s=1))


def _assert_same(a, b):
    assert set(a) == set(b)
    for k in a:
        if k in ("init_time", "run_time"):
            continue
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


def test_shard_bounds_counts_and_weights():
    assert shard.shard_bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert shard.shard_bounds(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    # node-steps of simulations with uneven durations: the cut balances them
    w = np.array([900, 60, 60, 60, 300, 300, 600, 600], float)
    b = shard.shard_bounds(len(w), 2, weights=w)
    assert b[0][0] == 0 and b[-1][1] == len(w) and b[0][1] == b[1][0]
    loads = [w[s:e].sum() for s, e in b]
    assert max(loads) - min(loads) <= w.max()
    with pytest.raises(ValueError):
        shard.shard_bounds(4, 0)


def test_slice_and_merge_reproduce_the_whole_batch():
    args = _small_batch()
    whole_args = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    whole = oracle.run_simulations(*whole_args)
    parts = []
    for b, e in shard.shard_bounds(args[14], 3):
        parts.append(oracle.run_simulations(*shard.slice_args(args, b, e)))
    _assert_same(shard.merge_outputs(parts), whole)


def _worker(rank, world, port, path, dst):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        args = _small_batch()
        out = shard.run_sharded(args, runner=oracle.run_simulations, dst=dst)
        slowest = shard.max_over_ranks(float(rank + 1))
        if out is None:
            np.savez(os.path.join(path, f"rank{rank}.npz"), none=1, slowest=slowest)
        else:
            np.savez(os.path.join(path, f"rank{rank}.npz"), wie=args[5][2], slowest=slowest,
                     **{k: np.asarray(v) for k, v in out.items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("dst", [0, None])
def test_run_sharded_over_gloo_world2(dst):
    """dst=0: rank 0 receives the merged batch (and the FIC write-back), rank 1 None;
    dst=None: every rank receives it."""
    import torch.multiprocessing as mp
    args = _small_batch()
    whole = oracle.run_simulations(*args)  # writes the analytical-FIC wIE into args[5]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), d, dst), nprocs=2, join=True, start_method="spawn")
        for r in range(2):
            got = dict(np.load(os.path.join(d, f"rank{r}.npz")))
            assert float(got.pop("slowest")) == 2.0
            if dst is not None and r != dst:
                assert "none" in got
                continue
            np.testing.assert_array_equal(got.pop("wie"), args[5][2])  # FIC write-back
            _assert_same({k: v for k, v in got.items()}, {k: np.asarray(v) for k, v in whole.items()})
