"""The benchmark's workloads (bench.py --config c0 ... c4) pass the library's own
argument and size checks (cbnm_query_sizes, no GPU needed): every group has BOLD
volumes left after the removed ones and, where FCD is asked for, at least one
pair of windows."""
import ctypes as C

import numpy as np
import pytest

import bench
from cubnm_b200 import _abi
from cubnm_b200._lib import check, lib


def _sizes(args):
    s = _abi.Sizes()
    check(lib().cbnm_query_sizes(C.byref(_abi.Prepared(*args).args), C.byref(s)))
    return s


def test_headline_workload():
    s = _sizes(bench.workload_args(64, bench.DURATION_S, "fp32", 0))
    assert s.bold_len == 60 and s.n_pairs == 4950 and s.n_window_pairs > 0


def test_c0_readme_grid():
    s = _sizes(bench.c0_args())
    assert s.bold_len == 60 and s.n_window_pairs > 0


@pytest.mark.parametrize("scale", [15.0, 30.0])
def test_c2_groups(scale):
    groups = bench.c2_groups(scale, sims_per_group=16)
    assert len(groups) == 16
    for g in groups:
        s = _sizes(g)
        assert s.bold_len >= 2


def test_c3_and_c4():
    sc, a3 = bench.c3_args(16, 300)
    assert sc.shape == (200, 200)
    assert _sizes(a3).n_window_pairs > 0
    for dur in (4, 10):
        s = _sizes(bench.c4_args(16, dur))
        assert s.bold_len == dur


def test_batch_roofline_sums_the_groups():
    groups = bench.c2_groups(15.0, sims_per_group=4)
    r = bench.batch_roofline(groups, 2.0)
    expect = 0.0
    for g in groups:
        n = g[15]
        nnz = np.count_nonzero(np.asarray(g[1]).reshape(n, n)) / n
        expect += g[14] * n * (g[16] / g[20]) * nnz * 4.0
    assert abs(r["algorithmic_bytes"] - expect) <= 1e-9 * expect
    assert abs(r["achieved"] - expect / 2.0 / 1e9) <= 1e-9 * r["achieved"]
    assert r["bound"] == "hbm" and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
