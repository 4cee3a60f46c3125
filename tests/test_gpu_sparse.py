"""Sparse (ELLPACK) coupling of the per-simulation kernels, through the C ABI.

Skipping zero SC weights leaves every FP64 sum unchanged (a zero weight adds a
signed zero), and the nonzeros are summed in ascending source order as in the
dense loop, so the FP64 sparse path must be bit-identical to the FP64 dense path
and within the usual bound of the oracle.  CBNM_COUPLING forces either path.
"""
import numpy as np
import pytest

import cases
from cubnm_b200 import core
from oracle import oracle

pytestmark = pytest.mark.gpu

KEYS = ("sim_bold", "sim_fc_trils", "sim_fcd_trils", "_sim_states")


def _sparse_args(model, N, nodes, duration_s, density, delay, precision="fp64", seed=3):
    args = list(cases.synthetic_args(model, N=N, nodes=nodes, duration_s=duration_s, seed=seed, density=density,
                                     G=np.linspace(0.2, 2.0, N), bold_remove_s=duration_s // 4,
                                     window_size=4, window_step=2, precision=precision))
    if delay:
        rng = np.random.default_rng(seed)
        pts = rng.normal(size=(nodes, 3))
        pts = pts / np.linalg.norm(pts, axis=1, keepdims=True) * rng.uniform(0, 70, (nodes, 1))
        args[3] = np.ascontiguousarray((np.linalg.norm(pts[:, None] - pts[None], axis=2) * 1.3).ravel())
        args[6] = np.full(N, 6.0)
        args[11] = True
    return args


def _run(args, monkeypatch, mode):
    monkeypatch.setenv("CBNM_COUPLING", mode)
    return core.run_simulations(*[x.copy() if isinstance(x, np.ndarray) else x for x in args])


@pytest.mark.parametrize("model,delay", [("rWW", False), ("rWW", True), ("WC", True), ("JR", False), ("JR", True),
                                         ("rWWEx", True), ("Kuramoto", False), ("Kuramoto", True)])
def test_fp64_sparse_equals_dense(model, delay, monkeypatch):
    args = _sparse_args(model, 8, 96, 8, 0.1, delay)
    dense, sparse = _run(args, monkeypatch, "dense"), _run(args, monkeypatch, "sparse")
    for k in KEYS:
        np.testing.assert_array_equal(sparse[k], dense[k], err_msg=k)


@pytest.mark.parametrize("model,delay", [("rWW", True), ("WC", False)])
def test_fp64_sparse_matches_oracle(model, delay, monkeypatch):
    args = _sparse_args(model, 6, 80, 10, 0.15, delay)
    got = _run(args, monkeypatch, "sparse")
    ref = oracle.run_simulations(*[x.copy() if isinstance(x, np.ndarray) else x for x in args])
    for k in KEYS:
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-8, atol=1e-12, err_msg=k)


def test_fp32_sparse_within_bounds(monkeypatch):
    args = _sparse_args("rWW", 16, 160, 30, 0.1, True)
    o64 = _run(args, monkeypatch, "sparse")
    a32 = list(args)
    a32[7] = dict(args[7], precision="fp32")
    o32 = _run(a32, monkeypatch, "sparse")
    assert np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max() <= 2e-3


def test_large_sparse_network_wc_1000_nodes(monkeypatch):
    """The shape of the large-network case: Wilson-Cowan, 1,000 nodes, SC at 10%
    density, conduction delays (6 m/s); FP32 vs FP64 on the sparse path."""
    args = _sparse_args("WC", 4, 1000, 10, 0.1, True)
    a64 = list(args)
    o64 = _run(a64, monkeypatch, "auto")
    a32 = list(args)
    a32[7] = dict(args[7], precision="fp32")
    o32 = _run(a32, monkeypatch, "auto")
    assert np.isfinite(o64["sim_bold"]).all()
    assert np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"])) <= 2e-3
