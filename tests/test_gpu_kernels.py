"""The FP32 kernels against each other and against the FP64 path.

* the single-tile tensor-core rWW kernel (default) against the two-tile one
  (CBNM_FP32_TC=pp, or ws for its warp-specialised form) and both against FP64: same bounds as the mixed-precision
  mode (|dFC| <= 2e-3, |dGOF| <= 1e-3), and the two tile forms close to each
  other (they differ only in the FP32 order in which the BF16x3 partial
  products are added);
* the lane kernel (simulations on the lanes; delays and > 128 nodes) against
  the per-simulation FP32 kernel (CBNM_FP32_KERNEL=simt, sparse coupling) on
  the same inputs: the same node-update arithmetic and coupling order, so the
  time-averaged states agree to rounding and the BOLD to the Balloon-Windkessel
  form (series vs pow, a few ulp);
* work distribution: uneven work-item counts (singles and pairs), mixed SCs and
  delay tables, empty lanes.
All calls go through the C ABI.
"""
import numpy as np
import pytest

import cases
from cubnm_b200 import core, utils

pytestmark = pytest.mark.gpu

FC_TOL, GOF_TOL = 2e-3, 1e-3


def _copy(args):
    return [a.copy() if isinstance(a, np.ndarray) else a for a in args]


def _with(args, **cfg):
    a = _copy(args)
    a[7] = dict(args[7], **cfg)
    return a


def _gof(o, nodes, vols, window, step):
    emp = cases.synthetic_emp_bold(nodes, vols, 7)
    return utils.gof(o["sim_fc_trils"], utils.calculate_fc(emp), o["sim_fcd_trils"],
                     utils.calculate_fcd(emp, window, step))


def _bounds(o64, o32, nodes, vols, window=10, step=2):
    dfc = float(np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"])))
    g64, g32 = _gof(o64, nodes, vols, window, step), _gof(o32, nodes, vols, window, step)
    dg = max(float(np.nanmax(np.abs(g64[k] - g32[k]))) for k in g64)
    assert dfc <= FC_TOL and dg <= GOF_TOL, (dfc, dg)
    return dfc, dg


@pytest.mark.parametrize("N", [5, 96, 200, 700])
def test_two_tile_kernel_matches_single_tile_and_fp64(N, monkeypatch):
    """N = 5 (one single), 96 (a pair and a single), 200 / 700 (pairs split into
    singles to fill every CTA): every simulation must come out."""
    nodes = 100
    args = cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=16, seed=N, window_size=4, window_step=2,
                                bold_remove_s=4)
    o64 = core.run_simulations(*_with(args, precision="fp64"))
    v5 = core.run_simulations(*_with(args, precision="fp32"))
    assert core.last_integrator() == "tc1"
    monkeypatch.setenv("CBNM_FP32_TC", "pp")
    pp = core.run_simulations(*_with(args, precision="fp32"))
    assert core.last_integrator() == "tc2"
    monkeypatch.setenv("CBNM_FP32_TC", "ws")
    ws = core.run_simulations(*_with(args, precision="fp32"))
    assert core.last_integrator() == "tc2ws"
    monkeypatch.delenv("CBNM_FP32_TC")
    assert np.isfinite(pp["sim_bold"]).all()
    _bounds(o64, pp, nodes, 16, 4, 2)
    _bounds(o64, v5, nodes, 16, 4, 2)
    # the two two-tile forms run the same arithmetic in the same order
    np.testing.assert_array_equal(ws["sim_bold"], pp["sim_bold"])
    np.testing.assert_array_equal(ws["_sim_states"], pp["_sim_states"])
    assert np.abs(pp["sim_bold"] - v5["sim_bold"]).max() < 1e-4
    np.testing.assert_allclose(pp["_sim_states"], v5["_sim_states"], rtol=1e-3, atol=1e-4)


@pytest.mark.parametrize("tc", ["v5", "pp"])
def test_tile_kernels_mixed_scs_and_128_nodes(tc, monkeypatch):
    """Simulations over three SCs interleaved (tiles / pairs within an SC only), 128
    nodes (every TMEM lane live; the two-tile kernel's state sums no longer fit in
    shared memory)."""
    N, nodes = 150, 128
    scs = np.stack([cases.synthetic_sc(nodes, 0.3, s).reshape(-1) for s in range(3)])
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=12, seed=5, window_size=4, window_step=2,
                                     bold_remove_s=2))
    args[1] = scs
    args[2] = (np.arange(N) % 3).astype(np.intc)
    o64 = core.run_simulations(*_with(args, precision="fp64"))
    monkeypatch.setenv("CBNM_FP32_TC", tc)
    o32 = core.run_simulations(*_with(args, precision="fp32"))
    assert core.last_integrator() == ("tc1" if tc == "v5" else "tc2")
    _bounds(o64, o32, nodes, 12, 4, 2)
    np.testing.assert_allclose(o32["_sim_states"], o64["_sim_states"], rtol=2e-3, atol=2e-3)


def _delayed(model, nodes, N, duration_s, seed, density=0.2, v=6.0, window=(4, 2)):
    args = list(cases.synthetic_args(model, N=N, nodes=nodes, duration_s=duration_s, seed=seed, density=density,
                                     G=np.linspace(0.2, 2.0, N), window_size=window[0], window_step=window[1],
                                     bold_remove_s=2))
    args[3] = np.ascontiguousarray(cases.synthetic_lengths(nodes, seed).ravel())
    args[6] = np.full(N, v)
    args[11] = True
    return args


@pytest.mark.parametrize("model,nodes,N,delay", [("rWW", 100, 40, True), ("rWW", 400, 20, True),
                                                 ("WC", 300, 18, True), ("rWWEx", 68, 33, True),
                                                 ("rWW", 200, 24, False), ("JR", 160, 17, True)])
def test_lane_kernel_matches_per_simulation_kernel(model, nodes, N, delay, monkeypatch):
    args = _delayed(model, nodes, N, 10, seed=nodes) if delay else list(
        cases.synthetic_args(model, N=N, nodes=nodes, duration_s=10, seed=nodes, density=0.25, window_size=4,
                             window_step=2, bold_remove_s=2))
    monkeypatch.setenv("CBNM_FP32_KERNEL", "lanes")
    lanes = core.run_simulations(*_with(args, precision="fp32"))
    assert core.last_integrator() == "lanes"
    monkeypatch.setenv("CBNM_FP32_KERNEL", "simt")
    monkeypatch.setenv("CBNM_COUPLING", "sparse")
    simt = core.run_simulations(*_with(args, precision="fp32"))
    assert np.isfinite(lanes["sim_bold"]).all()
    np.testing.assert_allclose(lanes["_sim_states"], simt["_sim_states"], rtol=1e-5, atol=1e-7)
    scale = np.abs(simt["sim_bold"]).max()
    assert np.abs(lanes["sim_bold"] - simt["sim_bold"]).max() <= 1e-6 * scale
    np.testing.assert_allclose(lanes["sim_fc_trils"], simt["sim_fc_trils"], rtol=0, atol=1e-4)


def test_lane_kernel_mixed_velocities_and_scs(monkeypatch):
    """Groups are formed per (SC, delay table): two SCs x three velocities, with a
    count that leaves partly empty groups."""
    monkeypatch.setenv("CBNM_FP32_KERNEL", "lanes")
    N, nodes = 45, 80
    args = _delayed("rWW", nodes, N, 10, seed=8)
    args[1] = np.stack([cases.synthetic_sc(nodes, 0.2, s).reshape(-1) for s in (8, 9)])
    args[2] = (np.arange(N) % 2).astype(np.intc)
    args[6] = np.array([3.0, 6.0, 12.0])[np.arange(N) % 3]
    o64 = core.run_simulations(*_with(args, precision="fp64"))
    o32 = core.run_simulations(*_with(args, precision="fp32"))
    _bounds(o64, o32, nodes, 10, 4, 2)


@pytest.mark.parametrize("nodes,N", [(100, 48), (400, 16)])
def test_lane_kernel_uneven_batch_shapes_within_bounds(nodes, N, monkeypatch):
    """The uneven-batch shapes (delays up to ~30 ms at 6 m/s, SC 20 %) in FP32
    against FP64 on the same noise."""
    monkeypatch.setenv("CBNM_FP32_KERNEL", "lanes")
    args = _delayed("rWW", nodes, N, 20 if nodes == 100 else 8, seed=nodes,
                    window=(4, 2) if nodes == 100 else (2, 1))
    o64 = core.run_simulations(*_with(args, precision="fp64"))
    o32 = core.run_simulations(*_with(args, precision="fp32"))
    _bounds(o64, o32, nodes, 20 if nodes == 100 else 8, *((4, 2) if nodes == 100 else (2, 1)))


@pytest.mark.parametrize("kernel", ["lanes", "simt"])
def test_large_sparse_wilson_cowan(kernel, monkeypatch):
    """1,000 nodes at 10 % with delays (the large-network shape), FP32 vs FP64, on
    the lane kernel and the per-simulation kernel (the default)."""
    monkeypatch.setenv("CBNM_FP32_KERNEL", kernel)
    N, nodes = 4, 1000
    args = _delayed("WC", nodes, N, 8, seed=4, density=0.1, window=(2, 1))
    reg = args[5].reshape(8, N, nodes)
    reg[6] = reg[7] = 0.01
    o64 = core.run_simulations(*_with(args, precision="fp64"))
    o32 = core.run_simulations(*_with(args, precision="fp32"))
    assert np.abs(o64["sim_bold"] - o32["sim_bold"]).max() < 1e-3
    assert np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"])) <= FC_TOL
