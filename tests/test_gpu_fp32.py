"""FP32 / tensor-core path against the FP64 path on the same inputs and noise.

Bounds (stated for the mixed-precision mode): |dFC| <= 2e-3 and |dGOF| <= 1e-3
against the FP64 run of the same seeded noise, for every term.
All calls go through the C ABI.
"""
import numpy as np
import pytest

import cases
from cubnm_b200 import core, utils

pytestmark = pytest.mark.gpu

FC_TOL = 2e-3
GOF_TOL = 1e-3


def _pair(args):
    a64 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a32 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a64[7] = dict(args[7], precision="fp64")
    a32[7] = dict(args[7], precision="fp32")
    return core.run_simulations(*a64), core.run_simulations(*a32)


def _gof_err(o64, o32, nodes, vols, window=10, seed=7):
    emp = cases.synthetic_emp_bold(nodes, vols, seed)
    efc = utils.calculate_fc(emp)
    efcd = utils.calculate_fcd(emp, window, 2)
    g64 = utils.gof(o64["sim_fc_trils"], efc, o64["sim_fcd_trils"], efcd)
    g32 = utils.gof(o32["sim_fc_trils"], efc, o32["sim_fcd_trils"], efcd)
    return {k: float(np.nanmax(np.abs(g64[k] - g32[k]))) for k in g64}


def test_rww_readme_grid_within_bounds():
    """4x5x5 grid over G, w_p, J_N, 100 nodes, 60 s, FC + FCD w10/s2."""
    G, wp, jn = cases.rww_grid()
    args = cases.synthetic_args("rWW", N=100, nodes=100, duration_s=60, seed=0, G=G, w_p=wp, J_N=jn)
    o64, o32 = _pair(args)
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, 100, 60)
    assert max(errs.values()) <= GOF_TOL, errs
    # BOLD and time-averaged states track closely too
    assert np.abs(o64["sim_bold"] - o32["sim_bold"]).max() < 1e-3
    np.testing.assert_allclose(o32["_sim_states"], o64["_sim_states"], rtol=1e-3, atol=1e-3)


@pytest.mark.parametrize("model", ["WC", "rWWEx"])
def test_other_models_within_bounds(model):
    N, nodes = 32, 68
    G = np.linspace(0.1, 2.0, N)
    args = cases.synthetic_args(model, N=N, nodes=nodes, duration_s=40, seed=4, G=G, window_size=10, window_step=2,
                                bold_remove_s=10)
    o64, o32 = _pair(args)
    dfc = np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]))
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, nodes, 40)
    assert max(errs.values()) <= GOF_TOL, errs


def test_jr_short_horizon():
    """Jansen-Rit at these couplings is chaotic: an FP64 run perturbed by 1e-9 diverges
    exponentially (BOLD difference 1e-11 -> 1e-5 over 40 s), so pointwise FC bounds do not
    apply over long runs.  Over the first 5 s the FP32 BOLD follows the FP64 BOLD."""
    N, nodes = 32, 68
    args = cases.synthetic_args("JR", N=N, nodes=nodes, duration_s=5, seed=4, G=np.linspace(0.1, 2.0, N),
                                window_size=2, window_step=1, bold_remove_s=1)
    o64, o32 = _pair(args)
    scale = np.abs(o64["sim_bold"]).max()
    assert np.abs(o64["sim_bold"] - o32["sim_bold"]).max() < 1e-4 * scale


def test_mixed_sc_tiles_and_partial_tile():
    """Simulations using three different SCs, interleaved, with N not a multiple of the tile."""
    N, nodes = 37, 48
    scs = np.stack([cases.synthetic_sc(nodes, 0.3, s).reshape(-1) for s in range(3)])
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=40, seed=2, G=np.linspace(0.5, 4, N),
                                     bold_remove_s=10))
    args[1] = scs
    args[2] = (np.arange(N) % 3).astype(np.intc)
    o64, o32 = _pair(args)
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc


def _with_delay(args, nodes, velocity=6.0, seed=0):
    """Tract lengths from points in a 70-mm sphere x 1.3, one conduction velocity (m/s)."""
    a = list(args)
    rng = np.random.default_rng(seed)
    pts = rng.normal(size=(nodes, 3))
    pts = pts / np.linalg.norm(pts, axis=1, keepdims=True) * rng.uniform(0, 70, (nodes, 1))
    dist = np.linalg.norm(pts[:, None] - pts[None], axis=2) * 1.3
    a[3] = np.ascontiguousarray(dist.ravel())
    a[6] = np.full(a[14], velocity)
    a[11] = True
    return tuple(a)


@pytest.mark.parametrize("model", ["rWW", "WC", "rWWEx"])
def test_delays_in_fp32(model):
    """Conduction delays run on the FP32 per-simulation kernel (ring buffers in FP32)."""
    N, nodes = 32, 68
    args = cases.synthetic_args(model, N=N, nodes=nodes, duration_s=40, seed=4, G=np.linspace(0.1, 2.0, N),
                                bold_remove_s=10)
    o64, o32 = _pair(_with_delay(args, nodes))
    dfc = np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]))
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, nodes, 40)
    assert max(errs.values()) <= GOF_TOL, errs


def test_jr_delay_short_horizon():
    N, nodes = 32, 68
    args = cases.synthetic_args("JR", N=N, nodes=nodes, duration_s=5, seed=4, G=np.linspace(0.1, 2.0, N),
                                window_size=2, window_step=1, bold_remove_s=1)
    o64, o32 = _pair(_with_delay(args, nodes))
    scale = np.abs(o64["sim_bold"]).max()
    assert np.abs(o64["sim_bold"] - o32["sim_bold"]).max() < 1e-4 * scale


def test_numerical_fic_in_fp32():
    """Numerical FIC (restart with adjusted wIE) in FP32: same trial counts and
    failure flags as FP64, wIE and FC close."""
    N, nodes = 16, 68
    args = cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=40, seed=5, G=np.linspace(0.5, 3, N), do_fic=2,
                                bold_remove_s=10)
    a64 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a32 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a64[7] = dict(args[7], precision="fp64")
    a32[7] = dict(args[7], precision="fp32")
    o64, o32 = core.run_simulations(*a64), core.run_simulations(*a32)
    assert o64["_global_ints"].max() > 0  # some simulations needed FIC trials
    np.testing.assert_array_equal(o32["_global_ints"], o64["_global_ints"])
    np.testing.assert_array_equal(o32["_global_bools"], o64["_global_bools"])
    np.testing.assert_allclose(a32[5][2], a64[5][2], rtol=1e-6, atol=1e-9)  # wIE written back
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc


@pytest.mark.parametrize("nodes", [200, 400])
def test_large_networks_in_fp32(nodes):
    """More nodes than TMEM lanes: the FP32 per-simulation kernel."""
    N = 32
    args = cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=40, seed=6, G=np.linspace(0.5, 3, N),
                                bold_remove_s=10)
    o64, o32 = _pair(args)
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, nodes, 40)
    assert max(errs.values()) <= GOF_TOL, errs


def test_per_simulation_kernel_on_readme_grid(monkeypatch):
    """CBNM_FP32_KERNEL=simt sends a shared-SC batch to the FP32 per-simulation
    kernel instead of the tensor-core tiles: same bounds."""
    monkeypatch.setenv("CBNM_FP32_KERNEL", "simt")
    G, wp, jn = cases.rww_grid()
    args = cases.synthetic_args("rWW", N=100, nodes=100, duration_s=60, seed=0, G=G, w_p=wp, J_N=jn)
    o64, o32 = _pair(args)
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, 100, 60)
    assert max(errs.values()) <= GOF_TOL, errs


def test_analytical_fic_in_fp32(golden):
    """Analytical FIC runs on the host before either integrator: same wIE in both modes."""
    args = list(cases.golden_args("rWW", 0, 1, N=4, golden=golden))
    args[4] = np.array([[0.2, 0.5, 1.0, 1.5]])
    o64, o32 = _pair(args)
    dfc = np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]).max()
    assert dfc <= FC_TOL, dfc


def test_kuramoto_in_fp32():
    """Kuramoto in FP32 mode: phase, frequency and noise scale in double, the coupling
    sum of sines in FP32.  Without delays it holds the FC / GOF bounds over 40 s."""
    N, nodes = 32, 68
    args = cases.synthetic_args("Kuramoto", N=N, nodes=nodes, duration_s=40, seed=4, G=np.linspace(0.1, 2.0, N),
                                bold_remove_s=10)
    o64, o32 = _pair(args)
    dfc = np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"]))
    assert dfc <= FC_TOL, dfc
    errs = _gof_err(o64, o32, nodes, 40)
    assert max(errs.values()) <= GOF_TOL, errs


def test_kuramoto_delay_no_worse_than_input_rounding():
    """Kuramoto with delays is chaotic: the reference's own CPU and GPU outputs
    agree to 4e-13 at 1 s and differ by 4e-4 at 2 s.  Pointwise bounds do not
    apply; instead the FP32 run may be no further from the FP64 run than an FP64
    run whose SC is perturbed by 1e-7 (relative, the size of FP32 rounding) is,
    up to a factor of 10, at every BOLD volume of the first 2 s (sampled every
    100 ms)."""
    N, nodes = 16, 68
    args = list(cases.synthetic_args("Kuramoto", N=N, nodes=nodes, duration_s=2, seed=4, G=np.linspace(0.1, 2.0, N),
                                     window_size=4, window_step=2, bold_remove_s=0))
    args[17] = 100  # BOLD_TR (ms)
    args[18] = 100  # states_sampling (ms)
    args = _with_delay(tuple(args), nodes)
    o64, o32 = _pair(args)
    pert = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    pert[1] = pert[1] * (1.0 + 1e-7)
    pert[7] = dict(args[7], precision="fp64")
    op = core.run_simulations(*pert)
    b64 = o64["sim_bold"].reshape(N, -1, nodes)
    e32 = np.abs(o32["sim_bold"].reshape(N, -1, nodes) - b64).max(axis=(0, 2))
    ep = np.abs(op["sim_bold"].reshape(N, -1, nodes) - b64).max(axis=(0, 2))
    scale = np.abs(b64).max()
    assert np.all(e32 <= 10 * ep + 1e-6 * scale), (e32, ep)
