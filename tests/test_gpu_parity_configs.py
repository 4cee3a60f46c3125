"""FP64 parity at the benchmark configurations, the states time series and the
Balloon-Windkessel constants.

* The README grid workload exactly (rWW, 4 x 5 x 5 = 100 simulations over G,
  w_p, J_N; 100 nodes; 60 s at dt 0.1 ms; TR 1 s; FC + FCD window 10 / step 2;
  SC at 30 % density), FIC off and analytical FIC on: FP64 GPU path against the
  oracle on the same inputs and noise, |a - b| <= 1e-8 |b| + 1e-12 for BOLD
  and states and 1e-8 |b| + 1e-10 for FC and FCD (correlations: the absolute
  term covers entries near zero), and every GOF term (through this library's GOF kernels)
  within 1e-8 of scipy's on the oracle's FC / FCD (the reference's CPU GOF,
  src/cubnm/sim/base.py:1176-1189).
* The uneven-batch shapes with conduction delays (6 m/s over tract lengths of
  points in a 70-mm sphere x 1.3, so ring buffers of up to ~300 steps; SC at
  20 %; regional w_p = w_p0 + w_p1 * map) at 100 and 400 nodes, FP64, same bound.
* states_ts = True (states sampled every states_sampling ms,
  src/ext/bnm.cu:377-389): the FP64 kernel against the oracle at the bound
  above; the FP32 per-simulation kernel and the tensor-core kernel against the
  FP64 run.
* set_const (src/ext/core.cpp:157-192): the heinzle2016-3T constants
  (src/cubnm/utils.py:130-160) and a V_0 change, against the oracle with the
  same constants.
All calls go through the C ABI.
"""
import numpy as np
import pytest
import scipy.stats

import cases
from cubnm_b200 import core, utils
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-8, 1e-12
# FC and FCD are correlations (|r| <= 1): entries near zero get an absolute floor,
# since there the relative difference is set by BOLD's last-ulp differences (CUDA's
# and glibc's exp / pow); measured up to 7.4e-12 on 3 of 495,000 README-grid entries
ATOL_R = 1e-10
GOF_ATOL = 1e-8


def _copy(args):
    return [a.copy() if isinstance(a, np.ndarray) else a for a in args]


def _close(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    atol = ATOL_R if what in ("sim_fc_trils", "sim_fcd_trils") else ATOL
    bad = np.abs(a - b) > RTOL * np.abs(b) + atol
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} outside 1e-8 relative; max abs {np.abs(a - b).max():.3e}"


def _compare(o_gpu, o_cpu):
    for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils", "_sim_states"):
        _close(o_gpu[k], o_cpu[k], k)
    np.testing.assert_array_equal(o_gpu["_global_bools"], o_cpu["_global_bools"])
    np.testing.assert_array_equal(o_gpu["_global_ints"], o_cpu["_global_ints"])


def _scipy_gof(fc, fcd, emp_fc, emp_fcd):
    return {
        "fc_corr": np.array([scipy.stats.pearsonr(r, emp_fc).statistic for r in fc]),
        "fc_diff": np.abs(fc.mean(axis=1) - emp_fc.mean()),
        "fc_normec": np.linalg.norm(fc - emp_fc, axis=1) / (2 * np.sqrt(fc.shape[1])),
        "fcd_ks": np.array([scipy.stats.ks_2samp(r, emp_fcd).statistic for r in fcd]),
    }


@pytest.mark.parametrize("do_fic", [0, 1])
def test_readme_grid_fp64_matches_oracle(do_fic):
    G, wp, jn = cases.rww_grid()
    args = list(cases.synthetic_args("rWW", N=100, nodes=100, duration_s=60, seed=0, G=G, w_p=wp, J_N=jn,
                                     do_fic=do_fic, precision="fp64"))
    ga, oa = _copy(args), _copy(args)
    o_gpu = core.run_simulations(*ga)
    o_cpu = oracle.run_simulations(*oa)
    _compare(o_gpu, o_cpu)
    if do_fic:
        _close(ga[5][2], oa[5][2], "wIE written back by the analytical FIC")
    emp = cases.synthetic_emp_bold(100, 60, 7)
    emp_fc = utils.calculate_fc(emp)
    emp_fcd = utils.calculate_fcd(emp, 10, 2)
    g_gpu = utils.gof(o_gpu["sim_fc_trils"], emp_fc, o_gpu["sim_fcd_trils"], emp_fcd)
    g_ref = _scipy_gof(o_cpu["sim_fc_trils"], o_cpu["sim_fcd_trils"], emp_fc, emp_fcd)
    for k, v in g_ref.items():
        ok = np.isfinite(v)
        np.testing.assert_array_equal(np.isfinite(g_gpu[k]), ok)
        err = float(np.abs(g_gpu[k][ok] - v[ok]).max())
        assert err <= GOF_ATOL, (k, err)


def _delayed_args(nodes, N, duration_s, seed, precision="fp64", states_ts=False, states_sampling=1000, window=(4, 2)):
    """Uneven-batch shape with delays: 6 m/s, lengths of points in a 70-mm sphere x 1.3,
    SC at 20 %, regional w_p = w_p0 + w_p1 * map (map ~ N(0, 1) per node)."""
    rng = np.random.default_rng(seed)
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=duration_s, seed=seed, density=0.2,
                                     G=rng.uniform(0.5, 3.0, N), J_N=rng.uniform(0.05, 0.4, N),
                                     precision=precision, window_size=window[0], window_step=window[1],
                                     bold_remove_s=2))
    fmap = np.random.default_rng(seed + 100).standard_normal(nodes)
    wp0, wp1 = rng.uniform(0, 2, N), rng.uniform(-1, 1, N)
    args[5][0] = (wp0[:, None] + wp1[:, None] * fmap[None, :]).ravel()
    args[3] = np.ascontiguousarray(cases.synthetic_lengths(nodes, seed).ravel())
    args[6] = np.full(N, 6.0)
    args[11] = True            # do_delay
    args[9] = states_ts
    args[18] = states_sampling
    return args


@pytest.mark.parametrize("nodes,N,duration_s,window", [(100, 8, 20, (4, 2)), (400, 2, 6, (2, 1))])
def test_delayed_uneven_batch_shapes_fp64_match_oracle(nodes, N, duration_s, window):
    args = _delayed_args(nodes, N, duration_s, seed=nodes, window=window)
    # the longest delay is tens of ms: ring buffers of a few hundred 0.1-ms steps
    steps = np.rint(args[3].max() / (6.0 * 0.1))
    assert steps > 150, steps
    _compare(core.run_simulations(*_copy(args)), oracle.run_simulations(*_copy(args)))


def _states_ts_args(precision, delay):
    if delay:
        return _delayed_args(68, 6, 10, seed=5, precision=precision, states_ts=True, states_sampling=100)
    args = list(cases.synthetic_args("rWW", N=40, nodes=60, duration_s=6, seed=6, precision=precision,
                                     window_size=2, window_step=1, bold_remove_s=1))
    args[9] = True   # states_ts
    args[18] = 100   # a sample every 100 ms
    return args


@pytest.mark.parametrize("delay", [False, True])
def test_states_time_series_fp64_matches_oracle(delay):
    args = _states_ts_args("fp64", delay)
    o_gpu = core.run_simulations(*_copy(args))
    o_cpu = oracle.run_simulations(*_copy(args))
    assert o_gpu["_sim_states"].shape == (6, args[14], args[15] * (args[16] // args[18]))
    _compare(o_gpu, o_cpu)


@pytest.mark.parametrize("kernel", ["tc", "simt"])
def test_states_time_series_fp32_kernels_follow_fp64(kernel, monkeypatch):
    """FP32 state time series against the FP64 run of the same inputs and noise: the
    tensor-core tile kernel (shared SC, no delays) and the FP32 per-simulation kernel
    (forced, and with delays)."""
    if kernel == "simt":
        monkeypatch.setenv("CBNM_FP32_KERNEL", "simt")
    for delay in ([False] if kernel == "tc" else [False, True]):
        o64 = core.run_simulations(*_states_ts_args("fp64", delay))
        o32 = core.run_simulations(*_states_ts_args("fp32", delay))
        s64, s32 = o64["_sim_states"], o32["_sim_states"]
        assert s32.shape == s64.shape
        # per state variable, relative to its range (I_E, I_I in nA; r_E, r_I in Hz; S_E, S_I in [0, 1])
        for v in range(s64.shape[0]):
            scale = max(1.0, float(np.abs(s64[v]).max()))
            err = float(np.abs(s32[v] - s64[v]).max()) / scale
            assert err < 2e-3, (kernel, delay, v, err)
        assert np.abs(o32["sim_bold"] - o64["sim_bold"]).max() < 1e-3


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_set_const_heinzle2016_matches_oracle(precision):
    """set_const k1..k3 (heinzle2016-3T) and V_0 change the BOLD the integrators write,
    exactly as in the oracle; init() restores the defaults."""
    args = list(cases.synthetic_args("rWW", N=6, nodes=40, duration_s=12, seed=8, precision="fp64",
                                     window_size=4, window_step=2, bold_remove_s=2))
    base = core.run_simulations(*_copy(args))
    consts = dict(utils.get_bw_params("heinzle2016-3T"), V_0=0.03)
    try:
        for k, v in consts.items():
            core.set_const(k, v)
            oracle.set_const(k, v)
        o_cpu = oracle.run_simulations(*_copy(args))
        o64 = core.run_simulations(*_copy(args))
        _compare(o64, o_cpu)
        assert np.abs(o64["sim_bold"] - base["sim_bold"]).max() > 1e-3  # the constants matter
        if precision == "fp32":
            a32 = _copy(args)
            a32[7] = dict(args[7], precision="fp32")
            o32 = core.run_simulations(*a32)
            assert np.abs(o32["sim_bold"] - o64["sim_bold"]).max() < 1e-3
            assert np.abs(o32["sim_fc_trils"] - o64["sim_fc_trils"]).max() <= 2e-3
    finally:
        core.init()
        oracle.init()
    again = core.run_simulations(*_copy(args))
    np.testing.assert_array_equal(again["sim_bold"], base["sim_bold"])
