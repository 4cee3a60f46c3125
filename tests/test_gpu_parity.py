"""GPU parity of the FP64 path (the reference's precision).

* against the reference's own stored outputs (tests/golden): within
  |a-b| <= 1e-8 |b| + 1e-12 wherever the reference's own CPU and GPU outputs
  agree to that bound (rWW, rWWEx, Kuramoto without delays); for WC and JR,
  whose stored CPU and GPU outputs differ by up to 3e-6 (last-ulp differences
  of exp amplified over 60 s), at atol 1e-6 as tests/sim/test.py:104-111
  checks them;
* against the oracle on the same inputs and noise: BOLD, FC, FCD within
  1e-8 relative (|a-b| <= 1e-8 |b| + 1e-12), states likewise;
* noise and shuffles bit-exact with the oracle;
* GOF terms within 1e-8 of scipy (the reference's CPU GOF, base.py:1176-1189).
All calls go through the C ABI (ctypes over libcubnm_b200.so).
"""
import numpy as np
import pytest
import scipy.stats

import cases
from cubnm_b200 import core, utils
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-8, 1e-12       # FP64 mode vs the oracle
GOLDEN_TOL = 1e-6              # reference's own test tolerance

ALL_KEYS = [("rWW", d, f) for d in (0, 1) for f in (0, 1, 2)] + [
    (m, d, 0) for m in ("WC", "JR", "Kuramoto", "rWWEx") for d in (0, 1)]


def _res(out, model, nodes=100):
    sel = cases.MODELS[model][2].index(cases.MODELS[model][3])
    return {
        "sim_bold": out["sim_bold"].reshape(out["sim_bold"].shape[0], -1, nodes),
        "sim_fc_trils": out["sim_fc_trils"],
        "sim_fcd_trils": out["sim_fcd_trils"],
        "sim_sel_state": out["_sim_states"][sel],
    }


def _golden_param(m, d, f):
    if m == "Kuramoto" and d:
        # chaotic: last-ulp differences between CUDA's and glibc's sin grow to O(1); the
        # reference marks its own CPU-vs-GPU comparison of this case as a known issue
        # (issue #24, tests/sim/test.py:54-59).  Short-horizon parity with the oracle
        # is checked in test_fp64_kuramoto_delay_short_horizon instead.
        return pytest.param(m, d, f, marks=pytest.mark.xfail(reason="reference issue #24 (chaotic)", strict=False))
    return pytest.param(m, d, f)


def _reference_self_consistent(golden, model, delay, fic):
    """True where the reference's stored CPU and GPU outputs agree to the strict bound."""
    for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils", "sim_sel_state"):
        a = golden[f"{model}|{cases.golden_key(model, 1, delay, fic)}|{k}"]
        b = golden[f"{model}|{cases.golden_key(model, 0, delay, fic)}|{k}"]
        if (np.abs(a - b) > RTOL * np.abs(b) + ATOL).any():
            return False
    return True


@pytest.mark.parametrize("model,delay,fic", [_golden_param(*k) for k in ALL_KEYS])
def test_fp64_matches_reference_outputs(golden, model, delay, fic):
    out = core.run_simulations(*cases.golden_args(model, delay, fic, golden=golden))
    res = _res(out, model)
    strict = _reference_self_consistent(golden, model, delay, fic)
    if model in ("rWW", "rWWEx") or (model == "Kuramoto" and not delay):
        assert strict  # the stored outputs themselves agree at 1e-8 relative
    for force_cpu in (1, 0):
        if model == "Kuramoto" and delay and force_cpu == 0:
            continue  # the reference's own CPU and GPU disagree here (issue #24, tests/sim/test.py:54-59)
        key = cases.golden_key(model, force_cpu, delay, fic)
        for k, v in res.items():
            ref = golden[f"{model}|{key}|{k}"]
            if strict:
                _assert_close(v, ref, f"{key} {k}")
            else:
                err = float(np.abs(v - ref).max())
                assert err < GOLDEN_TOL, (key, k, err)


def _assert_close(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = np.abs(a - b) > RTOL * np.abs(b) + ATOL
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} outside rtol {RTOL}; max abs diff {np.abs(a - b).max():.3e}"


def _compare_all(o1, o2, model):
    for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils", "_sim_states"):
        _assert_close(o1[k], o2[k], k)
    np.testing.assert_array_equal(o1["_global_ints"], o2["_global_ints"])
    np.testing.assert_array_equal(o1["_global_bools"], o2["_global_bools"])


@pytest.mark.parametrize("model", ["rWW", "WC", "JR", "rWWEx"])
def test_fp64_matches_oracle_batch(model):
    """A batch of simulations with different parameters, 20 s, synthetic SC."""
    N, nodes = 12, 64
    G = np.linspace(0.5, 3.0, N)
    args = list(cases.synthetic_args(model, N=N, nodes=nodes, duration_s=20, G=G, seed=3, window_size=4,
                                     window_step=2, bold_remove_s=4))
    if model == "rWW":
        args[5][0] = np.repeat(np.linspace(0.2, 1.6, N), nodes)   # w_p
        args[5][1] = np.repeat(np.linspace(0.05, 0.4, N), nodes)  # J_N
    o_gpu = core.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    o_cpu = oracle.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    _compare_all(o_gpu, o_cpu, model)


def test_fp64_matches_oracle_fic_and_delay(golden):
    """Analytical + numerical FIC with conduction delays and heterogeneous velocities."""
    N = 4
    args = list(cases.golden_args("rWW", 1, 2, N=N, golden=golden))
    args[4] = np.array([[0.3, 0.5, 0.8, 1.2]])
    args[6] = np.array([0.5, 1.0, 2.5, 1.0])
    args[7] = cases.model_config("rWW", 2, bold_remove_s=10)
    args[16] = 30000
    ga = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    oa = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    o_gpu = core.run_simulations(*ga)
    o_cpu = oracle.run_simulations(*oa)
    _compare_all(o_gpu, o_cpu, "rWW")
    _assert_close(ga[5], oa[5], "written-back regional params (wIE)")


def test_gpu_analytical_fic_matches_oracle():
    """Analytical FIC runs on the GPU (one thread per node, the Brent iteration of
    the host code); wIE and the failure flags equal the oracle's host FIC, including
    simulations where it fails: with J_N < -1.62 the steady-state equation has no
    root in [0, 2], and the simulation gets wIE = 1 in every node."""
    N, nodes = 48, 68
    rng = np.random.default_rng(9)
    J_N = np.concatenate([rng.uniform(0.001, 0.5, N - 6), np.full(6, -2.0)])
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=2, seed=9, G=np.linspace(0.001, 10, N),
                                     w_p=rng.uniform(0, 2, N), J_N=J_N, do_fic=1, do_fc=False, do_fcd=False,
                                     bold_remove_s=0))
    ga = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    oa = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    o_gpu = core.run_simulations(*ga)
    o_cpu = oracle.run_simulations(*oa)
    np.testing.assert_array_equal(o_gpu["_global_bools"][0], o_cpu["_global_bools"][0])
    assert o_cpu["_global_bools"][0].sum() >= 1 and o_cpu["_global_bools"][0].sum() < N
    np.testing.assert_allclose(ga[5][2], oa[5][2], rtol=1e-12, atol=0)
    np.testing.assert_allclose(o_gpu["sim_bold"], o_cpu["sim_bold"], rtol=1e-8, atol=1e-12)


def test_fp64_kuramoto_matches_oracle():
    N, nodes = 3, 32
    args = list(cases.synthetic_args("Kuramoto", N=N, nodes=nodes, duration_s=12, G=np.array([0.2, 1.0, 4.0]),
                                     seed=5, window_size=4, window_step=2, bold_remove_s=2))
    _compare_all(core.run_simulations(*args), oracle.run_simulations(*args), "Kuramoto")


def test_fp64_kuramoto_delay_short_horizon(golden):
    """Kuramoto with delays against the oracle over the first second.  The system is
    chaotic (the reference's own CPU and GPU outputs agree to 4e-13 at 1 s and differ
    by 4e-4 at 2 s), so parity is checked before last-ulp sin differences grow."""
    args = list(cases.golden_args("Kuramoto", 1, 0, golden=golden))
    args[7] = cases.model_config("Kuramoto", 0, do_fc=False, do_fcd=False)
    args[16] = 1000
    args[17] = 100
    args[18] = 100
    o_gpu = core.run_simulations(*args)
    o_cpu = oracle.run_simulations(*args)
    _assert_close(o_gpu["sim_bold"], o_cpu["sim_bold"], "sim_bold")


def test_identical_sims_are_identical(golden):
    """tests/sim/test.py:113-146: two identical simulations in one launch."""
    out = core.run_simulations(*cases.golden_args("rWW", 0, 1, N=2, golden=golden))
    for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils"):
        np.testing.assert_array_equal(out[k][0], out[k][1])


def test_noise_bit_exact_and_reconstructable():
    """Noise, shuffles (tests/sim/test.py:188-259 configuration)."""
    from cubnm_b200 import sim
    nodes = 10
    sc = np.ones((nodes, nodes))
    np.fill_diagonal(sc, 0)
    sg = sim.rWWSimGroup(duration=8, noise_segment_length=3, TR=0.1, dt="0.2", bw_dt="0.8", sc=sc, do_fc=False,
                         do_fcd=False, gof_terms=[], noise_out=True)
    sg.N = 1
    sg.param_lists["G"] = np.array([0.5])
    sg._set_default_params(missing=True)
    sg.run()
    args = list(sg._run_args(False))
    ref = oracle.run_simulations(*args)
    np.testing.assert_array_equal(sg._noise, ref["_noise"])
    np.testing.assert_array_equal(sg._shuffled_nodes, ref["_shuffled_nodes"])
    np.testing.assert_array_equal(sg._shuffled_ts, ref["_shuffled_ts"])
    recon = sg.get_noise()
    mimic = np.empty_like(recon)
    noise_bw_it = int(3000 / 0.8)
    sh_ts, sh_nodes = sg._shuffled_ts.flatten(), sg._shuffled_nodes.flatten()
    rep = 0
    for bw_i in range(sg.bw_it):
        t = sh_ts[(bw_i % noise_bw_it) + rep * noise_bw_it]
        for inner in range(sg.inner_it):
            for j in range(nodes):
                idx = (t * sg.inner_it + inner) * nodes * 2 + sh_nodes[rep * nodes + j] * 2
                mimic[0, j, bw_i, inner] = sg._noise[idx]
                mimic[1, j, bw_i, inner] = sg._noise[idx + 1]
        if (bw_i + 1) % noise_bw_it == 0 and bw_i + 1 < sg.bw_it:
            rep += 1
    np.testing.assert_array_equal(recon, mimic)


def test_gof_matches_scipy():
    """tests/utils/test.py: fc_corr vs pearsonr, fcd_ks vs ks_2samp; plus fc_diff, fc_normec."""
    rng = np.random.default_rng(0)
    sim_fc = rng.random((100, 4950)) * 2 - 1
    emp_fc = rng.random(4950) * 2 - 1
    sim_fcd = rng.random((1000, 300)) * 2 - 1
    emp_fcd = rng.random(500) * 2 - 1
    corr = utils.fc_corr_device(sim_fc, emp_fc)
    ks = utils.fcd_ks_device(sim_fcd, emp_fcd)
    ref_corr = np.array([scipy.stats.pearsonr(s, emp_fc).statistic for s in sim_fc])
    ref_ks = np.array([scipy.stats.ks_2samp(s, emp_fcd).statistic for s in sim_fcd])
    np.testing.assert_allclose(corr, ref_corr, rtol=1e-8, atol=1e-12)
    # the reference divides counts by sample sizes (utils.py:26-61); scipy 1.18 multiplies by 1/n
    np.testing.assert_allclose(ks, ref_ks, rtol=1e-12, atol=0)
    g = utils.gof(sim_fc, emp_fc, terms=["fc_diff", "fc_normec"])
    np.testing.assert_allclose(g["fc_diff"], np.abs(sim_fc.mean(1) - emp_fc.mean()), rtol=1e-8, atol=1e-14)
    np.testing.assert_allclose(g["fc_normec"], np.linalg.norm(sim_fc - emp_fc, axis=1) / (2 * np.sqrt(4950)),
                               rtol=1e-8)


def test_gof_ties_and_nan():
    """KS with ties between and within samples; a NaN row scores NaN (base.py:1202-1204 maps it later)."""
    rng = np.random.default_rng(1)
    sim_fcd = np.round(rng.random((64, 45)) * 10) / 10
    emp_fcd = np.round(rng.random(300) * 10) / 10
    sim_fcd[3, 5] = np.nan
    ks = utils.fcd_ks_device(sim_fcd, emp_fcd)
    for i in range(64):
        if i == 3:
            assert np.isnan(ks[i])
        else:
            assert abs(ks[i] - scipy.stats.ks_2samp(sim_fcd[i], emp_fcd).statistic) < 1e-12


def test_simgroup_score_end_to_end():
    """SimGroup.run + score on the GPU against scipy on the same FC/FCD."""
    from cubnm_b200 import sim
    sc = cases.synthetic_sc(40, 0.3, 0)
    emp_bold = cases.synthetic_emp_bold(40, 60, 1)
    sg = sim.rWWSimGroup(duration=60, TR=1, sc=sc, window_size=10, window_step=2, do_fic=False,
                         gof_terms=["+fc_corr", "-fc_diff", "-fc_normec", "-fcd_ks"])
    sg.N = 6
    sg.param_lists["G"] = np.linspace(0.5, 4, 6)
    sg._set_default_params()
    sg.run()
    sc_df = sg.score(emp_bold=emp_bold)
    emp_fc = utils.calculate_fc(emp_bold)
    emp_fcd = utils.calculate_fcd(emp_bold, 10, 2)
    for i in range(6):
        assert abs(sc_df.loc[i, "+fc_corr"] - scipy.stats.pearsonr(sg.sim_fc_trils[i], emp_fc).statistic) < 1e-8
        assert abs(sc_df.loc[i, "-fcd_ks"] + scipy.stats.ks_2samp(sg.sim_fcd_trils[i], emp_fcd).statistic) < 1e-12
    gof = sc_df[["+fc_corr", "-fc_diff", "-fc_normec", "-fcd_ks"]].sum(axis=1)
    np.testing.assert_allclose(sc_df["+gof"], gof)
