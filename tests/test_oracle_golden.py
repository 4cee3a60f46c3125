"""The oracle against the reference's own stored outputs (CPU).

tests/golden/sim_golden.npz holds the reference's tests/expected/sim/*.pkl.gz
(made by its tests/sim/gen_expected.py); the reference checks them at
atol=1e-6 (tests/sim/test.py:104-111).  The oracle is held to that tolerance on
every key its CPU path produced; in practice it reproduces them to ~1e-12.
"""
import numpy as np
import pytest

import cases
from oracle import oracle

CPU_KEYS = [("rWW", d, f) for d in (0, 1) for f in (0, 1, 2)] + [
    (m, d, 0) for m in ("WC", "JR", "Kuramoto", "rWWEx") for d in (0, 1)]

TOL = 1e-6  # tests/sim/test.py:104-111


def _compare(out, golden, model, key):
    sel = cases.MODELS[model][2].index(cases.MODELS[model][3])
    res = {
        "sim_bold": out["sim_bold"].reshape(1, -1, out["_sim_states"].shape[2]),
        "sim_fc_trils": out["sim_fc_trils"],
        "sim_fcd_trils": out["sim_fcd_trils"],
        "sim_sel_state": out["_sim_states"][sel],
    }
    errs = {}
    for k, v in res.items():
        ref = golden[f"{model}|{key}|{k}"]
        assert v.shape == ref.shape, (k, v.shape, ref.shape)
        errs[k] = float(np.abs(v - ref).max())
    return errs


@pytest.mark.parametrize("model,delay,fic", CPU_KEYS)
def test_oracle_matches_reference_cpu_outputs(golden, model, delay, fic):
    out = oracle.run_simulations(*cases.golden_args(model, delay, fic, golden=golden))
    errs = _compare(out, golden, model, cases.golden_key(model, 1, delay, fic))
    assert max(errs.values()) < TOL, errs


def test_oracle_fic_outputs(golden):
    """Analytical + numerical FIC: wIE is written back in place, trial count and flags returned."""
    args = list(cases.golden_args("rWW", 1, 2, golden=golden))
    reg_before = args[5].copy()
    out = oracle.run_simulations(*args)
    assert np.all(reg_before[2] == 0)             # do_fic zeroes wIE in SimGroup (rww.py:163-168)
    assert np.all(args[5][2] > 0)                 # ... and the run writes the FIC wIE back
    assert out["_global_ints"].shape == (1, 1)
    assert out["_global_bools"].shape == (2, 1)
    assert 0 <= out["_global_ints"][0, 0] <= 5


def test_sample_past_the_buffer_is_dropped():
    """bw_dt 0.1 ms, TR 150 ms, 300 s: the truncated counts (base.hpp:51-68)
    give bold_tr_iters = 1499 and 2,001 BOLD samples for a 2,000-volume buffer.
    The sample without a slot is dropped (the reference writes it past the end
    of its buffer); the run completes with finite outputs of the queried size."""
    import ctypes as C
    import cases
    from cubnm_b200 import _abi
    from cubnm_b200._lib import lib
    bw_dt, tr, T = 0.1, 150, 300_000
    tri = int((tr / 1000.0) / (bw_dt / 1000.0))
    bw_it = int((T / 1000.0) / (bw_dt / 1000.0))
    assert (tri, bw_it // tri, T // tr) == (1499, 2001, 2000)
    args = list(cases.synthetic_args("rWW", N=1, nodes=4, duration_s=300, seed=2, window_size=10, window_step=2,
                                     bold_remove_s=30))
    args[9] = True                      # states time series, sampled every TR as well
    args[17], args[18], args[20], args[21] = tr, tr, 0.1, bw_dt
    p = _abi.Prepared(*args)
    sz = _abi.Sizes()
    assert lib().cbnm_query_sizes(C.byref(p.args), C.byref(sz)) == 0
    assert sz.bold_len == 2000 and sz.states_len == 2000
    out = oracle.run_simulations(*args)
    assert out["sim_bold"].shape == (1, 2000 * 4)
    assert np.isfinite(out["sim_bold"]).all() and np.isfinite(out["_sim_states"]).all()
    assert out["_sim_states"].shape == (6, 1, 2000 * 4)


def test_time_shuffle_of_long_noise_segments():
    """A noise segment of 100,000 bw steps (bw_dt 0.1 ms, 10 s): n^2 exceeds the
    32-bit generator range, so libstdc++'s shuffle draws one position per element
    instead of pairs; each repeat's time shuffle is a permutation."""
    args = list(cases.synthetic_args("rWW", N=1, nodes=4, duration_s=12, seed=2, window_size=2, window_step=1,
                                     bold_remove_s=0))
    args[7] = dict(args[7], noise_time_steps="10000")
    args[10] = True                     # noise_out
    args[20], args[21] = 0.1, 0.1
    out = oracle.run_simulations(*args)
    sh = out["_shuffled_ts"]
    assert sh.shape == (2, 100_000)
    for r in range(2):
        assert np.array_equal(np.sort(sh[r]), np.arange(100_000))
    assert not np.array_equal(sh[0], sh[1])
