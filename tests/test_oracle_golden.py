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
