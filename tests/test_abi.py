"""C-ABI library: loads, exports every declared symbol, and its host-side
logic (sizes, config parsing, error behaviour) matches the oracle / the
reference.  No kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cases
from cubnm_b200 import _abi, core
from cubnm_b200._lib import lib
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", name)).read()
            syms |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cbnm_\w+)\s*\(", txt, re.M))
    return sorted(syms)


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert "cbnm_run_simulations" in syms and "cbnm_gof" in syms
    L = lib()
    for s in syms:
        assert hasattr(L, s), f"{s} is declared in include/ but not exported"


def _sizes(L, prefix, args):
    p = _abi.Prepared(*args)
    sz = _abi.Sizes()
    st = getattr(L, prefix + "query_sizes")(C.byref(p.args), C.byref(sz))
    return st, {f: getattr(sz, f) for f, _ in _abi.Sizes._fields_}


@pytest.mark.parametrize("model,delay,fic,kw", [
    ("rWW", 0, 0, {}), ("rWW", 1, 1, {}), ("WC", 0, 0, {"window_size": 10, "window_step": 3}),
    ("JR", 0, 0, {"exc_inter": True}), ("Kuramoto", 0, 0, {"drop_edges": False}),
    ("rWWEx", 0, 0, {"do_fcd": False}), ("rWW", 0, 2, {"bold_remove_s": 0}),
])
def test_sizes_match_oracle(golden, model, delay, fic, kw):
    args = list(cases.golden_args(model, delay, fic, golden=golden))
    cfg = cases.model_config(model, fic, **kw)
    args[7] = cfg
    st1, s1 = _sizes(lib(), "cbnm_", args)
    st2, s2 = _sizes(oracle.lib(), "oracle_", args)
    assert st1 == 0 and st2 == 0
    assert s1 == s2


def test_sizes_of_reference_test_case(golden):
    st, s = _sizes(lib(), "cbnm_", cases.golden_args("rWW", 0, 0, golden=golden))
    assert st == 0
    assert (s["bold_len"], s["n_pairs"], s["n_windows"], s["n_window_pairs"]) == (60, 4950, 10, 45)
    assert s["noise_size"] == 100 * 30000 * 10 * 2 and s["noise_repeats"] == 2


def test_unknown_model_returns_none(golden, capsys):
    args = list(cases.golden_args("rWW", 0, 0, golden=golden))
    args[0] = "NoSuchModel"
    assert core.run_simulations(*args) is None  # core.cpp:271-274
    assert "not found" in capsys.readouterr().err


def test_use_cpu_is_rejected(golden):
    args = list(cases.golden_args("rWW", 0, 0, golden=golden))
    args[13] = True
    with pytest.raises(RuntimeError, match="GPU"):
        core.run_simulations(*args)


def test_config_errors(golden):
    args = list(cases.golden_args("rWW", 0, 0, golden=golden))
    args[7] = cases.model_config("rWW", 0, bold_remove_s=59)     # corr_len 1 < 2
    with pytest.raises(RuntimeError, match="too low"):
        core.run_simulations(*args)
    args[7] = cases.model_config("rWW", 0, window_size=60)       # no window fits (utils.cpp:50-52)
    with pytest.raises(RuntimeError, match="windows is 0"):
        core.run_simulations(*args)
    cfg = cases.model_config("rWW", 0)
    cfg["precision"] = "fp16"
    args[7] = cfg
    with pytest.raises(RuntimeError, match="precision"):
        core.run_simulations(*args)
    args[7] = {"do_fc": 1}
    with pytest.raises(TypeError):
        core.run_simulations(*args)
    # two nodes, one per hemisphere: no FC pair (rejected before any device work)
    two = list(cases.synthetic_args("rWW", N=2, nodes=2, duration_s=60))
    two[7] = dict(two[7], exc_interhemispheric="1")
    with pytest.raises(RuntimeError, match="no node pairs"):
        core.run_simulations(*two)


def test_wrong_argument_count_returns_none(capsys):
    assert core.run_simulations("rWW") is None
    assert "parsing" in capsys.readouterr().err


def test_gof_rejects_fcd_longer_than_the_ks_kernel_holds():
    """The KS kernel sorts one simulation's FCD, padded to a power of two, in
    shared memory; longer FCDs are refused before any device work."""
    from cubnm_b200 import utils
    with pytest.raises(RuntimeError, match=r"FCD too long for the KS kernel: 16385 .*at most 16384"):
        utils.gof(sim_fcd_trils=np.zeros((2, 16385)), emp_fcd_tril=np.zeros(10), terms=["fcd_ks"])


def test_run_batch_argument_errors():
    """An empty batch and a group without the 22 arguments are refused before
    any device work."""
    with pytest.raises(RuntimeError, match="no groups"):
        core.run_batch([])
    with pytest.raises(TypeError, match="22"):
        core.run_batch([("rWW",)])
