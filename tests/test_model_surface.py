"""The models' parameter / variable surface against the reference's
code-generation recipes (``codegen/recipes/*.yaml``, recorded in
``tests/golden/model_surface.json`` by ``tests/golden/make_model_surface.py``).

The reference generates its SimGroup classes and kernels from those recipes;
here the SimGroup classes of ``cubnm_b200.sim`` and the library's size query
(state variables, parameters and global outputs per model, the C ABI's
``cbnm_query_sizes``) must expose the same names, order, counts and defaults.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

import cases
from cubnm_b200 import _abi, sim
from cubnm_b200._lib import lib

SURFACE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "model_surface.json")))
CLASSES = {"rWW": sim.rWWSimGroup, "WC": sim.WCSimGroup, "JR": sim.JRSimGroup, "Kuramoto": sim.KuramotoSimGroup,
           "rWWEx": sim.rWWExSimGroup}


def _default(text):
    return None if text is None else (np.pi if text == "np.pi" else float(text))


@pytest.mark.parametrize("model", sorted(CLASSES))
def test_simgroup_surface_equals_recipe(model):
    ref, cls = SURFACE[model], CLASSES[model]
    assert cls.model_name == model
    assert cls.state_names == ref["state_vars"]
    assert cls.global_param_names == ref["global_params"]
    assert cls.regional_param_names == ref["regional_params"]
    assert cls.n_noise == len(ref["noise"])
    assert cls.sel_state_var == ref["sel_state_var"]
    for p in ref["global_params"]:
        assert cls.default_params[p] is None  # G has no default (base.py:569-573)
    for p, text in ref["regional_defaults"].items():
        assert cls.default_params[p] == _default(text), p


@pytest.mark.parametrize("model", sorted(CLASSES))
def test_library_sizes_equal_recipe(model):
    ref = SURFACE[model]
    args = list(cases.synthetic_args(model, N=3, nodes=10, duration_s=10, seed=0, window_size=4, window_step=2,
                                     bold_remove_s=2))
    L = lib()
    p = _abi.Prepared(*args)
    sz = _abi.Sizes()
    assert L.cbnm_query_sizes(C.byref(p.args), C.byref(sz)) == 0, L.cbnm_last_error().decode()
    assert sz.n_global_params == len(ref["global_params"])
    assert sz.n_regional_params == len(ref["regional_params"])
    assert sz.n_state_vars == len(ref["state_vars"])
    assert sz.n_global_out_bool == len(ref["global_out_bool"])
    assert sz.n_global_out_int == len(ref["global_out_int"])
