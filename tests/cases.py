"""Argument builders for parity tests.

``golden_args`` reproduces, argument for argument, what the reference's
``SimGroup.run`` (src/cubnm/sim/base.py:673-766) passes to
``cubnm.core.run_simulations`` for the test instance of
``SimGroup._get_test_instance`` (base.py:1267-1301, rww.py:323-345): 60 s,
TR 1 s, window 10 s / step 2 s, G = 0.5, model defaults, dt 0.1 ms without
delay, dt 1.0 ms and v = 0.5 m/s with delay.

``synthetic_args`` builds seeded synthetic inputs with the benchmark's shapes.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sim_golden.npz")

from cubnm_b200.synthetic import (MODELS, base_config, default_params, model_config, rww_grid,  # noqa: E402,F401
                                 synthetic_args, synthetic_emp_bold, synthetic_lengths, synthetic_sc)


def load_golden():
    return np.load(GOLDEN)


def golden_args(model, do_delay, do_fic=0, N=1, G=0.5, golden=None):
    golden = golden if golden is not None else load_golden()
    sc = golden["sc_strength"]
    nodes = sc.shape[0]
    dist = golden["sc_length"] if do_delay else np.zeros_like(sc)
    dt = 1.0 if do_delay else 0.1
    glob, reg = default_params(model, N, nodes, G, do_fic=do_fic)
    v = np.full(N, 0.5) if do_delay else np.zeros(N)
    return (
        model, np.ascontiguousarray(sc.flatten())[None, :], np.repeat(0, N).astype(np.intc),
        np.ascontiguousarray(dist.flatten()), glob, reg, np.ascontiguousarray(v),
        model_config(model, do_fic), True, False, False, bool(do_delay), False, False,
        N, nodes, 60000, 1000, 1000, 0, dt, 1.0,
    )


def golden_key(model, force_cpu, do_delay, do_fic=0):
    key = f"force_cpu:{force_cpu},do_delay:{do_delay}"
    if model == "rWW":
        key += f",do_fic:{do_fic}"
    return key


