"""Drop-in replacement of the reference's ``cubnm.core`` extension module.

Same three functions, same arguments, same output dict
(reference: src/ext/core.cpp:147-626, imported by src/cubnm/_core.py:9-17):

``run_simulations(model_name, SC, SC_indices, SC_dist, global_params,
regional_params, v_list, model_config, ext_out, states_ts, noise_out, do_delay,
force_reinit, use_cpu, N_SIMS, nodes, time_steps, BOLD_TR, states_sampling,
sim_seed, dt, bw_dt)`` returns a dict with ``init_time``, ``run_time``,
``sim_bold`` (N, bold_len*nodes), ``sim_fc_trils``, ``sim_fcd_trils``,
``_sim_states``, ``_global_bools``, ``_global_ints`` and, with ``noise_out``,
``_noise``, ``_shuffled_nodes``, ``_shuffled_ts``.  Modified parameters (rWW
FIC ``wIE``) are written back into ``regional_params`` in place.

Errors follow the reference: an unknown model prints to stderr and returns
None (core.cpp:271-274); everything else raises RuntimeError, with CUDA
failures prefixed by "CUDA Error".  ``use_cpu=True`` is rejected: this module
has no CPU path.  An extra ``model_config`` key ``"precision"`` selects
``"fp64"`` (default, the reference's precision) or ``"fp32"`` (FP32 node state
with tensor-core coupling).
"""
import ctypes as C
import sys

from . import _abi
from ._lib import lib, check

_CBNM_ERR_MODEL = 2


def init():
    """core.cpp:147-155: reset the Balloon-Windkessel constants."""
    check(lib().cbnm_init())


def set_const(key, value):
    """core.cpp:157-192: set k1, k2, k3 or V_0 of the Balloon-Windkessel model."""
    check(lib().cbnm_set_const(key.encode(), float(value)))


def run_simulations(*args):
    if len(args) != 22:
        print("Error parsing arguments", file=sys.stderr)
        return None
    try:
        return _abi.run(lib(), "cbnm_", *args)
    except RuntimeError as e:
        if str(e).startswith("Model ") and str(e).endswith("not found"):
            print(str(e), file=sys.stderr)
            return None
        raise


def run_batch(groups):
    """Runs several independent groups concurrently on the GPU: ``groups`` is a list
    of 22-argument tuples exactly as for :func:`run_simulations`; returns one
    output dict per group.  Groups may differ in model, node count, duration,
    delays and precision; the outputs equal those of separate calls, and modified
    parameters (rWW FIC) are written back into each group's own arrays."""
    groups = [tuple(g) for g in groups]
    for g in groups:
        if len(g) != 22:
            raise TypeError("every group needs the 22 run_simulations arguments")
    return _abi.run_batch(lib(), groups)


def last_timing():
    """CUDA-event timings (ms) and transfer sizes of the last run."""
    t = _abi.Timing()
    check(lib().cbnm_last_timing(C.byref(t)))
    return {f: getattr(t, f) for f, _ in _abi.Timing._fields_}


def reset():
    """Frees the cached session (device buffers and noise)."""
    check(lib().cbnm_reset())


def last_integrator():
    """Which integrator the last run on this thread used: "fp64", or for precision
    "fp32" one of "tc2", "tc1", "lanes", "lanes512", "simt"."""
    f = lib().cbnm_last_integrator
    f.restype = C.c_char_p
    return f().decode()


def tune_reset():
    """Forgets the autotuner's choices (model_config "autotune" = "1")."""
    check(lib().cbnm_tune_reset())


init()
