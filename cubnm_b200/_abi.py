"""ctypes mirror of include/cubnm_b200.h and the run_simulations calling convention.

The reference's boundary is ``cubnm.core.run_simulations`` (src/ext/core.cpp:194-493):
22 positional arguments in, a dict of numpy arrays out, parameters written back
in place when the model modifies them (rWW FIC, core.cpp:437-450).  This module
turns those arguments into a ``cbnm_run_args`` struct, asks the library for the
output sizes, allocates the numpy outputs and builds the same dict.
"""
import ctypes as C
import time

import numpy as np


class RunArgs(C.Structure):
    _fields_ = [
        ("model_name", C.c_char_p),
        ("sc", C.POINTER(C.c_double)),
        ("n_scs", C.c_int),
        ("sc_indices", C.POINTER(C.c_int32)),
        ("sc_dist", C.POINTER(C.c_double)),
        ("global_params", C.POINTER(C.c_double)),
        ("regional_params", C.POINTER(C.c_double)),
        ("v_list", C.POINTER(C.c_double)),
        ("config_keys", C.POINTER(C.c_char_p)),
        ("config_values", C.POINTER(C.c_char_p)),
        ("n_config", C.c_int),
        ("ext_out", C.c_int),
        ("states_ts", C.c_int),
        ("noise_out", C.c_int),
        ("do_delay", C.c_int),
        ("force_reinit", C.c_int),
        ("use_cpu", C.c_int),
        ("n_sims", C.c_int),
        ("nodes", C.c_int),
        ("time_steps", C.c_int),
        ("bold_tr", C.c_int),
        ("states_sampling", C.c_int),
        ("sim_seed", C.c_int),
        ("dt", C.c_double),
        ("bw_dt", C.c_double),
    ]


class Sizes(C.Structure):
    _fields_ = [
        ("n_global_params", C.c_int),
        ("n_regional_params", C.c_int),
        ("n_state_vars", C.c_int),
        ("n_global_out_bool", C.c_int),
        ("n_global_out_int", C.c_int),
        ("bold_len", C.c_int),
        ("n_pairs", C.c_int),
        ("n_windows", C.c_int),
        ("n_window_pairs", C.c_int),
        ("states_len", C.c_int),
        ("do_fc", C.c_int),
        ("do_fcd", C.c_int),
        ("modifies_params", C.c_int),
        ("noise_repeats", C.c_int),
        ("noise_bw_it", C.c_int),
        ("noise_size", C.c_int64),
    ]


class Outputs(C.Structure):
    _fields_ = [
        ("sim_bold", C.POINTER(C.c_double)),
        ("sim_fc_trils", C.POINTER(C.c_double)),
        ("sim_fcd_trils", C.POINTER(C.c_double)),
        ("sim_states", C.POINTER(C.c_double)),
        ("global_bools", C.POINTER(C.c_uint8)),
        ("global_ints", C.POINTER(C.c_int32)),
        ("noise", C.POINTER(C.c_double)),
        ("shuffled_nodes", C.POINTER(C.c_int32)),
        ("shuffled_ts", C.POINTER(C.c_int32)),
        ("init_time", C.c_double),
        ("run_time", C.c_double),
    ]


class Timing(C.Structure):
    _fields_ = [
        ("integrate_ms", C.c_double),
        ("fc_ms", C.c_double),
        ("h2d_ms", C.c_double),
        ("d2h_ms", C.c_double),
        ("total_ms", C.c_double),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("kernel_launches", C.c_int),
    ]


def _ptr(arr, ctype):
    if arr is None:
        return None
    return arr.ctypes.data_as(C.POINTER(ctype))


def declare(lib, prefix):
    """Attach argtypes/restype for the run/query/init/set_const/last_error family."""
    getattr(lib, prefix + "query_sizes").argtypes = [C.POINTER(RunArgs), C.POINTER(Sizes)]
    getattr(lib, prefix + "query_sizes").restype = C.c_int
    getattr(lib, prefix + "run_simulations").argtypes = [C.POINTER(RunArgs), C.POINTER(Outputs)]
    getattr(lib, prefix + "run_simulations").restype = C.c_int
    getattr(lib, prefix + "init").argtypes = []
    getattr(lib, prefix + "init").restype = C.c_int
    getattr(lib, prefix + "set_const").argtypes = [C.c_char_p, C.c_double]
    getattr(lib, prefix + "set_const").restype = C.c_int
    getattr(lib, prefix + "last_error").argtypes = []
    getattr(lib, prefix + "last_error").restype = C.c_char_p


class Prepared:
    """Arguments of one run_simulations call converted to C, with the arrays kept alive."""

    def __init__(self, model_name, SC, SC_indices, SC_dist, global_params, regional_params, v_list,
                 model_config, ext_out, states_ts, noise_out, do_delay, force_reinit, use_cpu,
                 N_SIMS, nodes, time_steps, BOLD_TR, states_sampling, sim_seed, dt, bw_dt):
        # core.cpp:230-237 converts params/SC to C-contiguous double arrays; the
        # write-back of modified parameters (core.cpp:437-450) lands in the caller's
        # array only when no conversion copy was needed -- same here.
        self.global_params = np.require(global_params, np.float64, ["C"])
        self.regional_params = np.require(regional_params, np.float64, ["C"])
        self.SC = np.require(SC, np.float64, ["C"])
        if self.SC.ndim == 1:
            self.SC = self.SC[None, :]
        self.SC_indices = np.require(SC_indices, np.int32, ["C"])
        self.SC_dist = np.require(SC_dist, np.float64, ["C"])
        self.v_list = np.require(v_list, np.float64, ["C"])
        if not isinstance(model_config, dict):
            raise TypeError("Parameter must be a dictionary.")
        for k, v in model_config.items():
            if not isinstance(k, str) or not isinstance(v, str):
                raise TypeError("Dictionary keys and values must be strings.")
        keys = [k.encode() for k in model_config]
        vals = [v.encode() for v in model_config.values()]
        self._keys = (C.c_char_p * max(1, len(keys)))(*keys)
        self._vals = (C.c_char_p * max(1, len(vals)))(*vals)
        self._name = model_name.encode()
        # N_SCs is max(SC_indices)+1 in the reference (core.cpp:238-242)
        n_scs = int(self.SC_indices.max()) + 1 if self.SC_indices.size else 1
        if self.SC.shape[0] < n_scs:
            raise ValueError("SC has fewer matrices than SC_indices refers to")
        self.args = RunArgs(
            self._name, _ptr(self.SC, C.c_double), n_scs, _ptr(self.SC_indices, C.c_int32),
            _ptr(self.SC_dist, C.c_double), _ptr(self.global_params, C.c_double),
            _ptr(self.regional_params, C.c_double), _ptr(self.v_list, C.c_double),
            self._keys, self._vals, len(keys), int(ext_out), int(states_ts), int(noise_out),
            int(do_delay), int(force_reinit), int(use_cpu), int(N_SIMS), int(nodes), int(time_steps),
            int(BOLD_TR), int(states_sampling), int(sim_seed), float(dt), float(bw_dt),
        )
        self.N = int(N_SIMS)
        self.nodes = int(nodes)
        self.ext_out = bool(ext_out)
        self.states_ts = bool(states_ts)
        self.noise_out = bool(noise_out)


class _Pending:
    """One run's C structs and the numpy outputs they point into."""

    def __init__(self, lib, prefix, args):
        self.p = p = Prepared(*args)
        self.sizes = sizes = Sizes()
        st = getattr(lib, prefix + "query_sizes")(C.byref(p.args), C.byref(sizes))
        if st != 0:
            raise RuntimeError(getattr(lib, prefix + "last_error")().decode())
        N, n = p.N, p.nodes
        self.bold = np.empty((N, sizes.bold_len * n), dtype=np.float64)
        self.fc = np.empty((N, sizes.n_pairs), dtype=np.float64) if sizes.do_fc else None
        self.fcd = np.empty((N, sizes.n_window_pairs), dtype=np.float64) if sizes.do_fcd else None
        ext = n * (sizes.states_len if p.states_ts else 1)
        self.states = np.empty((sizes.n_state_vars, N, ext), dtype=np.float64) if p.ext_out else None
        self.gbools = np.zeros((sizes.n_global_out_bool, N), dtype=np.uint8)
        self.gints = np.zeros((sizes.n_global_out_int, N), dtype=np.int32)
        self.noise = self.sh_nodes = self.sh_ts = None
        if p.noise_out:
            self.noise = np.empty(sizes.noise_size, dtype=np.float64)
            self.sh_nodes = np.empty((sizes.noise_repeats, n), dtype=np.int32)
            self.sh_ts = np.empty((sizes.noise_repeats, sizes.noise_bw_it), dtype=np.int32)
        self.out = Outputs(
            _ptr(self.bold, C.c_double), _ptr(self.fc, C.c_double), _ptr(self.fcd, C.c_double),
            _ptr(self.states, C.c_double), _ptr(self.gbools, C.c_uint8), _ptr(self.gints, C.c_int32),
            _ptr(self.noise, C.c_double), _ptr(self.sh_nodes, C.c_int32), _ptr(self.sh_ts, C.c_int32), 0.0, 0.0,
        )

    def result(self, wall):
        out, sizes, p = self.out, self.sizes, self.p
        res = {
            "init_time": float(out.init_time),
            "run_time": float(out.run_time) if out.run_time > 0 else wall,
            "sim_bold": self.bold,
        }
        if sizes.do_fc:
            res["sim_fc_trils"] = self.fc
            if sizes.do_fcd:
                res["sim_fcd_trils"] = self.fcd
        if p.ext_out:
            res["_sim_states"] = self.states
            res["_global_bools"] = self.gbools.astype(bool)
            res["_global_ints"] = self.gints
        if p.noise_out:
            res["_noise"] = self.noise
            res["_shuffled_nodes"] = self.sh_nodes
            res["_shuffled_ts"] = self.sh_ts
        return res


def run(lib, prefix, *args):
    """Calls ``<prefix>run_simulations`` and returns the reference's output dict."""
    pend = _Pending(lib, prefix, args)
    t0 = time.perf_counter()
    st = getattr(lib, prefix + "run_simulations")(C.byref(pend.p.args), C.byref(pend.out))
    t1 = time.perf_counter()
    if st != 0:
        raise RuntimeError(getattr(lib, prefix + "last_error")().decode())
    return pend.result(t1 - t0)


def run_batch(lib, groups):
    """Calls ``cbnm_run_batch`` on a list of 22-argument tuples; returns one
    output dict per group (the same dicts as :func:`run`)."""
    pends = [_Pending(lib, "cbnm_", g) for g in groups]
    n = len(pends)
    args = (RunArgs * n)(*[q.p.args for q in pends])
    outs = (Outputs * n)(*[q.out for q in pends])
    statuses = (C.c_int * n)()
    f = lib.cbnm_run_batch
    f.argtypes = [C.POINTER(RunArgs), C.POINTER(Outputs), C.c_int, C.POINTER(C.c_int)]
    f.restype = C.c_int
    t0 = time.perf_counter()
    st = f(args, outs, n, statuses)
    t1 = time.perf_counter()
    if st != 0:
        raise RuntimeError(lib.cbnm_last_error().decode())
    for i, q in enumerate(pends):  # the library filled the structs of the array (init / run times)
        q.out = outs[i]
    return [q.result(t1 - t0) for q in pends]
