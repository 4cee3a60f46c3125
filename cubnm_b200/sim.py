"""SimGroup classes with the reference's run / score interface.

Restates the parts of src/cubnm/sim/base.py that sit on the simulation path
(``SimGroup.__init__`` settings, ``run`` base.py:673-766, ``_process_out``
:768-818, ``get_noise`` :843-895, ``score`` :1084-1207,
``MultiSimGroupMixin`` :1303-1438), the hooks and result helpers that
``cubnm.optimize.BNMProblem`` and the optimisers call (``_problem_init`` /
``_problem_evaluate`` :1055-1082, ``get_state_averages``, ``get_sim_fc`` /
``get_sim_fcd``, ``slice``, ``clear`` :820-1053) and the per-model parameter
surface of src/cubnm/sim/{rww,wc,jr,kuramoto,rwwex}.py.  Simulations run
through ``cubnm_b200.core.run_simulations``; the goodness-of-fit terms through
the library's GPU kernels.  Plotting / saving helpers (``save``, ``labels``)
are not part of this path.
"""
import copy
import os
from decimal import Decimal

import numpy as np
import pandas as pd

from . import __version__, core, utils

def _load_matrix(m):
    """An SC / distance matrix given as an array or as a .txt / .npy path."""
    if isinstance(m, (str, os.PathLike)):
        m = str(m)
        if m.endswith(".txt"):
            return np.loadtxt(m)
        if m.endswith(".npy"):
            return np.load(m)
        raise ValueError(f"Unsupported matrix file (expected .txt or .npy): {m}")
    return m


WORST_SCORES = {"+fc_corr": -1.0, "-fc_diff": -2.0, "-fc_normec": -1.0, "-fcd_ks": -1.0}


class SimGroup:
    model_name = None
    global_param_names = []
    regional_param_names = []
    state_names = []
    sel_state_var = None
    n_noise = 1
    default_params = {}

    def __init__(self, duration, TR, sc, sc_dist=None, out_dir=None, dt="0.1", bw_dt="1.0", states_ts=False,
                 states_sampling=None, noise_out=False, do_fc=True, do_fcd=True, window_size=30, window_step=5,
                 sim_seed=0, exc_interhemispheric=False, force_cpu=False, force_gpu=False,
                 gof_terms=("+fc_corr", "-fcd_ks"), bw_params="friston2003", bold_remove_s=30,
                 fcd_drop_edges=True, noise_segment_length=30, sim_verbose=False, progress_interval=500,
                 precision="fp64"):
        if force_cpu:
            raise ValueError("force_cpu is not supported: cubnm_b200 runs the simulations on the GPU")
        # the reference's assignment order (base.py:209-286): the property setters
        # below derive and check the millisecond / TR-count values from these
        self.input_sc = sc
        self.sc = np.asarray(_load_matrix(sc), dtype=float)
        self.duration = duration
        self.TR = TR
        self._dt = Decimal(dt)
        self._bw_dt = Decimal(bw_dt)
        self._check_dt()
        self.states_sampling = states_sampling
        self.states_ts = states_ts
        self.gof_terms = list(gof_terms)
        self.do_fc = do_fc
        self.do_fcd = do_fcd
        self.window_size = window_size
        self.window_step = window_step
        self.sim_seed = sim_seed
        self.exc_interhemispheric = exc_interhemispheric
        self.force_cpu = force_cpu
        self.force_gpu = force_gpu
        self.bold_remove_s = bold_remove_s
        self.fcd_drop_edges = fcd_drop_edges
        self.noise_segment_length = noise_segment_length
        self.noise_out = noise_out
        self.sim_verbose = sim_verbose
        self.progress_interval = progress_interval
        self.precision = precision
        self.nodes = self.sc.shape[-1]
        self.input_sc_dist = sc_dist
        if sc_dist is None:
            self.sc_dist = np.zeros((self.nodes, self.nodes))
            self.do_delay = False
        else:
            self.sc_dist = np.asarray(_load_matrix(sc_dist), dtype=float)
            self.do_delay = True
        self.bw_params = bw_params
        self.param_lists = {k: None for k in self.global_param_names + self.regional_param_names + ["v"]}
        # where the reference's save() writes (base.py:269-278); saving is not part of this library
        self.input_out_dir = out_dir
        if out_dir == "same":
            assert isinstance(sc, (str, os.PathLike)), "When `out_dir` is set to 'same' `sc` must be a path-like string"
            self.out_dir = str(sc).replace(".txt", "").replace(".npy", "")
        else:
            self.out_dir = out_dir
        self.last_N = 0
        self.last_config = self.get_config(for_reinit=True)
        self.it = 0
        self._N = 0
        self.post_init()

    def post_init(self):  # base.py:288-294
        """Hook run at the end of __init__ (nothing by default)."""

    # -- properties mirrored from base.py
    @property
    def do_fc(self):
        return self._do_fc

    @do_fc.setter
    def do_fc(self, do_fc):  # base.py:486-496
        if hasattr(self, "gof_terms") and not do_fc and \
                any(t in self.gof_terms for t in ("+fc_corr", "-fc_diff", "-fc_normec")):
            raise ValueError("Cannot calculate FC goodness-of-fit terms without FC."
                             " Set do_fc to True or remove FC-related goodness-of-fit terms.")
        if getattr(self, "_do_fcd", False) and not do_fc:
            raise ValueError("Cannot calculate FCD without FC. Set do_fcd to False.")
        self._do_fc = do_fc

    @property
    def do_fcd(self):
        return self._do_fcd

    @do_fcd.setter
    def do_fcd(self, do_fcd):  # base.py:502-513
        if getattr(self, "_do_fc", False):
            self._do_fcd = do_fcd
        elif do_fcd:
            raise ValueError("Cannot calculate FCD without FC")
        else:
            self._do_fcd = False
        if hasattr(self, "gof_terms") and not self._do_fcd and "-fcd_ks" in self.gof_terms:
            raise ValueError("Cannot calculate FCD goodness-of-fit terms without FCD."
                             " Set do_fcd to True or remove FCD-related goodness-of-fit terms.")

    @property
    def N(self):
        return self._N

    @N.setter
    def N(self, N):
        self._N = N
        if not self.do_delay:
            self.param_lists["v"] = np.zeros(N, dtype=float)

    @property
    def duration(self):
        return self._duration

    @duration.setter
    def duration(self, duration):  # base.py:339-352
        self._duration = duration
        msec = Decimal(duration) * Decimal(1000)
        if msec % 1 != 0:
            raise ValueError(
                f"Duration {duration} seconds equals {msec} milliseconds, which is not a whole number. Duration "
                "must be expressible in whole milliseconds, i.e., must not have more than 3 decimal places.")
        self.duration_msec = int(msec)
        if hasattr(self, "_noise_segment_length") and self.noise_segment_length is None:
            self.noise_segment_length = self.duration

    @property
    def TR(self):
        return self._TR

    @TR.setter
    def TR(self, TR):  # base.py:358-367
        self._TR = TR
        self.TR_msec = int(TR * 1000)
        if hasattr(self, "_states_sampling") and (self.states_sampling is None or self.states_sampling == self.TR):
            self.states_sampling = self.TR
        if hasattr(self, "_window_size"):
            self.window_size_TRs = int(np.round(self.window_size / (self.TR * 2))) * 2
        if hasattr(self, "_window_step"):
            self.window_step_TRs = int(np.round(self.window_step / self.TR))

    @property
    def states_sampling(self):
        return self._states_sampling

    @states_sampling.setter
    def states_sampling(self, states_sampling):  # base.py:373-387
        if states_sampling is not None and states_sampling < 0.001:
            raise ValueError("states_sampling cannot be lower than 0.001s which is model dt")
        self._states_sampling = self.TR if (hasattr(self, "_TR") and states_sampling is None) else states_sampling
        self.states_sampling_msec = int(self.states_sampling * 1000)

    @property
    def noise_segment_length(self):
        return self._noise_segment_length

    @noise_segment_length.setter
    def noise_segment_length(self, noise_segment_length):  # base.py:397-402
        if hasattr(self, "_duration") and noise_segment_length is None:
            self._noise_segment_length = self.duration
        else:
            self._noise_segment_length = noise_segment_length

    @property
    def dt(self):
        return self._dt

    @dt.setter
    def dt(self, dt):  # base.py:408-411
        self._dt = Decimal(dt)
        self._check_dt()

    @property
    def bw_dt(self):
        return self._bw_dt

    @bw_dt.setter
    def bw_dt(self, bw_dt):  # base.py:417-420
        self._bw_dt = Decimal(bw_dt)
        self._check_dt()

    def _check_dt(self):  # base.py:524-535
        assert self.bw_dt >= self.dt, "Ballon-Windkessel dt must be greater than or equal to model dt"
        assert (self.bw_dt % self.dt) == Decimal(0), "Ballon-Windkessel dt must be divisible by model dt"
        assert (self.duration_msec % self.bw_dt) == Decimal(0), "Duration must be divisible by Ballon-Windkessel dt"

    @property
    def bw_params(self):
        return self._bw_params

    @bw_params.setter
    def bw_params(self, bw_params):  # base.py:441-447
        self._bw_params = bw_params
        p = utils.get_bw_params(bw_params)
        for k in ("k1", "k2", "k3"):
            core.set_const(k, p[k])

    @property
    def window_size(self):
        return self._window_size

    @window_size.setter
    def window_size(self, window_size):  # base.py:467-472 (nearest even number of TRs)
        self._window_size = window_size
        self.window_size_TRs = int(np.round(window_size / (self.TR * 2))) * 2

    @property
    def window_step(self):
        return self._window_step

    @window_step.setter
    def window_step(self, window_step):  # base.py:478-481
        self._window_step = window_step
        self.window_step_TRs = int(np.round(window_step / self.TR))

    @property
    def bw_it(self):
        return int(self.duration_msec / self.bw_dt)

    @property
    def inner_it(self):
        return int(self.bw_dt / self.dt)

    @property
    def n_states_samples_remove(self):
        return int(self.bold_remove_s / self.states_sampling)

    @property
    def use_cpu(self):  # base.py:660-671; there is no CPU path here
        return False

    def get_config(self, include_N=False, for_reinit=False):  # base.py:581-633
        """The group's configuration: with `for_reinit` only what requires a new
        session (memory and noise) when it changes, which run() compares."""
        config = {
            "duration": self.duration, "TR": self.TR, "nodes": self.nodes, "states_ts": self.states_ts,
            "states_sampling": self.states_sampling, "do_fc": self.do_fc, "do_fcd": self.do_fcd,
            "window_size": self.window_size, "window_step": self.window_step,
            "window_size_TRs": self.window_size_TRs, "window_step_TRs": self.window_step_TRs,
            "sim_seed": self.sim_seed, "exc_interhemispheric": self.exc_interhemispheric,
            "force_cpu": self.force_cpu, "force_gpu": self.force_gpu, "hardware_used": "gpu",
            "bold_remove_s": self.bold_remove_s, "fcd_drop_edges": self.fcd_drop_edges,
            "noise_segment_length": self.noise_segment_length,
            "precision": self.precision,  # this library's addition
        }
        if not for_reinit:
            config.update({"out_dir": self.input_out_dir, "gof_terms": self.gof_terms, "sc": self.input_sc,
                           "sc_dist": self.input_sc_dist, "bw_params": self.bw_params, "version": __version__})
            if include_N:
                config["N"] = self.N
        return config

    @property
    def _model_config(self):  # base.py:635-657
        return {
            "do_fc": str(int(self.do_fc)),
            "do_fcd": str(int(self.do_fcd)),
            "bold_remove_s": str(self.bold_remove_s),
            "exc_interhemispheric": str(int(self.exc_interhemispheric)),
            "window_size": str(self.window_size_TRs),
            "window_step": str(self.window_step_TRs),
            "drop_edges": str(int(self.fcd_drop_edges)),
            "noise_time_steps": str(int(self.noise_segment_length * 1000)),
            "verbose": str(int(self.sim_verbose)),
            "progress_interval": str(int(self.progress_interval)),
            "precision": self.precision,
        }

    def _set_default_params(self, missing=True):  # base.py:532-575
        defaults = copy.copy(self.default_params)
        if self.do_delay and "v" not in defaults:
            defaults["v"] = 0.5
        for param, v in defaults.items():
            cur = self.param_lists.get(param)
            if (not missing) or cur is None or np.asarray(cur).shape[0] != self.N:
                if v is None:
                    raise ValueError(f"Parameter {param} does not have a default value and must be set")
                if param in self.global_param_names:
                    self.param_lists[param] = np.repeat(v, self.N).astype(float)
                else:  # including the default velocity, (N, nodes) as base.py:567-575; the core reads v[:N]
                    if param == "wIE" and getattr(self, "do_fic", False):
                        continue
                    self.param_lists[param] = np.full((self.N, self.nodes), v, dtype=float)

    def _run_args(self, force_reinit):
        self._global_params = np.vstack(
            [np.ascontiguousarray(self.param_lists[p], dtype=float)[None, :] for p in self.global_param_names])
        self._regional_params = np.vstack(
            [np.ascontiguousarray(np.asarray(self.param_lists[p], dtype=float).flatten()) for p in self.regional_param_names])
        if self.sc.ndim == 2 or self.sc.shape[0] == 1:
            sc = np.ascontiguousarray(self.sc.reshape(-1))[None, :]
            sc_indices = np.zeros(self.N, dtype=np.intc)
        else:
            sc = np.ascontiguousarray(self.sc.reshape(self.sc.shape[0], -1))
            sc_indices = np.ascontiguousarray(np.asarray(self.sc_indices).astype(np.intc))
        return (self.model_name, sc, sc_indices, np.ascontiguousarray(self.sc_dist.flatten()), self._global_params,
                self._regional_params, np.ascontiguousarray(self.param_lists["v"], dtype=float), self._model_config,
                True, self.states_ts, self.noise_out, self.do_delay, force_reinit, False, self.N, self.nodes,
                self.duration_msec, self.TR_msec, self.states_sampling_msec, self.sim_seed, float(self.dt),
                float(self.bw_dt))

    def run(self, force_reinit=False):  # base.py:673-766
        cfg = self.get_config(for_reinit=True)
        force_reinit = force_reinit or (self.N != self.last_N) or (cfg != self.last_config)
        out = core.run_simulations(*self._run_args(force_reinit))
        self.last_N = self.N
        self.last_config = cfg
        self.it += 1
        self._process_out(out)

    def _process_out(self, out):  # base.py:768-818
        self.__dict__.update(out)
        self.sim_bold = self.sim_bold.reshape(self.N, -1, self.nodes)
        self.sim_states = {}
        for i, name in enumerate(self.state_names):
            self.sim_states[name] = self._sim_states[i, :, :]
            if self.states_ts:
                self.sim_states[name] = self.sim_states[name].reshape(self.N, -1, self.nodes)
        if self.do_fc:
            self.sim_fc_trils = self.sim_fc_trils.reshape(self.N, -1)
            if self.do_fcd:
                self.sim_fcd_trils = self.sim_fcd_trils.reshape(self.N, -1)

    def get_noise(self):  # base.py:843-895
        if not self.noise_out:
            raise ValueError("Noise was not saved in the simulation. Set `noise_out` to true and redo the simulation.")
        seg_outer = int(int(self.noise_segment_length * 1000) / self.bw_dt)
        seg = self._noise.reshape(seg_outer, self.inner_it, self.nodes, -1)
        parts = [seg[self._shuffled_ts[r]][:, :, self._shuffled_nodes[r]] for r in range(self._shuffled_nodes.shape[0])]
        return np.concatenate(parts, axis=0)[: self.bw_it].transpose(3, 2, 0, 1)

    def get_state_averages(self):  # base.py:820-841
        """Per-simulation averages of each state variable over time and nodes."""
        avg = {}
        for name in self.state_names:
            v = self.sim_states[name]
            avg[name] = v[:, self.n_states_samples_remove:, :].mean(axis=1).mean(axis=1) if self.states_ts \
                else v.mean(axis=1)
        return pd.DataFrame(avg)

    def get_sim_fc(self, idx):  # base.py:897-942
        """FC of simulation `idx` as a (nodes, nodes) matrix, diagonal 1 (NaN
        between hemispheres when they are excluded)."""
        if not self.do_fc:
            raise ValueError("FC is not calculated in this simulation group")
        if idx >= self.N:
            raise IndexError("Index out of range")
        tril = self.sim_fc_trils[idx]
        fc = np.zeros((self.nodes, self.nodes))
        if self.exc_interhemispheric:
            h = self.nodes // 2
            fc[:h, :h][np.tril_indices(h, -1)] = tril[: tril.shape[0] // 2]
            fc[h:, h:][np.tril_indices(h, -1)] = tril[tril.shape[0] // 2:]
            fc[:h, h:] = np.nan
            fc[h:, :h] = np.nan
        else:
            fc[np.tril_indices(self.nodes, -1)] = tril
        fc += fc.T
        np.fill_diagonal(fc, 1.0)
        return fc

    def get_sim_fcd(self, idx):  # base.py:944-987
        """FCD of simulation `idx` as a (windows, windows) matrix, diagonal 1."""
        if not self.do_fcd:
            raise ValueError("FCD is not calculated in this simulation group")
        if idx >= self.N:
            raise IndexError("Index out of range")
        tril = self.sim_fcd_trils[idx]
        w = (1 + np.sqrt(1 + 8 * tril.shape[0])) / 2  # windows from the pair count
        assert w.is_integer()
        w = int(w)
        fcd = np.zeros((w, w))
        fcd[np.tril_indices(w, -1)] = tril
        fcd += fcd.T
        np.fill_diagonal(fcd, 1.0)
        return fcd

    def slice(self, key, inplace=False):  # base.py:989-1028
        """The group reduced to simulation `key` (a shallow copy unless `inplace`)."""
        if not isinstance(key, int):
            raise ValueError("Only integer indexing is supported")
        if key >= self.N:
            raise IndexError("Index out of range")
        obj = self if inplace else copy.copy(self)
        obj.param_lists = {k: v[key][np.newaxis, ...] for k, v in self.param_lists.items()}
        obj.sim_bold = self.sim_bold[key][np.newaxis, ...]
        obj.sim_states = {k: v[key][np.newaxis, ...] for k, v in self.sim_states.items()}
        if obj.do_fc:
            obj.sim_fc_trils = self.sim_fc_trils[key][np.newaxis, ...]
            if obj.do_fcd:
                obj.sim_fcd_trils = self.sim_fcd_trils[key][np.newaxis, ...]
        obj.N = 1
        return obj

    @property
    def _to_clear(self):  # base.py:1030-1044
        names = ["sim_bold", "sim_fc_trils", "sim_fcd_trils", "sim_states", "_sim_states", "_noise",
                 "_shuffled_nodes", "_shuffled_ts"]
        return [n for n in names if hasattr(self, n)]

    def clear(self):  # base.py:1046-1053
        """Drops the simulation outputs."""
        for name in self._to_clear:
            if hasattr(self, name):
                delattr(self, name)

    def _problem_init(self, problem):  # base.py:1055-1065
        """BNMProblem initialisation hook (nothing by default)."""

    def _problem_evaluate(self, problem, X, out, *args, **kwargs):  # base.py:1067-1082
        """BNMProblem evaluation hook (nothing by default)."""

    def score(self, emp_fc_tril=None, emp_fcd_tril=None, emp_bold=None, force_cpu=False, usable_mem=None):
        """Goodness-of-fit terms per simulation (base.py:1084-1207), computed on the GPU."""
        if emp_bold is not None:
            if self.do_fc:
                emp_fc_tril = utils.calculate_fc(emp_bold, self.exc_interhemispheric, return_tril=True)
            if self.do_fcd:
                emp_fcd_tril = utils.calculate_fcd(emp_bold, self.window_size_TRs, self.window_step_TRs,
                                                   drop_edges=self.fcd_drop_edges,
                                                   exc_interhemispheric=self.exc_interhemispheric,
                                                   return_tril=True, return_dfc=False)
        columns = []
        if self.do_fc and emp_fc_tril is not None:
            columns += [c for c in ["+fc_corr", "-fc_diff", "-fc_normec"] if c in self.gof_terms]
            assert emp_fc_tril.size == self.sim_fc_trils.shape[1], \
                "Empirical FC lower triangle size does not match the simulated FC size"
        if self.do_fcd and emp_fcd_tril is not None:
            columns += [c for c in ["-fcd_ks"] if c in self.gof_terms]
        columns += ["+gof"]
        scores = pd.DataFrame(index=range(self.N), columns=columns, dtype=float)
        want = [c[1:] for c in columns if c != "+gof"]
        res = utils.gof(
            sim_fc_trils=self.sim_fc_trils if self.do_fc and emp_fc_tril is not None else None,
            emp_fc_tril=emp_fc_tril,
            sim_fcd_trils=self.sim_fcd_trils if self.do_fcd and emp_fcd_tril is not None else None,
            emp_fcd_tril=emp_fcd_tril, terms=want)
        sign = {"fc_corr": 1.0, "fc_diff": -1.0, "fc_normec": -1.0, "fcd_ks": -1.0}
        for c in columns:
            if c != "+gof":
                scores.loc[:, c] = sign[c[1:]] * res[c[1:]]
                scores.loc[:, c] = scores.loc[:, c].fillna(WORST_SCORES.get(c, np.nan))
        scores.loc[:, "+gof"] = scores.loc[:, [c for c in self.gof_terms if c in scores.columns]].sum(axis=1)
        return scores


class rWWSimGroup(SimGroup):
    """Reduced Wong-Wang E-I model (src/cubnm/sim/rww.py)."""
    model_name = "rWW"
    global_param_names = ["G"]
    regional_param_names = ["w_p", "J_N", "wIE", "sigma"]
    state_names = ["I_E", "I_I", "r_E", "r_I", "S_E", "S_I"]
    sel_state_var = "r_E"
    n_noise = 2
    default_params = {"G": None, "w_p": 1.4, "J_N": 0.15, "wIE": 1.0, "sigma": 0.01}

    def __init__(self, *args, do_fic=True, max_fic_trials=0, I_SAMPLING_START=1000, I_SAMPLING_END=10000,
                 init_delta=0.02, fic_penalty_scale=0.5, **kwargs):
        self.do_fic = do_fic
        self.max_fic_trials = max_fic_trials
        self.I_SAMPLING_START = I_SAMPLING_START
        self.I_SAMPLING_END = I_SAMPLING_END
        self.init_delta = init_delta
        self.fic_penalty_scale = fic_penalty_scale
        super().__init__(*args, **kwargs)

    @SimGroup.N.setter
    def N(self, N):
        SimGroup.N.fset(self, N)
        if self.do_fic:
            self.param_lists["wIE"] = np.zeros((N, self.nodes), dtype=float)

    def get_config(self, *args, **kwargs):  # rww.py:102-112
        config = super().get_config(*args, **kwargs)
        config.update({"do_fic": self.do_fic, "max_fic_trials": self.max_fic_trials,
                       "I_SAMPLING_START": self.I_SAMPLING_START, "I_SAMPLING_END": self.I_SAMPLING_END,
                       "init_delta": self.init_delta, "fic_penalty_scale": self.fic_penalty_scale})
        return config

    @property
    def _model_config(self):
        cfg = super()._model_config
        cfg.update({"do_fic": str(int(self.do_fic)), "max_fic_trials": str(self.max_fic_trials),
                    "I_SAMPLING_START": str(self.I_SAMPLING_START), "I_SAMPLING_END": str(self.I_SAMPLING_END),
                    "init_delta": str(self.init_delta), "fic_penalty_scale": str(self.fic_penalty_scale)})
        return cfg

    def _process_out(self, out):  # rww.py:170-178
        super()._process_out(out)
        if self.do_fic:
            self.fic_unstable = self._global_bools[0]
            self.fic_failed = self._global_bools[1]
            self.fic_ntrials = self._global_ints[0]
            self.param_lists["wIE"] = self._regional_params[2].reshape(self.N, -1)

    @property
    def _to_clear(self):  # rww.py:153-162
        names = super()._to_clear + ["fic_unstable", "fic_failed", "fic_ntrials"]
        return [n for n in names if hasattr(self, n)]

    def _problem_init(self, problem):  # rww.py:254-271
        """Rejects wIE as a free regional parameter under FIC and adds the FIC
        penalty as an objective of multi-objective problems."""
        if self.do_fic and "wIE" in problem.het_params:
            raise ValueError("In rWW wIE should not be specified as a heterogeneous parameter when FIC is done")
        if problem.multiobj and self.do_fic and self.fic_penalty_scale > 0:
            problem.obj_names.append("-fic_penalty")
            problem.n_obj += 1

    def _problem_evaluate(self, problem, X, out, *args, **kwargs):  # rww.py:273-291
        """Adds the FIC penalty of the last scores to the cost (a column of its
        own for multi-objective problems)."""
        scores = kwargs["scores"][-1]
        if self.do_fic and self.fic_penalty_scale > 0:
            if problem.multiobj:
                out["F"] = np.concatenate([out["F"], -scores.loc[:, ["-fic_penalty"]].values], axis=1)
            else:
                out["F"] -= scores.loc[:, "-fic_penalty"].values

    def score(self, emp_fc_tril=None, emp_fcd_tril=None, emp_bold=None, **kwargs):  # rww.py:180-234
        scores = super().score(emp_fc_tril, emp_fcd_tril, emp_bold, **kwargs)
        if self.do_fic and self.fic_penalty_scale > 0:
            mean_r_E = self.sim_states["r_E"]
            if self.states_ts:
                mean_r_E = mean_r_E[:, self.n_states_samples_remove:].mean(axis=1)
            for idx in range(self.N):
                diff = np.abs(mean_r_E[idx, :] - 3)
                if (diff > 1).sum() > 0:
                    diff[diff <= 1] = np.nan
                    scores.loc[idx, "-fic_penalty"] = (
                        -np.nansum(1 - np.exp(-0.05 * (diff - 1))) * self.fic_penalty_scale / self.nodes)
                else:
                    scores.loc[idx, "-fic_penalty"] = 0
        return scores


class WCSimGroup(SimGroup):
    """Wilson-Cowan E-I model (src/cubnm/sim/wc.py)."""
    model_name = "WC"
    global_param_names = ["G"]
    regional_param_names = ["c_EE", "c_IE", "c_EI", "c_II", "P_E", "P_I", "sigma_E", "sigma_I"]
    state_names = ["E", "I"]
    sel_state_var = "E"
    n_noise = 2
    default_params = {"G": None, "c_EE": 16, "c_IE": 12, "c_EI": 15, "c_II": 3, "P_E": 0.5, "P_I": 0.0,
                      "sigma_E": 5e-05, "sigma_I": 5e-05}


class JRSimGroup(SimGroup):
    """Jansen-Rit model (src/cubnm/sim/jr.py)."""
    model_name = "JR"
    global_param_names = ["G"]
    regional_param_names = ["J", "a_1", "a_2", "a_3", "a_4", "sigma"]
    state_names = ["y0", "y1", "y2", "y3", "y4", "y5", "y1_y2", "s_y1_y2"]
    sel_state_var = "y1_y2"
    n_noise = 1
    default_params = {"G": None, "J": 135.0, "a_1": 1.0, "a_2": 0.8, "a_3": 0.25, "a_4": 0.25, "sigma": 0.0001}


class KuramotoSimGroup(SimGroup):
    """Kuramoto oscillators (src/cubnm/sim/kuramoto.py)."""
    model_name = "Kuramoto"
    global_param_names = ["G"]
    regional_param_names = ["init_theta", "omega", "sigma"]
    state_names = ["theta"]
    sel_state_var = "theta"
    n_noise = 1
    default_params = {"G": None, "init_theta": None, "omega": np.pi, "sigma": 0.17}

    def __init__(self, *args, random_init_theta=True, **kwargs):
        self.random_init_theta = random_init_theta
        super().__init__(*args, **kwargs)

    @SimGroup.N.setter
    def N(self, N):
        SimGroup.N.fset(self, N)
        if self.random_init_theta:  # kuramoto.py:120-133
            rng = np.random.default_rng(self.sim_seed)
            self.param_lists["init_theta"] = np.tile(rng.uniform(0, 2 * np.pi, self.nodes), (N, 1))
        else:
            self.param_lists["init_theta"] = np.zeros((N, self.nodes), dtype=float)

    def get_config(self, *args, **kwargs):  # kuramoto.py:92-97
        config = super().get_config(*args, **kwargs)
        config["random_init_theta"] = self.random_init_theta
        return config

    @property
    def _model_config(self):
        cfg = super()._model_config
        cfg["random_init_theta"] = str(int(self.random_init_theta))
        return cfg


class rWWExSimGroup(SimGroup):
    """Excitatory-only reduced Wong-Wang model (src/cubnm/sim/rwwex.py)."""
    model_name = "rWWEx"
    global_param_names = ["G"]
    regional_param_names = ["w", "I0", "sigma"]
    state_names = ["x", "r", "S"]
    sel_state_var = "r"
    n_noise = 1
    default_params = {"G": None, "w": 0.9, "I0": 0.3, "sigma": 0.001}


class MultiSimGroupMixin:
    """Runs several SimGroups as one launch (base.py:1303-1438)."""

    def __init__(self, sim_groups):
        self.children = sim_groups
        self.__dict__.update(copy.deepcopy({k: v for k, v in sim_groups[0].__dict__.items() if k != "children"}))

    @property
    def N(self):
        return sum(child.N for child in self.children)

    def run(self, **kwargs):
        scs, idx = [], []
        for child in self.children:
            cs = child.sc if child.sc.ndim == 3 else child.sc[None]
            ci = np.zeros(child.N, dtype=int) if cs.shape[0] == 1 else np.asarray(child.sc_indices)
            remap = {}
            for k, m in enumerate(cs):
                hit = [i for i, s in enumerate(scs) if np.allclose(s, m)]
                if hit:
                    remap[k] = hit[0]
                else:
                    scs.append(m)
                    remap[k] = len(scs) - 1
            idx.append(np.array([remap[k] for k in ci], dtype=int))
        self.sc = np.stack(scs) if len(scs) > 1 else scs[0]
        self.sc_indices = np.concatenate(idx)
        for p in self.param_lists:
            self.param_lists[p] = np.concatenate([np.asarray(c.param_lists[p]) for c in self.children])
        self._N = self.N
        SimGroup.run(self, **kwargs)

    def _process_out(self, out):
        start = 0
        for child in self.children:
            end = start + child.N
            child._regional_params = self._regional_params[:, start * child.nodes:end * child.nodes]
            child._global_params = self._global_params[:, start:end]
            oc = {}
            for k, v in out.items():
                if k in ("init_time", "run_time", "_noise", "_shuffled_nodes", "_shuffled_ts"):
                    oc[k] = v
                elif k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils"):
                    oc[k] = v[start:end]
                else:
                    oc[k] = v[:, start:end]
            start = end
            child._process_out(oc)


def create_multi_sim_group(sim_group_cls):
    """MultiSimGroup class for a model's SimGroup (base.py:1440-1461)."""
    return type("MultiSimGroup", (MultiSimGroupMixin, sim_group_cls), {})
