"""Records the arguments the reference's ``SimGroup.run()`` hands to its compiled
core, for the CPU test of ``cubnm_b200.sim`` (``tests/test_sim_marshalling.py``).

Run once, in a checkout that has the reference next to it:

    python tests/golden/make_simgroup_args.py /path/to/cubnm

It imports the reference's Python package (``src/cubnm``) with its compiled
extension replaced by a recorder: ``cubnm._core.run_simulations`` stores its 22
positional arguments (``src/cubnm/sim/base.py:727-750``) and stops the run, and
``cubnm._setup_opts`` (written by the reference's build) is given the flags of a
regular NVIDIA GPU build (no many-nodes mode); every group is made with
``force_gpu=True``.  Nothing is simulated.

Each case of ``CASES``, ``MULTI``, ``MUTATED`` (settings changed after
construction) and ``RANDOM`` (60 seeded random groups) below is built through
``build(simmod, case)`` for any module with the reference's SimGroup classes,
so the test builds the same groups with ``cubnm_b200.sim``.

The cases of ``SCORE_CASES`` are run once more with the recorder answering
``fake_outputs()`` (no simulation: seeded arrays of the output shapes), then
scored by the reference's ``score()`` against ``empirical()``; with no CuPy the
reference computes every term on the CPU with scipy (``base.py:1163-1188``).

``UTIL_CASES`` records the reference's empirical helpers
(``src/cubnm/utils.py:130-304``: ``get_bw_params``, ``calculate_fc``,
``calculate_fcd``) on seeded BOLD arrays with zeroed (outlier) volumes,
inter-hemispheric exclusion, edge windows kept and windows dropped as outliers.

Output: ``tests/golden/simgroup_args.npz`` with, per case, the array arguments
as ``<case>|<index>``, the rest as JSON in ``<case>|meta``, and for the scored
groups ``<case>|<child>|score|<column>`` plus the processed rWW FIC outputs.
"""
import hashlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "simgroup_args.npz")
NODES = 10
ARRAY_ARGS = (1, 2, 3, 4, 5, 6)  # sc, sc_indices, sc_dist, global, regional, v


def _sc(seed, nodes=NODES):
    rng = np.random.default_rng(seed)
    w = np.triu(rng.lognormal(0.0, 1.0, (nodes, nodes)) * (rng.random((nodes, nodes)) < 0.4), 1)
    w = w + w.T
    return w / w.sum(axis=1).mean()


def _dist(seed, nodes=NODES):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(-50, 50, (nodes, 3))
    return np.linalg.norm(pts[:, None] - pts[None], axis=2) * 1.3


# name: (class, constructor kwargs, N, parameters, extra attributes)
CASES = {
    "rww_fic": ("rWWSimGroup", dict(duration=60, TR=1, window_size=10, window_step=2), 3,
                {"G": [0.5, 1.0, 2.0]}, {}),
    "rww_delay": ("rWWSimGroup", dict(duration=20, TR=0.5, dt="0.1", bw_dt="0.5", states_ts=True, noise_out=True,
                                      do_fic=False, bold_remove_s=2, window_size=5, window_step=1, sim_seed=7,
                                      noise_segment_length=10, gof_terms=["+fc_corr", "-fc_diff", "-fcd_ks"],
                                      sc_dist="dist"), 4,
                  {"G": [0.1, 0.2, 0.3, 0.4], "w_p": "per_node", "v": [1.0, 2.0, 3.0, 4.0]}, {}),
    "rww_numfic": ("rWWSimGroup", dict(duration=30, TR=1, do_fic=True, max_fic_trials=5, fcd_drop_edges=False,
                                       exc_interhemispheric=False), 2, {"G": [0.3, 0.6], "J_N": [0.12, 0.2]}, {}),
    "wc": ("WCSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2), 2,
           {"G": [0.5, 1.5]}, {}),
    "jr": ("JRSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2, do_fcd=False,
                                   gof_terms=["+fc_corr"]), 2,
           {"G": [1.0, 2.0]}, {}),
    "kuramoto": ("KuramotoSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2,
                                          sim_seed=3), 2, {"G": [0.2, 0.4]}, {}),
    "rwwex": ("rWWExSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2,
                                    do_fc=False, do_fcd=False, gof_terms=[]), 2, {"G": [0.2, 0.4]}, {}),
    "rww_hemi": ("rWWSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2,
                                     exc_interhemispheric=True, states_ts=True, fic_penalty_scale=1.0), 3,
                 {"G": [0.2, 0.4, 0.6]}, {}),
    "wc_delay_default_v": ("WCSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2,
                                              sc_dist="dist"), 2, {"G": [0.5, 1.5]}, {}),
    "rww_child": ("rWWSimGroup", dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2,
                                      do_fic=False), 2, {"G": [0.2, 0.4]}, {}),
}

# groups of children run as one (MultiSimGroupMixin): (case, SC seed, N) per child;
# the third child repeats the first one's SC
MULTI = {
    "rww_multi": ("rWWSimGroup", [("rww_child", 1, 2), ("rww_child", 2, 3), ("rww_child", 1, 1)]),
}


def build(simmod, name, sc_seed=1, N=None):
    """The SimGroup of case `name` (of ``CASES`` or ``MULTI``), from the classes
    of module `simmod`, with N and its parameters set and the defaults filled in."""
    if name in RANDOM:
        return build_random(simmod, name)
    if name in RANDOM_SCORE:
        cls, kw, N = RANDOM_SCORE[name]
        sg = getattr(simmod, cls)(**dict(kw, force_gpu=True, sc=_sc(1)))
        sg.N = N
        sg.param_lists["G"] = np.linspace(0.1, 1, N)
        sg._set_default_params()
        return sg
    if name in MUTATED:
        base, changes = MUTATED[name]
        sg = build(simmod, base)
        for k, v in changes:
            setattr(sg, k, v)
        return sg
    if name in MULTI:
        cls, children = MULTI[name]
        kids = [build(simmod, c, seed, n) for c, seed, n in children]
        return simmod.create_multi_sim_group(getattr(simmod, cls))(kids)
    cls, kw, n_default, params, extra = CASES[name]
    N = n_default if N is None else N
    kw = dict(kw, force_gpu=True)  # the GPU path, whether or not this host has a GPU
    kw["sc"] = _sc(sc_seed)
    if kw.get("sc_dist") == "dist":
        kw["sc_dist"] = _dist(5)
    sg = getattr(simmod, cls)(**kw)
    sg.N = N
    rng = np.random.default_rng(11 + sc_seed)
    for p, v in params.items():
        if isinstance(v, str):
            sg.param_lists[p] = rng.uniform(0.5, 1.5, (N, sg.nodes))
        else:
            v = np.resize(np.asarray(v, dtype=float), N)
            if p in sg.regional_param_names:
                v = np.repeat(v[:, None], sg.nodes, axis=1)
            sg.param_lists[p] = v
    for k, v in extra.items():
        setattr(sg, k, np.asarray(v))
    sg._set_default_params()
    return sg


def random_cases(n=60, seed=5):
    """n seeded random groups over model, TR, windows, dt, sampling, noise segment,
    delays and FIC options: {name: (class, constructor kwargs, N)}, JSON-able
    (sc_dist given as the flag "dist")."""
    rng = np.random.default_rng(seed)
    out = {}
    for i in range(n):
        cls = str(rng.choice(["rWWSimGroup", "WCSimGroup", "JRSimGroup", "KuramotoSimGroup", "rWWExSimGroup"]))
        kw = dict(duration=int(rng.choice([10, 30, 60])), TR=float(rng.choice([0.5, 0.72, 1, 2])),
                  window_size=int(rng.choice([4, 10, 30])), window_step=int(rng.choice([1, 2, 5])),
                  bold_remove_s=int(rng.choice([0, 2, 5])), dt=str(rng.choice(["0.1", "0.5", "1.0"])), bw_dt="1.0",
                  sim_seed=int(rng.integers(0, 5)), states_ts=bool(rng.integers(0, 2)),
                  noise_out=bool(rng.integers(0, 2)), noise_segment_length=[None, 5, 30][int(rng.integers(0, 3))],
                  fcd_drop_edges=bool(rng.integers(0, 2)))
        if rng.random() < 0.3:
            kw["states_sampling"] = float(rng.choice([0.5, 1, 2]))
        if cls == "rWWSimGroup":
            kw["do_fic"] = bool(rng.integers(0, 2))
            kw["max_fic_trials"] = int(rng.choice([0, 3]))
        if rng.random() < 0.3:
            kw["sc_dist"] = "dist"
        out[f"random_{i:02d}"] = (cls, kw, int(rng.integers(1, 4)))
    return out


RANDOM = random_cases()


def random_score_cases(n=20, seed=9):
    """n seeded random rWW / WC groups for scoring: random subsets of the GOF
    terms, FIC penalty scales, state time series and hemisphere exclusion."""
    rng = np.random.default_rng(seed)
    terms_all = ["+fc_corr", "-fc_diff", "-fc_normec", "-fcd_ks"]
    out = {}
    for i in range(n):
        cls = str(rng.choice(["rWWSimGroup", "WCSimGroup"]))
        terms = [str(t) for t in rng.choice(terms_all, size=int(rng.integers(1, 5)), replace=False)]
        kw = dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2, gof_terms=terms,
                  states_ts=bool(rng.integers(0, 2)), exc_interhemispheric=bool(rng.integers(0, 2)))
        if cls == "rWWSimGroup":
            kw["do_fic"] = bool(rng.integers(0, 2))
            kw["fic_penalty_scale"] = float(rng.choice([0.0, 0.5, 2.0]))
        out[f"score_random_{i:02d}"] = (cls, kw, int(rng.integers(1, 5)))
    return out


RANDOM_SCORE = random_score_cases()


def build_random(simmod, name):
    """The group of random case `name` with G = linspace(0.1, 1, N) and defaults."""
    cls, kw, N = RANDOM[name]
    kw = dict(kw, force_gpu=True, sc=_sc(2))
    if kw.get("sc_dist") == "dist":
        kw["sc_dist"] = _dist(3)
    sg = getattr(simmod, cls)(**kw)
    sg.N = N
    sg.param_lists["G"] = np.linspace(0.1, 1, N)
    sg._set_default_params()
    return sg


# groups whose settings are changed after construction: (case, [(attribute, value), ...])
MUTATED = {
    "rww_mutated": ("rww_fic", [("duration", 30), ("TR", 0.5), ("window_step", 3), ("dt", "0.05"),
                                ("noise_segment_length", None), ("bold_remove_s", 4)]),
    "wc_mutated": ("wc", [("window_size", 6), ("states_sampling", 2), ("bw_dt", "0.5"), ("duration", 12.5)]),
}

# cases whose run() is answered by fake_outputs() and then scored
SCORE_CASES = ("rww_fic", "rww_delay", "wc", "rww_multi", "rww_hemi")  # + RANDOM_SCORE, defined below
N_EMP_FCD = 12


def fake_outputs(args, n_state, n_noise=1):
    """A deterministic stand-in for run_simulations' output dict (the keys and
    shapes of ``src/ext/core.cpp:453-492``), seeded from N and nodes: FC rows
    (row 1 all NaN), FCD rows, time-averaged states with the rWW r_E state
    spread over 1-5 Hz (so the FIC penalty sees both branches), FIC flags, and
    with ``noise_out`` a noise segment with node / time shuffles."""
    N, nodes, cfg = args[14], args[15], args[7]
    rng = np.random.default_rng(1000 + 31 * N + nodes)
    bold_len = args[16] // args[17]
    out = {"init_time": 0.0, "run_time": 0.0,
           "sim_bold": rng.normal(size=(N, bold_len * nodes)),
           "_sim_states": rng.uniform(1.0, 5.0, (n_state, N, (args[16] // args[18] if args[9] else 1) * nodes)),
           "_global_bools": (rng.random((2, N)) < 0.5),
           "_global_ints": rng.integers(0, 5, (1, N)).astype(np.intc)}
    if args[10]:  # noise_out
        bw_dt = args[21]
        seg = int(int(cfg["noise_time_steps"]) / bw_dt)
        inner = int(round(bw_dt / args[20]))
        reps = -(-int(args[16] / bw_dt) // seg)
        out["_noise"] = rng.normal(size=seg * inner * nodes * n_noise)
        out["_shuffled_nodes"] = np.stack([rng.permutation(nodes) for _ in range(reps)]).astype(np.intc)
        out["_shuffled_ts"] = np.stack([rng.permutation(seg) for _ in range(reps)]).astype(np.intc)
    if cfg["do_fc"] == "1":
        fc = rng.uniform(-1, 1, (N, n_pairs(nodes, cfg["exc_interhemispheric"] == "1")))
        if N > 1:
            fc[1] = np.nan
        out["sim_fc_trils"] = fc
        if cfg["do_fcd"] == "1":
            out["sim_fcd_trils"] = rng.uniform(-1, 1, (N, 10))
    return out


def n_pairs(nodes, exc_interhemispheric):
    h = nodes // 2
    return 2 * (h * (h - 1) // 2) if exc_interhemispheric else nodes * (nodes - 1) // 2


def empirical(sg):
    rng = np.random.default_rng(77)
    return rng.uniform(-1, 1, n_pairs(sg.nodes, sg.exc_interhemispheric)), rng.uniform(-1, 1, N_EMP_FCD)


def config_record(sg):
    """get_config(include_N=True) and get_config(for_reinit=True) of a group
    (base.py:581-633) as JSON: array values by their kind only, the package
    version by its presence."""
    def enc(cfg):
        out = {}
        for k, v in cfg.items():
            if isinstance(v, np.ndarray):
                v = "<array>"
            elif k == "version":
                v = "<version>"
            elif isinstance(v, (np.generic,)):
                v = v.item()
            out[k] = v
        return out
    return json.dumps({"full": enc(sg.get_config(include_N=True)), "reinit": enc(sg.get_config(for_reinit=True))},
                      sort_keys=True)


def problem_hooks(grp, scores):
    """What the group's BNMProblem hooks (base.py:1055-1082, rww.py:254-291) do
    to a single- and a multi-objective problem and its cost."""
    res = {}
    for multi in (False, True):
        prob = types.SimpleNamespace(het_params=["w_p"], multiobj=multi, obj_names=["+fc_corr"], n_obj=1)
        grp._problem_init(prob)
        F = np.arange(grp.N, dtype=float)
        out = {"F": F[:, None].copy() if multi else F.copy()}
        grp._problem_evaluate(prob, None, out, scores=[scores])
        res[f"obj_names_{int(multi)}"] = np.array(json.dumps(prob.obj_names))
        res[f"n_obj_{int(multi)}"] = np.asarray(prob.n_obj)
        res[f"F_{int(multi)}"] = np.asarray(out["F"], dtype=float)
    return res


def helpers(grp):
    """Outputs of the group's result helpers (base.py:820-1053)."""
    res = {}
    avg = grp.get_state_averages()
    res["state_avg_cols"] = np.array(json.dumps(list(avg.columns)))
    res["state_avg"] = avg.to_numpy(dtype=float)
    if grp.do_fc:
        for i in (0, grp.N - 1):
            res[f"sim_fc_{i}"] = grp.get_sim_fc(i)
        if grp.do_fcd:
            res["sim_fcd_0"] = grp.get_sim_fcd(0)
    sl = grp.slice(grp.N - 1)
    res["slice_N"] = np.asarray(sl.N)
    res["slice_bold"] = np.asarray(sl.sim_bold)
    for k, v in sl.param_lists.items():
        res[f"slice_param_{k}"] = np.asarray(v, dtype=float)
    for k, v in sl.sim_states.items():
        res[f"slice_state_{k}"] = np.asarray(v, dtype=float)
    if sl.do_fc:
        res["slice_fc"] = np.asarray(sl.sim_fc_trils)
    cleared = list(grp._to_clear)
    grp.clear()
    res["cleared"] = np.array(json.dumps(cleared))
    res["left"] = np.array(json.dumps([a for a in cleared if hasattr(grp, a)]))
    return res


# empirical-helper cases: (BOLD seed, zeroed volumes, FC kwargs, FCD args and kwargs)
UTIL_CASES = {
    "plain": (21, [], {}, (10, 2), {}),
    "outliers_hemi": (22, [5, 6, 40], {"exc_interhemispheric": True}, (8, 2),
                      {"exc_interhemispheric": True, "return_dfc": True}),
    "no_drop_edges": (23, [], {}, (6, 3), {"drop_edges": False}),
    "outlier_windows": (24, list(range(10, 19)), {}, (6, 2), {"outlier_threshold": 0.5}),
}


def util_bold(seed, zeroed, nodes=NODES, vols=60):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(nodes, vols)).cumsum(axis=1)
    x[:, zeroed] = 0.0
    return x


def _reference_sim(ref_root):
    """Imports src/cubnm/sim from the reference with a recording core."""
    class Stop(Exception):
        pass

    rec = {}

    def run_simulations(*args):
        rec["args"] = args
        if rec.get("answer"):
            return fake_outputs(args, rec["n_state"], rec["n_noise"])
        raise Stop()

    def stub(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    pkg = stub("cubnm")
    pkg.__path__ = [os.path.join(ref_root, "src", "cubnm")]
    pkg._core = stub("cubnm._core", run_simulations=run_simulations, set_const=lambda *a: None, init=lambda: None)
    pkg._setup_opts = stub("cubnm._setup_opts", many_nodes_flag=False, gpu_enabled_flag=True, max_nodes_reg=200,
                           max_nodes_many=500, noise_segment_flag=True, gpu_model_flag="nvidia")
    pkg._version = stub("cubnm._version", get_versions=lambda: {"version": "0+recorded"})
    import cubnm.sim as refsim
    return refsim, rec, Stop


def main(ref_root):
    refsim, rec, Stop = _reference_sim(ref_root)
    out = {}
    for name in list(CASES) + list(MULTI) + list(MUTATED) + list(RANDOM):
        sg = build(refsim, name)
        rec.clear()
        try:
            sg.run()
        except Stop:
            pass
        args = rec["args"]
        assert len(args) == 22, len(args)
        for i in ARRAY_ARGS:
            out[f"{name}|{i}"] = np.asarray(args[i])
        meta = {str(i): args[i] for i in range(22) if i not in ARRAY_ARGS and i != 7}
        meta["model_config"] = args[7]
        out[f"{name}|meta"] = np.array(json.dumps(meta, sort_keys=True))
        out[f"{name}|config"] = np.array(config_record(sg))
    if not hasattr(np, "NaN"):  # the reference's rww.py:220 predates numpy 2
        np.NaN = np.nan
    for name in list(SCORE_CASES) + list(RANDOM_SCORE):
        sg = build(refsim, name)
        rec.clear()
        rec["answer"] = True
        rec["n_state"], rec["n_noise"] = len(sg.state_names), sg.n_noise
        sg.run()
        if sg.noise_out:
            noise = np.ascontiguousarray(sg.get_noise())
            out[f"{name}|noise_shape"] = np.asarray(noise.shape)
            out[f"{name}|noise_sha256"] = np.array(hashlib.sha256(noise.tobytes()).hexdigest())
        emp_fc, emp_fcd = empirical(sg)
        for g, grp in enumerate(getattr(sg, "children", [sg])):
            key = f"{name}|{g}"
            scores = grp.score(emp_fc, emp_fcd)
            for k, v in problem_hooks(grp, scores).items():
                out[f"{key}|hook|{k}"] = v
            out[f"{key}|score_columns"] = np.array(json.dumps(sorted(scores.columns)))
            for c in scores.columns:
                out[f"{key}|score|{c}"] = scores[c].to_numpy(dtype=float)
            out[f"{key}|bold_shape"] = np.asarray(grp.sim_bold.shape)
            if getattr(grp, "do_fic", False):
                out[f"{key}|wIE"] = np.asarray(grp.param_lists["wIE"], dtype=float)
                out[f"{key}|fic_ntrials"] = np.asarray(grp.fic_ntrials)
                out[f"{key}|fic_failed"] = np.asarray(grp.fic_failed)
            if name in SCORE_CASES:
                for k, v in helpers(grp).items():
                    out[f"{key}|helper|{k}"] = v
    import cubnm.utils as refutils
    for name, (seed, zeroed, fc_kw, fcd_args, fcd_kw) in UTIL_CASES.items():
        bold = util_bold(seed, zeroed)
        out[f"util|{name}|fc"] = refutils.calculate_fc(bold.copy(), **fc_kw)
        fcd = refutils.calculate_fcd(bold.copy(), *fcd_args, **fcd_kw)
        if fcd_kw.get("return_dfc"):
            out[f"util|{name}|fcd"], out[f"util|{name}|dfc"] = fcd
        else:
            out[f"util|{name}|fcd"] = fcd
    for src in ("friston2003", "heinzle2016-3T"):
        p = refutils.get_bw_params(src)
        out[f"util|bw|{src}"] = np.array([p["k1"], p["k2"], p["k3"]])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(CASES) + len(MULTI) + len(MUTATED) + len(RANDOM)} cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUBNM_REFERENCE", "../cubnm"))
