"""SimGroup marshalling against the reference's own SimGroup (CPU).

``tests/golden/simgroup_args.npz`` holds the 22 arguments that the reference's
``SimGroup.run()`` (``src/cubnm/sim/base.py:673-752``) and
``MultiSimGroupMixin.run()`` (``base.py:1323-1385``) pass to
``run_simulations`` for the groups of ``tests/golden/make_simgroup_args.py``.
Here the same groups are built with ``cubnm_b200.sim`` and run with
``core.run_simulations`` replaced by a recorder: every argument must be equal,
and ``model_config`` may differ only by the ``precision`` key this library adds.
The checks of ``do_fc`` / ``do_fcd`` / ``gof_terms`` follow ``base.py:486-513``.

The fixture also holds the reference's ``score()`` of groups whose run was
answered by ``fake_outputs()``; the same outputs go through this library's
``_process_out`` / ``score`` with the GPU goodness-of-fit call replaced by the
reference's CPU formulas (``base.py:1164-1188``), so what is compared is the
output handling, signs, NaN fill, ``+gof``, the rWW FIC penalty, the noise
reconstruction of ``get_noise``, the BNMProblem hooks (``_problem_init`` /
``_problem_evaluate``) and the result helpers (``get_state_averages``,
``get_sim_fc`` / ``get_sim_fcd``, ``slice``, ``clear``).
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest
import scipy.stats

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_simgroup_args as G  # noqa: E402
from cubnm_b200 import sim  # noqa: E402

FIXTURE = np.load(os.path.join(os.path.dirname(__file__), "golden", "simgroup_args.npz"))


class _Stop(Exception):
    pass


def _recorded_args(sg, monkeypatch):
    rec = {}

    def run_simulations(*args):
        rec["args"] = args
        raise _Stop()

    monkeypatch.setattr(sim.core, "run_simulations", run_simulations)
    with pytest.raises(_Stop):
        sg.run()
    return rec["args"]


@pytest.mark.parametrize("case", list(G.CASES) + list(G.MULTI) + list(G.MUTATED) + list(G.RANDOM))
def test_run_arguments_equal_the_reference(case, monkeypatch):
    sg = G.build(sim, case)
    args = _recorded_args(sg, monkeypatch)
    assert len(args) == 22
    for i in G.ARRAY_ARGS:
        ref = FIXTURE[f"{case}|{i}"]
        got = np.asarray(args[i])
        assert got.shape == ref.shape, (i, got.shape, ref.shape)
        np.testing.assert_array_equal(got, ref, err_msg=f"argument {i}")
    meta = json.loads(str(FIXTURE[f"{case}|meta"]))
    ref_cfg = meta.pop("model_config")
    for k, v in meta.items():
        assert args[int(k)] == v, (k, args[int(k)], v)
    cfg = dict(args[7])
    assert cfg.pop("precision") == "fp64"
    assert cfg == ref_cfg
    # get_config (base.py:581-633), without the precision key this library adds
    got = json.loads(G.config_record(sg))
    for part in got.values():
        assert part.pop("precision") == "fp64"
    assert got == json.loads(str(FIXTURE[f"{case}|config"]))


def test_fc_fcd_and_gof_term_checks():
    sc = G._sc(1)
    with pytest.raises(ValueError, match="FCD without FC"):
        sim.rWWSimGroup(duration=10, TR=1, sc=sc, do_fc=False, gof_terms=[])
    with pytest.raises(ValueError, match="FC goodness-of-fit terms without FC"):
        sim.rWWSimGroup(duration=10, TR=1, sc=sc, do_fc=False, do_fcd=False)
    with pytest.raises(ValueError, match="FCD goodness-of-fit terms without FCD"):
        sim.rWWSimGroup(duration=10, TR=1, sc=sc, do_fcd=False)
    sg = sim.rWWSimGroup(duration=10, TR=1, sc=sc, do_fc=False, do_fcd=False, gof_terms=[])
    assert not sg.do_fc and not sg.do_fcd


def _cpu_gof(sim_fc_trils=None, emp_fc_tril=None, sim_fcd_trils=None, emp_fcd_tril=None, terms=None):
    """The reference's CPU goodness-of-fit formulas (base.py:1164-1188), as
    positive distances / correlations like ``utils.gof``."""
    out = {}
    if sim_fc_trils is not None:
        if "fc_corr" in terms:
            out["fc_corr"] = np.array([scipy.stats.pearsonr(r, emp_fc_tril).statistic for r in sim_fc_trils])
        if "fc_diff" in terms:
            out["fc_diff"] = np.abs(sim_fc_trils.mean(axis=1) - emp_fc_tril.mean())
        if "fc_normec" in terms:
            out["fc_normec"] = np.linalg.norm(sim_fc_trils - emp_fc_tril[None], axis=1) / (2 * np.sqrt(emp_fc_tril.size))
    if sim_fcd_trils is not None and "fcd_ks" in terms:
        out["fcd_ks"] = np.array([scipy.stats.ks_2samp(r, emp_fcd_tril).statistic for r in sim_fcd_trils])
    return out


@pytest.mark.parametrize("case", list(G.SCORE_CASES) + list(G.RANDOM_SCORE))
def test_processed_outputs_and_scores_equal_the_reference(case, monkeypatch):
    sg = G.build(sim, case)
    monkeypatch.setattr(sim.core, "run_simulations", lambda *a: G.fake_outputs(a, len(sg.state_names), sg.n_noise))
    monkeypatch.setattr(sim.utils, "gof", _cpu_gof)
    sg.run()
    if sg.noise_out:  # get_noise, base.py:843-895
        noise = np.ascontiguousarray(sg.get_noise())
        assert noise.shape == tuple(FIXTURE[f"{case}|noise_shape"])
        assert hashlib.sha256(noise.tobytes()).hexdigest() == str(FIXTURE[f"{case}|noise_sha256"])
    emp_fc, emp_fcd = G.empirical(sg)
    for g, grp in enumerate(getattr(sg, "children", [sg])):
        key = f"{case}|{g}"
        with np.errstate(invalid="ignore"):
            scores = grp.score(emp_fc, emp_fcd)
        assert sorted(scores.columns) == json.loads(str(FIXTURE[f"{key}|score_columns"]))
        for c in scores.columns:
            np.testing.assert_allclose(scores[c].to_numpy(dtype=float), FIXTURE[f"{key}|score|{c}"],
                                       rtol=1e-12, atol=1e-15, err_msg=c)
        assert tuple(grp.sim_bold.shape) == tuple(FIXTURE[f"{key}|bold_shape"])
        if getattr(grp, "do_fic", False):
            np.testing.assert_array_equal(grp.param_lists["wIE"], FIXTURE[f"{key}|wIE"])
            np.testing.assert_array_equal(grp.fic_ntrials, FIXTURE[f"{key}|fic_ntrials"])
            np.testing.assert_array_equal(grp.fic_failed, FIXTURE[f"{key}|fic_failed"])
        # BNMProblem hooks, then the result helpers (slice, clear, ...)
        parts = [("hook", G.problem_hooks(grp, scores))]
        if case in G.SCORE_CASES:
            parts.append(("helper", G.helpers(grp)))
        for part, got in parts:
            want = sorted(k.split("|", 3)[3] for k in FIXTURE.files if k.startswith(f"{key}|{part}|"))
            assert sorted(got) == want, part
            for k, v in got.items():
                ref = FIXTURE[f"{key}|{part}|{k}"]
                if ref.dtype.kind == "U":
                    assert str(v) == str(ref), k
                else:
                    np.testing.assert_allclose(np.asarray(v, dtype=float), ref, rtol=1e-12, atol=1e-15, err_msg=k)


def test_rww_problem_init_rejects_free_wie_under_fic():
    import types
    sg = G.build(sim, "rww_fic")
    with pytest.raises(ValueError, match="wIE should not be specified"):
        sg._problem_init(types.SimpleNamespace(het_params=["wIE"], multiobj=False, obj_names=[], n_obj=1))


@pytest.mark.parametrize("case", list(G.UTIL_CASES))
def test_empirical_fc_fcd_equal_the_reference(case):
    from cubnm_b200 import utils
    seed, zeroed, fc_kw, fcd_args, fcd_kw = G.UTIL_CASES[case]
    bold = G.util_bold(seed, zeroed)
    np.testing.assert_allclose(utils.calculate_fc(bold, **fc_kw), FIXTURE[f"util|{case}|fc"], rtol=1e-12, atol=1e-14)
    fcd = utils.calculate_fcd(bold, *fcd_args, **fcd_kw)
    if fcd_kw.get("return_dfc"):
        fcd, dfc = fcd
        np.testing.assert_allclose(dfc, FIXTURE[f"util|{case}|dfc"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(fcd, FIXTURE[f"util|{case}|fcd"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("src", ["friston2003", "heinzle2016-3T"])
def test_bw_params_equal_the_reference(src):
    from cubnm_b200 import utils
    p = utils.get_bw_params(src)
    np.testing.assert_array_equal([p["k1"], p["k2"], p["k3"]], FIXTURE[f"util|bw|{src}"])


def test_matrices_from_files(tmp_path, monkeypatch):
    """sc / sc_dist given as .txt and .npy paths (base.py:209-215, 252-264) and
    out_dir='same' (base.py:269-276) give the arguments of the array form."""
    sc, dist = G._sc(1), G._dist(5)
    np.savetxt(tmp_path / "sc.txt", sc)
    np.save(tmp_path / "dist.npy", dist)
    kw = dict(duration=10, TR=1, window_size=4, window_step=2, bold_remove_s=2, do_fic=False, force_gpu=True)
    groups = [sim.rWWSimGroup(sc=sc, sc_dist=dist, **kw),
              sim.rWWSimGroup(sc=str(tmp_path / "sc.txt"), sc_dist=str(tmp_path / "dist.npy"), out_dir="same", **kw)]
    assert groups[1].out_dir == str(tmp_path / "sc")
    got = []
    for sg in groups:
        sg.N = 2
        sg.param_lists["G"] = np.array([0.2, 0.4])
        sg._set_default_params()
        got.append(_recorded_args(sg, monkeypatch))
    for i in G.ARRAY_ARGS:
        np.testing.assert_allclose(np.asarray(got[1][i]), np.asarray(got[0][i]), rtol=1e-15, atol=0)
    with pytest.raises(ValueError, match="Unsupported"):
        sim.rWWSimGroup(sc=str(tmp_path / "sc.csv"), **kw)


def test_duration_must_be_whole_milliseconds():
    """Decimal(duration) as base.py:339-350: a float like 0.1 is not a whole
    number of milliseconds there, nor here."""
    with pytest.raises(ValueError, match="whole number"):
        sim.WCSimGroup(duration=0.1, TR=0.05, sc=G._sc(1), bw_dt="0.1", window_size=0.2, window_step=0.1)
    sg = sim.WCSimGroup(duration=0.5, TR=0.1, sc=G._sc(1), bw_dt="0.1", window_size=0.2, window_step=0.1)
    assert sg.duration_msec == 500
