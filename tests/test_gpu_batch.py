"""cbnm_run_batch (core.run_batch): independent groups run concurrently, each on
its own stream (or, for groups on the lane kernel, in one persistent launch per
round); every group's outputs must equal a separate run_simulations call of the
same arguments, bit for bit."""
import numpy as np
import pytest

import cases
from cubnm_b200 import core

pytestmark = pytest.mark.gpu


def _delay(args, nodes, seed=0):
    a = list(args)
    rng = np.random.default_rng(seed)
    pts = rng.normal(size=(nodes, 3))
    pts = pts / np.linalg.norm(pts, axis=1, keepdims=True) * rng.uniform(0, 70, (nodes, 1))
    a[3] = np.ascontiguousarray((np.linalg.norm(pts[:, None] - pts[None], axis=2) * 1.3).ravel())
    a[6] = np.full(a[14], 6.0)
    a[11] = True
    return a


def _groups():
    return [
        _delay(cases.synthetic_args("rWW", N=24, nodes=68, duration_s=12, seed=1, density=0.2, bold_remove_s=2,
                                    window_size=4, window_step=2), 68),
        list(cases.synthetic_args("WC", N=40, nodes=100, duration_s=8, seed=2, bold_remove_s=2, window_size=2,
                                  window_step=1, precision="fp32")),
        list(cases.synthetic_args("rWW", N=64, nodes=100, duration_s=10, seed=3, bold_remove_s=2, window_size=2,
                                  window_step=1, precision="fp32", do_fic=1)),
        list(cases.synthetic_args("Kuramoto", N=8, nodes=32, duration_s=6, seed=4, bold_remove_s=1, window_size=2,
                                  window_step=1)),
        list(cases.synthetic_args("rWWEx", N=16, nodes=200, duration_s=6, seed=5, density=0.1, bold_remove_s=1,
                                  window_size=2, window_step=1, precision="fp32")),
    ]


def _copy(a):
    return [x.copy() if isinstance(x, np.ndarray) else x for x in a]


@pytest.mark.parametrize("kernel", ["default", "lanes"])
def test_batch_equals_separate_calls(kernel, monkeypatch):
    """With the lane kernel forced, the delayed and large groups of a round run as
    one persistent work-queue launch (k_integrate_lanes_multi) and must still equal
    their separate calls, which run k_integrate_lanes, bit for bit."""
    if kernel == "lanes":
        monkeypatch.setenv("CBNM_FP32_KERNEL", "lanes")
    groups = _groups()
    sep_args = [_copy(g) for g in groups]
    sep = [core.run_simulations(*a) for a in sep_args]
    bat_args = [_copy(g) for g in groups]
    bat = core.run_batch(bat_args)
    for i, (a, b) in enumerate(zip(sep, bat)):
        for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils", "_sim_states", "_global_bools", "_global_ints"):
            np.testing.assert_array_equal(b[k], a[k], err_msg=f"group {i} {k}")
    # the FIC write-back lands in each group's own regional parameters
    np.testing.assert_array_equal(bat_args[2][5], sep_args[2][5])
    assert not np.array_equal(bat_args[2][5], groups[2][5])


def test_batch_twice_and_more_groups_than_workers():
    groups = [list(cases.synthetic_args("rWW", N=8, nodes=20 + 4 * i, duration_s=4, seed=i, bold_remove_s=1,
                                        window_size=2, window_step=1)) for i in range(20)]
    first = core.run_batch([_copy(g) for g in groups])
    second = core.run_batch([_copy(g) for g in groups])
    for a, b in zip(first, second):
        np.testing.assert_array_equal(a["sim_bold"], b["sim_bold"])
    ref = core.run_simulations(*_copy(groups[17]))
    np.testing.assert_array_equal(first[17]["sim_bold"], ref["sim_bold"])


def test_batch_reports_the_failing_group():
    """A group that sizes fine but is refused when it runs (use_cpu) fails the batch
    with its index in the message; the other groups still ran."""
    groups = _groups()[:3]
    bad = _copy(groups[1])
    bad[13] = True  # use_cpu
    with pytest.raises(RuntimeError, match="group 1: use_cpu"):
        core.run_batch([_copy(groups[0]), bad, _copy(groups[2])])


def test_batch_groups_with_different_fc_shared_memory():
    """Groups whose FC kernels stage windows of different sizes in shared memory
    (40 and 300 nodes) launch from several host threads at once: a shared-memory
    limit set per launch would let one group's setting fail another's launch."""
    groups = []
    for i in range(12):
        nodes = 300 if i % 2 else 40
        a = list(cases.synthetic_args("rWW", N=8, nodes=nodes, duration_s=40, seed=20 + i, density=0.2,
                                      bold_remove_s=2, window_size=10, window_step=2, precision="fp32"))
        groups.append(a)
    bat = core.run_batch([_copy(g) for g in groups])
    for i in (0, 1):
        ref = core.run_simulations(*_copy(groups[i]))
        np.testing.assert_array_equal(bat[i]["sim_fc_trils"], ref["sim_fc_trils"])
        np.testing.assert_array_equal(bat[i]["sim_fcd_trils"], ref["sim_fcd_trils"])
