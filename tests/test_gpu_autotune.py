"""The FP32 integrator autotuner (model_config "autotune" = "1"): the first run of
a workload probes the applicable integrators and keeps the fastest, recorded in
CBNM_TUNE_FILE; the outputs stay within the mixed-precision bounds whichever
integrator wins, and a second run reuses the choice without probing."""
import os

import numpy as np
import pytest

import cases
from cubnm_b200 import core

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("delay", [False, True])
def test_autotune_picks_an_applicable_integrator(delay, tmp_path, monkeypatch):
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("CBNM_TUNE_FILE", str(path))
    core.tune_reset()
    N, nodes = 96, 68
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=8, seed=21, density=0.2, window_size=4,
                                     window_step=2, bold_remove_s=2))
    if delay:
        args[3] = np.ascontiguousarray(cases.synthetic_lengths(nodes, 21).ravel())
        args[6] = np.full(N, 6.0)
        args[11] = True
    a64 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a64[7] = dict(args[7], precision="fp64")
    o64 = core.run_simulations(*a64)
    a32 = [x.copy() if isinstance(x, np.ndarray) else x for x in args]
    a32[7] = dict(args[7], precision="fp32", autotune="1")
    o32 = core.run_simulations(*a32)
    first = core.last_integrator()
    allowed = {"lanes", "lanes512", "simt"} if delay else {"tc2", "tc2ws", "tc1", "lanes", "lanes512", "simt"}
    assert first in allowed
    lines = path.read_text().split("\n")
    assert len([l for l in lines if l.strip()]) == 1 and lines[0].split()[1] == first
    assert np.nanmax(np.abs(o64["sim_fc_trils"] - o32["sim_fc_trils"])) <= 2e-3
    core.run_simulations(*a32)  # cached: no further probe, same integrator
    assert core.last_integrator() == first
    assert len([l for l in path.read_text().split("\n") if l.strip()]) == 1
    core.tune_reset()
    monkeypatch.delenv("CBNM_TUNE_FILE")
