"""bench.py's reference arm (the reference's CPU algorithm, timed on the host)
runs without a GPU: one JSON line with the contract's keys on rank 0, nothing
on the other ranks.  A short duration keeps it to seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--duration", "20",
       "--ref-budget", "2"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["config"]["sample_sims_per_step"] >= 2 * line["cpu_baseline"]["cores"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_config_roofline_counts_gathers_and_flops():
    """The c2-c4 roofline: ring-buffer bytes (4 per nonzero per node-step) for delayed
    networks, FP32 flops (2 per nonzero + the rWW update) without delays, per launch."""
    import numpy as np
    import bench
    from cubnm_b200 import synthetic
    args = list(synthetic.synthetic_args("rWW", N=4, nodes=20, duration_s=2, seed=1, density=0.25))
    n = 20
    sc = np.asarray(args[1]).reshape(n, n)
    nnz = np.count_nonzero(sc) / n
    node_steps = 4 * n * 2000 / 0.1
    r = bench.config_roofline(args, 1000.0, True)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["algorithmic_bytes"] - node_steps * nnz * 4) < 1e-6 * r["algorithmic_bytes"]
    assert abs(r["achieved"] - node_steps * nnz * 4 / 1e9) < 1e-9 * r["achieved"]
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    f = bench.config_roofline(args, 500.0, False, fp32_peak=70.0)
    flops = node_steps * (2 * nnz + bench.RWW_FP32_FLOPS)
    assert f["bound"] == "fp32" and abs(f["achieved"] - flops / 0.5 / 1e12) < 1e-9 * f["achieved"]
