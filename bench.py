"""Benchmark: rWW simulations x simulated seconds per wall second.

Workload (the reference's headline case): reduced Wong-Wang, 100 nodes,
32,768 simulations, 60 s each, dt 0.1 ms, BOLD TR 1 s, FC + FCD (window 10,
step 2), no FIC, no delay; G, w_p, J_N drawn uniformly from the grid ranges
G in [0.001, 10], w_p in [0, 2], J_N in [0.001, 0.5]; synthetic SC (symmetric,
30% density, lognormal weights, mean row sum 1); noise from the seeded
generator.  One "step" = one run of all simulations (integration + BOLD +
FC/FCD).  The BOLD output alone (1.57 GB) is larger than L2, so no L2 flush is
needed between steps.

value : FP32 / tensor-core path, inputs resident in HBM (device C-ABI entry).
e2e   : the same through the host C-ABI entry (cbnm_run_simulations with host
        buffers: parameters and SC copied in, BOLD/FC/FCD/states copied out)
        plus the GOF scoring call, timed on the host.
fp64  : the FP64 reference-precision path, measured on a 4,736-simulation
        subset (a full GPU wave), for the precision/speed comparison; beside it
        the FP32 path on the same subset, without and (end to end) with the
        reference's default analytical FIC.

--impl reference times the reference's own CPU algorithm (the oracle
restatement, OpenMP over simulations, all host threads) on a bounded sample.
Under torchrun every rank integrates its own 32,768 simulations (weak scaling;
simulations are independent, no collective on the data path).
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

N_SIMS = 32768
NODES = 100
DURATION_S = 60
# dram__bytes_read.sum + dram__bytes_write.sum of one integrator launch of the default
# workload, from an ncu capture of one launch on a reduced case scaled by the
# simulated node-steps (profiles/ names the capture); None until measured
TRAFFIC_DEFAULT_WORKLOAD = 6.242e9
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_integrate_tc launch on 9,472 sims x "
                  "8 s (240.6 MB), scaled by node-steps to 32,768 x 60 s "
                  "(profiles/k_integrate_tc_rww_9472x8s_counters.md)")
# FP32 flops of one rWW node update (rww.cpp:194-232): I_E 8, I_I 4, the two affine
# rate arguments 4, the two rates (without their exp) 6, dS_E 8, dS_I 6, the two
# state additions 2
RWW_FP32_FLOPS = 38
WORKLOAD = f"rWW {NODES} nodes, {N_SIMS} sims, {DURATION_S} s, dt 0.1 ms, TR 1 s, FC+FCD w10/s2"
# the kernel behind each integrator name of core.last_integrator()
KERNEL_OF = {"tc1": "k_integrate_tc<RWW32, Tile<32, 8, 3>>", "tc2": "k_integrate_pp<RWW32>",
             "tc2ws": "k_integrate_pp_ws<RWW32>", "simt": "k_integrate_sim<M, delay, float>",
             "lanes": "k_integrate_lanes<M, 1024, ...>", "lanes512": "k_integrate_lanes<M, 512, ...>",
             "fp64": "k_integrate_sim<M, delay, double>"}
METRIC = "rWW sims x sim-s per wall-s (100 nodes, 32k sims)"
UNIT = "sims*sim-s/s"


def workload_args(n_sims, duration_s, precision, seed):
    from cubnm_b200 import synthetic
    rng = np.random.default_rng(1000 + seed)
    G = rng.uniform(0.001, 10, n_sims)
    wp = rng.uniform(0, 2, n_sims)
    jn = rng.uniform(0.001, 0.5, n_sims)
    # the headline case removes 30 s of BOLD before FC; short profiling runs keep 3/4 of it
    remove = 30 if duration_s >= 60 else duration_s // 4
    window = 10 if duration_s - remove > 12 else 2
    return list(synthetic.synthetic_args("rWW", N=n_sims, nodes=NODES, duration_s=duration_s, seed=0, G=G, w_p=wp,
                                     J_N=jn, precision=precision, window_size=window, window_step=2,
                                     bold_remove_s=remove))


class Clocks:
    """Samples nvidia-smi clocks / throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(name)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def device_buffers(torch, args, sizes, dev):
    """Inputs copied to HBM once; outputs allocated on the device."""
    from cubnm_b200 import _abi
    t = {}
    t["sc"] = torch.from_numpy(np.ascontiguousarray(args[1])).to(dev)
    t["sc_idx"] = torch.from_numpy(np.ascontiguousarray(args[2], dtype=np.int32)).to(dev)
    t["dist"] = torch.from_numpy(np.ascontiguousarray(args[3])).to(dev)
    t["g"] = torch.from_numpy(np.ascontiguousarray(args[4])).to(dev)
    t["r"] = torch.from_numpy(np.ascontiguousarray(args[5])).to(dev)
    t["v"] = torch.from_numpy(np.ascontiguousarray(args[6])).to(dev)
    N, n = args[14], args[15]
    t["bold"] = torch.empty((N, sizes.bold_len * n), dtype=torch.float64, device=dev)
    t["fc"] = torch.empty((N, sizes.n_pairs), dtype=torch.float64, device=dev)
    t["fcd"] = torch.empty((N, max(1, sizes.n_window_pairs)), dtype=torch.float64, device=dev)
    t["states"] = torch.empty((sizes.n_state_vars, N, n), dtype=torch.float64, device=dev)
    t["gb"] = torch.empty((max(1, sizes.n_global_out_bool), N), dtype=torch.uint8, device=dev)
    t["gi"] = torch.empty((max(1, sizes.n_global_out_int), N), dtype=torch.int32, device=dev)
    dp = lambda x: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_double))  # noqa: E731
    p = _abi.Prepared(*args)
    a = p.args
    a.sc = dp(t["sc"])
    a.sc_indices = C.cast(C.c_void_p(t["sc_idx"].data_ptr()), C.POINTER(C.c_int32))
    a.sc_dist = dp(t["dist"])
    a.global_params = dp(t["g"])
    a.regional_params = dp(t["r"])
    a.v_list = dp(t["v"])
    o = _abi.Outputs(dp(t["bold"]), dp(t["fc"]), dp(t["fcd"]), dp(t["states"]),
                     C.cast(C.c_void_p(t["gb"].data_ptr()), C.POINTER(C.c_uint8)),
                     C.cast(C.c_void_p(t["gi"].data_ptr()), C.POINTER(C.c_int32)), None, None, None, 0.0, 0.0)
    return t, p, o


def run_ours(opts, rank, world, local_rank):
    import torch
    from cubnm_b200 import _abi, core, utils
    from cubnm_b200._lib import lib, check
    from cubnm_b200 import synthetic

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = lib()
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        from cubnm_b200.shard import max_over_ranks as shard_max
        return shard_max(x, device=dev) if dist is not None else x

    n_sims = opts.sims
    args = workload_args(n_sims, opts.duration, opts.precision, seed=rank)
    sizes = _abi.Sizes()
    check(L.cbnm_query_sizes(C.byref(_abi.Prepared(*args).args), C.byref(sizes)))
    bufs, prep, outs = device_buffers(torch, args, sizes, dev)
    st = torch.cuda.current_stream()

    def device_step():
        check(L.cbnm_run_simulations_device(C.byref(prep.args), C.byref(outs)))
        return core.last_timing()

    # warm-up (first call also generates the noise segment: session init)
    for _ in range(opts.warmup):
        device_step()
    clocks = Clocks(int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]) if world == 1 else local_rank)
    clocks.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    integ_ms, fc_ms, launches = [], [], 0
    for _ in range(opts.steps):
        tm = device_step()
        integ_ms.append(tm["integrate_ms"])
        fc_ms.append(tm["fc_ms"])
        launches += tm["kernel_launches"]
    e1.record(st)
    barrier()
    ck = clocks.stop()
    integrator = core.last_integrator()
    ms = max_over_ranks(e0.elapsed_time(e1) / opts.steps)
    value = world * n_sims * opts.duration / (ms / 1e3)

    # end to end through the host C ABI (host buffers; copies inside the timed region) + GOF scoring
    emp = synthetic.synthetic_emp_bold(NODES, opts.duration, 7)
    emp_fc = utils.calculate_fc(emp)
    emp_fcd = utils.calculate_fcd(emp, 10 if opts.duration >= 16 else 2, 2)
    host_args = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    core.run_simulations(*host_args)  # warm the host path
    e2e_steps = max(1, opts.steps // 2)
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(e2e_steps):
        out = core.run_simulations(*host_args)
        tm = core.last_timing()
        h2d += tm["h2d_bytes"]
        d2h += tm["d2h_bytes"]
        g = utils.gof(out["sim_fc_trils"], emp_fc, out["sim_fcd_trils"], emp_fcd)
        launches_e2e = tm["kernel_launches"]
        assert np.isfinite(g["fc_corr"]).mean() > 0.5
    barrier()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
    e2e_value = world * n_sims * opts.duration / e2e_s

    # FP64 reference-precision path on one full wave, same metric
    fp64 = None
    line_errors = None
    if not opts.skip_fp64:
        n64 = min(n_sims, 4736)
        a64 = workload_args(n64, opts.duration, "fp64", seed=rank)
        o64 = core.run_simulations(*a64)
        t64 = core.last_timing()
        fp32_sub = workload_args(n64, opts.duration, opts.precision, seed=rank)
        o32 = core.run_simulations(*fp32_sub)
        t32 = core.last_timing()
        err = precision_error(o64, o32, emp_fc, emp_fcd)
        err["sims"] = n64
        line_errors = err
        # the same subset with the reference's default rWW setting, analytical FIC on
        # (wIE solved per node on the GPU before the integrator), end to end
        fic_sub = workload_args(n64, opts.duration, opts.precision, seed=rank)
        fic_sub[7] = dict(fic_sub[7], do_fic="1")
        fic_sub[5][2] = 0.0
        core.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in fic_sub])
        t0 = time.perf_counter()
        core.run_simulations(*fic_sub)
        t_fic = time.perf_counter() - t0
        fp64 = {"value": n64 * opts.duration / ((t64["integrate_ms"] + t64["fc_ms"]) / 1e3),
                "fp32_same_subset": n64 * opts.duration / ((t32["integrate_ms"] + t32["fc_ms"]) / 1e3),
                "fp32_same_subset_fic_e2e": n64 * opts.duration / t_fic,
                "sims": n64, "unit": UNIT}

    # roofline of the dominant kernel (the integrator).  Its binding resource is the
    # FP32 / MUFU node update (ncu: profiles/), so the bound reported is FP32 FLOP/s of
    # the update against this GPU's measured FMA throughput; the coupling GEMM's
    # tensor-pipe fraction is reported beside it.
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak_tf = peaks.get("bf16_tflops_sustained") or 1400.0
    f1, f2 = C.c_double(), C.c_double()
    check(L.cbnm_measure_fp32_peak(C.byref(f1), C.byref(f2)))
    fp32_peak = max(f1.value, f2.value)
    node_steps = n_sims * NODES * (opts.duration * 1000 / 0.1)
    integ = float(np.mean(integ_ms)) / 1e3
    useful = 2.0 * NODES * node_steps  # coupling flops (2 n per node-step)
    issued = 3 * 2.0 * 128 * (((NODES + 15) // 16) * 16) * (n_sims * 1.0) * (opts.duration * 1e4)  # BF16x3 MMA work
    fp32_flops = RWW_FP32_FLOPS * node_steps
    traffic, traffic_src = opts.traffic, "--traffic" if opts.traffic is not None else None
    if (traffic is None and n_sims == N_SIMS and opts.duration == DURATION_S and opts.precision == "fp32"
            and integrator == "tc1"):  # the capture is of the single-tile kernel
        traffic, traffic_src = TRAFFIC_DEFAULT_WORKLOAD, TRAFFIC_SOURCE
    roof = {"bound": "fp32", "achieved": fp32_flops / integ / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": fp32_flops / integ / 1e12 / fp32_peak,
            "peak_source": f"measured on this GPU by cbnm_measure_fp32_peak (FFMA {f1.value:.1f}, "
                           f"FFMA2 {f2.value:.1f} TFLOP/s)",
            "work": f"{RWW_FP32_FLOPS} FP32 flops per node-step (rWW update), {node_steps:.3e} node-steps",
            "tensor": {"achieved": useful / integ / 1e12, "peak": peak_tf, "unit": "TFLOP/s",
                       "frac": useful / integ / 1e12 / peak_tf,
                       "peak_source": ("MEASURED_PEAKS.json bf16_tflops_sustained (of measured)" if peaks
                                       else "fallback"),
                       "mma_issued_tflops": issued / integ / 1e12},
            "traffic": traffic, "traffic_source": traffic_src,
            "algorithmic_bytes": N_SIMS * NODES * DURATION_S * 8.0 if n_sims == N_SIMS else None,
            "kernel": KERNEL_OF.get(integrator, integrator), "kernel_ms": integ * 1e3,
            "note": "per-pipe utilisation of this kernel: profiles/ (ncu)"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": opts.steps,
        "warmup": opts.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (BF16x3 tensor-core coupling, FP64 Balloon-Windkessel and FC/FCD)",
        "data": "synthetic (seeded SC, parameters and noise)",
        "config": {"workload": WORKLOAD, "sims_per_gpu": n_sims, "nodes": NODES, "duration_s": opts.duration,
                   "precision": opts.precision, "parallelism": f"independent sims x{world}",
                   "l2": "inputs/outputs larger than L2 (BOLD 1.57 GB per step); no flush"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e2e_steps,
                "d2h_bytes_per_step": d2h // e2e_steps, "includes": "H2D params/SC, kernels, D2H outputs, GOF"},
        "gpu_launches": launches,
        "kernel_ms": {"integrate": float(np.mean(integ_ms)), "fc_fcd": float(np.mean(fc_ms))},
        "integrator": integrator,
        "fp64_path": fp64,
        "error_vs_fp64": line_errors,
        "roofline": roof,
        "clocks": ck,
    }
    if not opts.skip_cpu and rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(opts)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# Bounds of the mixed-precision mode against the FP64 run of the same inputs and noise
FC_BOUND, GOF_BOUND = 2e-3, 1e-3


def precision_error(o64, o32, emp_fc, emp_fcd):
    """Largest |FP32 - FP64| of BOLD, FC, FCD and of every GOF term over a batch."""
    from cubnm_b200 import utils
    g64 = utils.gof(o64["sim_fc_trils"], emp_fc, o64["sim_fcd_trils"], emp_fcd)
    g32 = utils.gof(o32["sim_fc_trils"], emp_fc, o32["sim_fcd_trils"], emp_fcd)
    d = lambda a, b: float(np.nanmax(np.abs(np.asarray(a) - np.asarray(b))))  # noqa: E731
    err = {"bold": d(o64["sim_bold"], o32["sim_bold"]), "fc": d(o64["sim_fc_trils"], o32["sim_fc_trils"]),
           "fcd": d(o64["sim_fcd_trils"], o32["sim_fcd_trils"]),
           "gof": {k: d(g64[k], g32[k]) for k in g64}}
    err["within_bounds"] = bool(err["fc"] <= FC_BOUND and max(err["gof"].values()) <= GOF_BOUND)
    err["bounds"] = {"fc": FC_BOUND, "gof": GOF_BOUND}
    if not err["within_bounds"]:
        raise SystemExit(f"FP32 path outside its error bounds against FP64: {err}")
    return err


def cpu_baseline(opts, sample=None):
    """The reference's CPU algorithm (oracle restatement, OpenMP over sims, all host
    threads) on a sample of the workload: 16 simulations per thread (256 on 16
    threads), so that the OpenMP split is even and the sample is ~1 minute."""
    from oracle import oracle
    threads = oracle.num_threads()
    sample = sample or 16 * threads
    args = workload_args(sample, opts.duration, "fp64", seed=0)
    t0 = time.perf_counter()
    oracle.run_simulations(*args)
    el = time.perf_counter() - t0
    return {"value": sample * opts.duration / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample} sims x {opts.duration} s of the workload (same params distribution), "
                      f"{el:.1f} s wall"}


def run_reference(opts, rank, world):
    """The reference arm: the reference's CPU algorithm (the oracle port), all host
    threads.  Each step is a sample of the workload whose size is set from an untimed
    probe so that the K timed steps take about --ref-budget seconds together (default
    240; at least two simulations per thread, at most 512 simulations)."""
    if rank != 0:
        return
    from oracle import oracle
    threads = oracle.num_threads()
    probe = 2 * threads
    args = workload_args(probe, opts.duration, "fp64", seed=0)
    t0 = time.perf_counter()
    oracle.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    per_sim = (time.perf_counter() - t0) / probe
    budget_s = opts.ref_budget / max(1, opts.steps)
    sample = int(budget_s / per_sim) // threads * threads
    sample = max(2 * threads, min(512, sample))
    args = workload_args(sample, opts.duration, "fp64", seed=0)
    for _ in range(max(0, min(opts.warmup, 1))):
        oracle.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    t0 = time.perf_counter()
    for _ in range(opts.steps):
        oracle.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    el = (time.perf_counter() - t0) / opts.steps
    value = sample * opts.duration / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": opts.steps, "warmup": opts.warmup, "ms_per_step": el * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_sims_per_step": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{sample} sims x {opts.duration} s per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- other configurations
# --config c0|c2|c3|c4 runs the other workloads of the benchmark plan with the same
# JSON contract.  c0 is run at full size.  c2 and c4 are too long for a routine run at
# full size (c2: 8,192 simulations of 60-900 s, ~3.8e6 simulated s; c4: 2,048 x 300 s
# at 1,000 nodes): their durations are divided by --scale (the line says by how much);
# simulations, node counts, densities and delays are as specified.  c3's gradient is one
# forward + backward of the adjoint on --grad-sims simulations at the full duration.
C2_NODES = (68, 100, 200, 400)
C2_DURATIONS = (60, 300, 600, 900)


def c2_groups(scale, precision="fp32", sims_per_group=512):
    """Uneven batch: 8,192 rWW simulations over node counts x durations (16 groups of
    512), delays from 3-D points in a 70-mm sphere x 1.3 at 6 m/s, SC at 20 %, regional
    w_p = w_p0 + w_p1 map.  Durations divided by `scale` (at least 4 s)."""
    from cubnm_b200 import synthetic
    groups = []
    for gi, (nodes, dur) in enumerate([(n, d) for n in C2_NODES for d in C2_DURATIONS]):
        d = max(4, int(round(dur / scale)))  # at least 4 s: with fewer volumes no FC window fits
        rng = np.random.default_rng(500 + gi)
        N = sims_per_group
        remove = min(10, d // 4)
        window = 30 if d - remove >= 60 else 2
        step = 5 if window == 30 else 1
        a = list(synthetic.synthetic_args("rWW", N=N, nodes=nodes, duration_s=d, seed=nodes, density=0.2,
                                          G=rng.uniform(0.001, 10, N), J_N=rng.uniform(0.001, 0.5, N),
                                          precision=precision, window_size=window, window_step=step,
                                          bold_remove_s=remove))
        fmap = np.random.default_rng(nodes + 100).standard_normal(nodes)
        a[5][0] = (rng.uniform(0, 2, N)[:, None] + rng.uniform(-1, 1, N)[:, None] * fmap[None, :]).ravel()
        a[3] = np.ascontiguousarray(synthetic.synthetic_lengths(nodes, nodes).ravel())
        a[6] = np.full(N, 6.0)
        a[11] = True
        groups.append(a)
    return groups


def c0_args():
    """The README grid: rWW 4 x 5 x 5 = 100 sims (G x w_p x J_N), 100 nodes, 60 s, FP64."""
    from cubnm_b200 import synthetic
    G, wp, jn = synthetic.rww_grid()
    return list(synthetic.synthetic_args("rWW", N=100, nodes=100, duration_s=60, seed=0, G=G, w_p=wp, J_N=jn,
                                         precision="fp64"))


def c3_args(n_sims=512, duration_s=300):
    """The gradient configuration: rWW, 200 nodes, SC at 25 %, FP32, FC + FCD w30 / s5;
    G and J_N uniform over the reference's bounds.  Returns (SC [200, 200], args)."""
    from cubnm_b200 import synthetic
    nodes = 200
    sc = synthetic.synthetic_sc(nodes, 0.25, 3)
    rng = np.random.default_rng(33)
    args = list(synthetic.synthetic_args("rWW", N=n_sims, nodes=nodes, duration_s=duration_s, seed=3, density=0.25,
                                         G=rng.uniform(0.001, 10, n_sims), J_N=rng.uniform(0.001, 0.5, n_sims),
                                         precision="fp32", window_size=30, window_step=5, bold_remove_s=30))
    args[1] = np.ascontiguousarray(sc.ravel())[None, :]
    return sc, args


def c4_args(n_sims, duration_s, precision="fp32"):
    """Wilson-Cowan, 1,000 nodes, SC at 10 % (lognormal, row-sum normalised: a sparse
    gather), delays as c2 at 6 m/s, noise sigma 0.01, G ~ U[0.001, 5]."""
    from cubnm_b200 import synthetic
    nodes = 1000
    rng = np.random.default_rng(44)
    a = list(synthetic.synthetic_args("WC", N=n_sims, nodes=nodes, duration_s=duration_s, seed=4, density=0.1,
                                      G=rng.uniform(0.001, 5, n_sims), precision=precision,
                                      window_size=30 if duration_s >= 90 else 2,
                                      window_step=5 if duration_s >= 90 else 1,
                                      bold_remove_s=min(30, duration_s // 4)))
    reg = a[5].reshape(8, n_sims, nodes)
    reg[6] = 0.01   # sigma_E
    reg[7] = 0.01   # sigma_I
    a[3] = np.ascontiguousarray(synthetic.synthetic_lengths(nodes, 4).ravel())
    a[6] = np.full(n_sims, 6.0)
    a[11] = True
    return a


def _copy_args(args):
    return [x.copy() if isinstance(x, np.ndarray) else x for x in args]


def _oracle_sample(args, sample, duration_s=None):
    """The reference CPU algorithm (oracle) on the first `sample` simulations of a
    group (optionally a shorter duration): sims x sim-s per s and the wall time."""
    from oracle import oracle
    from cubnm_b200 import shard
    a = shard.slice_args(args, 0, sample)
    if duration_s is not None:
        a[16] = int(duration_s * 1000)
        a[7] = dict(a[7], do_fc="0", do_fcd="0")
    t0 = time.perf_counter()
    oracle.run_simulations(*a)
    el = time.perf_counter() - t0
    return sample * a[16] / 1000 / el, el


def config_roofline(args, integrate_ms, delayed, fp32_peak=None):
    """Roofline of the integrator of a c2-c4 workload (per launch, mean CUDA-event
    time of the integrator).  Delayed networks: the ring-buffer gathers, 4 bytes per
    nonzero of the target's SC column per node-step, against the measured HBM copy
    bandwidth (no credit taken for L2 hits).  Without delays (c3): the FP32 work of a
    node-step (2 flops per nonzero of the coupling + the rWW update) against the
    measured FP32 peak."""
    from cubnm_b200 import core
    N, n = args[14], args[15]
    sc = np.asarray(args[1]).reshape(-1, n, n)
    nnz = float(np.count_nonzero(sc[np.asarray(args[2], dtype=int)])) / (N * n)  # mean nonzeros per target
    node_steps = N * n * (args[16] / args[20])
    t = integrate_ms / 1e3
    kernel = KERNEL_OF.get(core.last_integrator(), core.last_integrator())
    if delayed:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        b = node_steps * nnz * 4.0
        return {"bound": "hbm", "achieved": b / t / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": b / t / 1e9 / peaks["hbm_gbs"], "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "traffic": None, "algorithmic_bytes": b,
                "work": f"{nnz:.1f} ring-buffer gathers x 4 B per node-step, {node_steps:.3e} node-steps",
                "kernel": kernel, "kernel_ms": integrate_ms}
    flops = node_steps * (2.0 * nnz + RWW_FP32_FLOPS)
    return {"bound": "fp32", "achieved": flops / t / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": flops / t / 1e12 / fp32_peak, "peak_source": "measured on this GPU by cbnm_measure_fp32_peak",
            "traffic": None, "work": f"2 x {nnz:.1f} coupling + {RWW_FP32_FLOPS} update FP32 flops per node-step, "
                                     f"{node_steps:.3e} node-steps", "kernel": kernel, "kernel_ms": integrate_ms}


def batch_roofline(groups, seconds):
    """Roofline of an uneven batch (c2): the ring-buffer gather bytes of all groups
    (4 bytes per nonzero of the target's SC column per node-step) over the batch's
    wall time, against the measured HBM bandwidth.  The groups' integrators, FC and
    copies run concurrently on their own streams, so there is no single launch to
    time: this is a lower bound on the gathers' achieved bandwidth."""
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    b = 0.0
    for g in groups:
        N, n = g[14], g[15]
        sc = np.asarray(g[1]).reshape(-1, n, n)
        nnz = float(np.count_nonzero(sc[np.asarray(g[2], dtype=int)])) / (N * n)
        b += N * n * (g[16] / g[20]) * nnz * 4.0
    return {"bound": "hbm", "achieved": b / seconds / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": b / seconds / 1e9 / peaks["hbm_gbs"], "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
            "traffic": None, "algorithmic_bytes": b,
            "work": "ring-buffer gathers of every group, 4 B per nonzero per node-step",
            "basis": "whole-batch wall time (the groups' kernels run concurrently on their own streams)"}


def run_config(opts):
    import torch
    from cubnm_b200 import _abi, core, synthetic, utils
    from cubnm_b200._lib import lib, check
    from oracle import oracle
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = lib()
    threads = oracle.num_threads()
    st = torch.cuda.current_stream()
    clocks = Clocks(int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]))
    extra = {}

    def device_runner(args):
        sizes = _abi.Sizes()
        check(L.cbnm_query_sizes(C.byref(_abi.Prepared(*args).args), C.byref(sizes)))
        bufs, prep, outs = device_buffers(torch, args, sizes, dev)

        def step():
            check(L.cbnm_run_simulations_device(C.byref(prep.args), C.byref(outs)))
            return core.last_timing()
        return step, bufs

    if opts.config == "c0":
        args = c0_args()
        workload = "README grid: rWW 4x5x5 = 100 sims, 100 nodes, 60 s, FP64, FC+FCD w10/s2, no FIC"
        sim_s = 100 * 60
        step, _ = device_runner(args)
        for _ in range(opts.warmup):
            step()
        clocks.start()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launches = 0
        for _ in range(opts.steps):
            launches += step()["kernel_launches"]
        e1.record(st)
        torch.cuda.synchronize()
        ck = clocks.stop()
        ms = e0.elapsed_time(e1) / opts.steps
        t0 = time.perf_counter()
        out = core.run_simulations(*_copy_args(args))
        e2e_s = time.perf_counter() - t0
        tm = core.last_timing()
        e2e = {"value": sim_s / e2e_s, "unit": UNIT, "h2d_bytes_per_step": tm["h2d_bytes"],
               "d2h_bytes_per_step": tm["d2h_bytes"]}
        # parity with the reference's CPU algorithm on the same inputs and noise
        t0 = time.perf_counter()
        ref = oracle.run_simulations(*_copy_args(args))
        cpu_s = time.perf_counter() - t0
        rel = {k: float(np.max(np.abs(out[k] - ref[k]) / (np.abs(ref[k]) + 1e-12)))
               for k in ("sim_bold", "sim_fc_trils", "sim_fcd_trils")}
        extra["parity_vs_oracle_max_rel"] = rel
        cpu = {"value": sim_s / cpu_s, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"the whole workload (100 sims x 60 s), {cpu_s:.1f} s wall"}
        value, dtype = sim_s / (ms / 1e3), "f64"
        roof = None
    elif opts.config == "c2":
        scale = opts.scale or 15.0
        groups = c2_groups(scale)
        sim_s = sum(g[14] * g[16] / 1000 for g in groups)
        workload = (f"uneven batch: 8,192 rWW sims = 16 groups of 512 over nodes {C2_NODES} x durations "
                    f"{C2_DURATIONS} s divided by {scale:g}, delays 6 m/s (70-mm sphere x 1.3), SC 20%, "
                    f"w_p = w_p0 + w_p1 map, FP32, one cbnm_run_batch call")
        for _ in range(opts.warmup):
            core.run_batch([_copy_args(g) for g in groups])
        clocks.start()
        times, launches, h2d, d2h = [], 0, 0, 0
        for _ in range(opts.steps):
            gs = [_copy_args(g) for g in groups]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            core.run_batch(gs)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            tm = core.last_timing()
            launches += tm["kernel_launches"]
            h2d, d2h = tm["h2d_bytes"], tm["d2h_bytes"]
        ck = clocks.stop()
        ms = 1e3 * float(np.mean(times))
        value = sim_s / (ms / 1e3)
        e2e = {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "note": "the batch entry point takes host buffers: value is end to end"}
        # CPU: 2 x threads simulations of every (nodes, duration) group for 2 s, summed per group
        per_group = []
        for g in groups:
            v, el = _oracle_sample(g, 2 * threads, duration_s=2)
            per_group.append(g[14] * g[16] / 1000 / v)  # extrapolated seconds for the group
        cpu = {"value": sim_s / sum(per_group), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{2 * threads} sims x 2 s of each group, extrapolated per group to the batch"}
        dtype = "f32 (FP64 Balloon-Windkessel)"
        roof = batch_roofline(groups, ms / 1e3)
        extra["scale"] = scale
    elif opts.config == "c3":
        nodes, N, dur = 200, 512, 300
        sc, args = c3_args(N, dur)
        workload = "gradient config: rWW 512 sims, 200 nodes, 300 s, SC 25%, FP32, FC+FCD w30/s5"
        sim_s = N * dur
        step, _ = device_runner(args)
        for _ in range(opts.warmup):
            step()
        clocks.start()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launches = 0
        integ = []
        for _ in range(opts.steps):
            t = step()
            launches += t["kernel_launches"]
            integ.append(t["integrate_ms"])
        e1.record(st)
        torch.cuda.synchronize()
        ck = clocks.stop()
        ms = e0.elapsed_time(e1) / opts.steps
        value = sim_s / (ms / 1e3)
        t0 = time.perf_counter()
        out = core.run_simulations(*_copy_args(args))
        e2e_s = time.perf_counter() - t0
        tm = core.last_timing()
        e2e = {"value": sim_s / e2e_s, "unit": UNIT, "h2d_bytes_per_step": tm["h2d_bytes"],
               "d2h_bytes_per_step": tm["d2h_bytes"]}
        # one adjoint gradient (forward + backward) of the fit loss on --grad-sims simulations
        from cubnm_b200 import grad
        gs = opts.grad_sims
        prob = grad.RWWProblem(sc, nodes, dur, segment_steps=1000)
        emp = synthetic.synthetic_emp_bold(nodes, dur, 7)
        efc = torch.from_numpy(utils.calculate_fc(emp)).to(dev)
        efcd = torch.from_numpy(utils.calculate_fcd(emp, 30, 5)).to(dev)
        G = torch.tensor(np.random.default_rng(34).uniform(0.5, 3, gs), dtype=torch.float64, device=dev,
                         requires_grad=True)
        wp = torch.full((gs, nodes), 1.0, dtype=torch.float64, device=dev, requires_grad=True)
        jn = torch.full((gs, nodes), 0.15, dtype=torch.float64, device=dev, requires_grad=True)
        wie = torch.ones((gs, nodes), dtype=torch.float64, device=dev)
        sig = torch.full((gs, nodes), 0.01, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bold = prob.bold(G, wp, jn, wie, sig)
        loss = grad.rww_fit_loss(bold, efc, efcd, 30, 30, 5).sum()
        loss.backward()
        torch.cuda.synchronize()
        extra["gradient"] = {"sims": gs, "seconds": time.perf_counter() - t0,
                             "forward_ms": prob.last_forward_ms, "backward_ms": prob.last_backward_ms,
                             "finite": bool(torch.isfinite(G.grad).all().item())}
        v, el = _oracle_sample(args, 2 * threads, duration_s=10)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{2 * threads} sims x 10 s of the workload, {el:.1f} s wall"}
        f1, f2 = C.c_double(), C.c_double()
        check(L.cbnm_measure_fp32_peak(C.byref(f1), C.byref(f2)))
        dtype = "f32 (FP64 Balloon-Windkessel)"
        roof = config_roofline(args, float(np.mean(integ)), False, max(f1.value, f2.value))
    else:  # c4
        scale = opts.scale or 30.0
        dur = max(2, int(round(300 / scale)))
        N = 2048
        args = c4_args(N, dur)
        sim_s = N * dur
        workload = (f"large sparse network: Wilson-Cowan 1,000 nodes, 2,048 sims, 300 s divided by {scale:g}, "
                    f"SC 10% (sparse gather), delays 6 m/s, FP32")
        step, _ = device_runner(args)
        for _ in range(opts.warmup):
            step()
        clocks.start()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launches = 0
        integ = []
        for _ in range(opts.steps):
            t = step()
            launches += t["kernel_launches"]
            integ.append(t["integrate_ms"])
        e1.record(st)
        torch.cuda.synchronize()
        ck = clocks.stop()
        ms = e0.elapsed_time(e1) / opts.steps
        value = sim_s / (ms / 1e3)
        t0 = time.perf_counter()
        core.run_simulations(*_copy_args(args))
        e2e_s = time.perf_counter() - t0
        tm = core.last_timing()
        e2e = {"value": sim_s / e2e_s, "unit": UNIT, "h2d_bytes_per_step": tm["h2d_bytes"],
               "d2h_bytes_per_step": tm["d2h_bytes"]}
        v, el = _oracle_sample(args, threads, duration_s=1)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{threads} sims x 1 s of the workload, {el:.1f} s wall"}
        dtype = "f32 (FP64 Balloon-Windkessel)"
        roof = config_roofline(args, float(np.mean(integ)), True)
        extra["scale"] = scale
    line = {"metric": f"sims x sim-s per wall-s ({opts.config})", "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": opts.steps, "warmup": opts.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)",
            "config": {"workload": workload, "name": opts.config}, "e2e": e2e, "gpu_launches": launches,
            "roofline": roof, "cpu_baseline": cpu, "clocks": ck}
    line.update(extra)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--sims", type=int, default=N_SIMS)
    ap.add_argument("--duration", type=int, default=DURATION_S)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--traffic", type=float, default=None, help="ncu dram bytes per integrator launch")
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "c3", "c4"],
                    help="c1 (default): the headline workload; c0/c2/c3/c4: the other workloads (one GPU)")
    ap.add_argument("--scale", type=float, default=None, help="c2 / c4: divide the durations by this")
    ap.add_argument("--grad-sims", type=int, default=64, help="c3: simulations of the timed adjoint gradient")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="reference arm: seconds the timed CPU steps should take together")
    opts = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:  # one GPU per process
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    if opts.impl == "reference":
        run_reference(opts, rank, world)
    elif opts.config != "c1":
        if rank == 0:
            run_config(opts)
    else:
        run_ours(opts, rank, world, local_rank)


if __name__ == "__main__":
    main()
