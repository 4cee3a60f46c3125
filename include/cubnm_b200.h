/*
 * cubnm_b200 C ABI -- the drop-in boundary of the B200 simulation path.
 *
 * The reference exposes this path as the CPython extension `cubnm.core`
 * (src/ext/core.cpp:507-626) with three functions: run_simulations, init and
 * set_const.  This header restates that boundary as plain C: pointers and
 * sizes, status codes instead of exceptions, no Python or torch types.  A thin
 * binding (ctypes, cgo, JNI, ...) rebuilds the `cubnm.core` module on top of it.
 *
 * Array layouts follow the reference exactly (row-major, C order):
 *   sc               [n_scs][nodes*nodes]    rows = source node, cols = target
 *   sc_indices       [n_sims]                int32, index into sc
 *   sc_dist          [nodes*nodes]           tract lengths (mm), used with do_delay
 *   global_params    [n_global][n_sims]      e.g. rWW: G
 *   regional_params  [n_regional][n_sims*nodes]  sim-major, node-minor
 *   v_list           [n_sims]                conduction velocity (m/s = mm/ms)
 * Outputs (caller-allocated, sized by cbnm_query_sizes):
 *   sim_bold         [n_sims][bold_len*nodes]   volume-major per simulation
 *   sim_fc_trils     [n_sims][n_pairs]          lower triangle, np.tril_indices(n,-1) order
 *   sim_fcd_trils    [n_sims][n_window_pairs]   lower triangle of the window-by-window matrix
 *   sim_states       [n_state_vars][n_sims][nodes (*states_len if states_ts)]
 *   global_bools     [n_global_out_bool][n_sims]  (uint8, 0/1)
 *   global_ints      [n_global_out_int][n_sims]
 *   noise            [noise_size]; shuffled_nodes [noise_repeats][nodes];
 *   shuffled_ts      [noise_repeats][noise_bw_it]
 *
 * Thread safety: like the reference (a process-global model object,
 * core.cpp:57-58), the library keeps one session per process; calls must not
 * overlap.  Errors return a non-zero status; cbnm_last_error() describes it.
 *
 * Devices: the session (stream, events, device buffers, noise cache) belongs to
 * the CUDA device that was current at the first call.  Use one device per
 * process; a run call made while another device is current returns
 * CBNM_ERR_CUDA.  cbnm_reset() frees the session on its own device, after which
 * the next call opens a new one on the then-current device.
 */
#ifndef CUBNM_B200_H
#define CUBNM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CBNM_OK 0
#define CBNM_ERR_ARG 1          /* invalid argument or size */
#define CBNM_ERR_MODEL 2        /* unknown model name */
#define CBNM_ERR_CONFIG 3       /* configuration rejected (e.g. no FC windows) */
#define CBNM_ERR_CUDA 4         /* CUDA runtime error; message starts with "CUDA Error" */
#define CBNM_ERR_TIMEOUT 5      /* a bounded device-side wait gave up */
#define CBNM_ERR_UNSUPPORTED 6  /* request outside what this library implements */

/* Arguments of one run; positional arguments of core.cpp:202-225 in order. */
typedef struct cbnm_run_args {
    const char *model_name;            /* "rWW", "WC", "JR", "Kuramoto", "rWWEx" */
    const double *sc;                  /* [n_scs][nodes*nodes] */
    int n_scs;
    const int32_t *sc_indices;         /* [n_sims] */
    const double *sc_dist;             /* [nodes*nodes] */
    double *global_params;             /* [n_global][n_sims]; written back when the model modifies params */
    double *regional_params;           /* [n_regional][n_sims*nodes]; idem (rWW FIC writes wIE) */
    const double *v_list;              /* [n_sims] */
    const char *const *config_keys;    /* model_config dict as parallel key/value string arrays */
    const char *const *config_values;
    int n_config;
    int ext_out;                       /* always 1 in the reference's caller (base.py:736) */
    int states_ts;
    int noise_out;
    int do_delay;
    int force_reinit;
    int use_cpu;                       /* must be 0: this library has no CPU path */
    int n_sims;
    int nodes;
    int time_steps;                    /* duration in ms */
    int bold_tr;                       /* ms */
    int states_sampling;               /* ms */
    int sim_seed;
    double dt;                         /* model step, ms */
    double bw_dt;                      /* Balloon-Windkessel step, ms */
} cbnm_run_args;

/* Output sizes for a given set of arguments (core.cpp:336-349). */
typedef struct cbnm_sizes {
    int n_global_params;
    int n_regional_params;
    int n_state_vars;
    int n_global_out_bool;
    int n_global_out_int;
    int bold_len;
    int n_pairs;
    int n_windows;
    int n_window_pairs;
    int states_len;
    int do_fc;
    int do_fcd;
    int modifies_params;
    int noise_repeats;
    int noise_bw_it;
    int64_t noise_size;
} cbnm_sizes;

typedef struct cbnm_outputs {
    double *sim_bold;
    double *sim_fc_trils;      /* may be NULL when do_fc is off */
    double *sim_fcd_trils;     /* may be NULL when do_fcd is off */
    double *sim_states;        /* may be NULL when ext_out is off */
    uint8_t *global_bools;
    int32_t *global_ints;
    double *noise;             /* only written when noise_out */
    int32_t *shuffled_nodes;
    int32_t *shuffled_ts;
    double init_time;          /* seconds, written by the library */
    double run_time;           /* seconds, written by the library */
} cbnm_outputs;

/* Device timings of the last run, in milliseconds (CUDA events). */
typedef struct cbnm_timing {
    double integrate_ms;       /* the integrator kernel (neural model + BOLD) */
    double fc_ms;              /* FC / FCD kernels */
    double h2d_ms;             /* host-to-device copies of the inputs */
    double d2h_ms;             /* device-to-host copies of the outputs */
    double total_ms;
    int64_t h2d_bytes;
    int64_t d2h_bytes;
    int kernel_launches;       /* kernels this library launched in the run */
} cbnm_timing;

/* core.cpp:147-155 -- resets the Balloon-Windkessel constants to their defaults. */
int cbnm_init(void);

/* core.cpp:157-192 -- sets k1, k2, k3 or V_0 of the Balloon-Windkessel model. */
int cbnm_set_const(const char *key, double value);

/* Sizes of every output of run_simulations for these arguments (core.cpp:336-349). */
int cbnm_query_sizes(const cbnm_run_args *args, cbnm_sizes *sizes);

/* core.cpp:194-493 (run_simulations) -- host buffers in, host buffers out.
 * Extra model_config key understood by this library: "precision" = "fp64"
 * (default; matches the reference's double build) or "fp32" (FP32 node state,
 * tensor-core coupling; FP64 Balloon-Windkessel and FC/FCD denominators). */
int cbnm_run_simulations(const cbnm_run_args *args, cbnm_outputs *out);

/* Same as cbnm_run_simulations, but every array pointer in args and out is a
 * device pointer on the current CUDA device (inputs already resident in HBM).
 * No reference counterpart: it is the device-resident form of core.cpp:194-493. */
int cbnm_run_simulations_device(const cbnm_run_args *args, cbnm_outputs *out);

/* cbnm_run_simulations_device plus the derivative of BOLD with respect to each
 * simulation's global coupling G, integrated alongside (forward mode: the
 * tangent of the node state, of the delayed coupling through the ring buffer and
 * of the FP64 Balloon-Windkessel state; the noise held fixed).  No counterpart
 * in the reference, which has no derivatives (src/cubnm/optimize.py fits by
 * grid / CMA-ES); it differentiates the reference's time loop
 * (src/ext/bnm.cu:117-505, models/wc.cpp:51-80, models/rww.cpp:194-232).
 * dL/dG of a loss on BOLD is then sum(dL/dBOLD * dBOLD/dG) per simulation.
 * Forward mode needs no checkpoints, so it serves delayed networks, whose
 * reverse pass would have to store D steps of ring buffer per checkpoint.
 * Scope: precision "fp32", models "rWW" and "WC", <= 1024 nodes, no numerical FIC.
 *   dbold_dG [n_sims][bold_len][nodes] (device), same layout as sim_bold. */
int cbnm_run_tangent_device(const cbnm_run_args *args, cbnm_outputs *out, double *dbold_dG);

/* Several independent runs ("groups": each a full cbnm_run_simulations call with
 * HOST buffers, possibly of different models, node counts, durations, delays and
 * precisions) executed concurrently.  No counterpart in the reference, whose
 * interface runs one group per call (src/ext/core.cpp:194-493); a group of a
 * few hundred small networks fills only part of a B200, so running the groups
 * of an uneven batch side by side fills it.  Up to 16 groups run at once, each
 * on its own stream with its own device buffers and noise cache (kept across
 * calls, freed by cbnm_reset).  Outputs equal those of separate
 * cbnm_run_simulations calls.  statuses (optional, [n_groups]) receives each
 * group's status; the return value is the first failing group's status (0 if
 * none) and cbnm_last_error() names that group. */
int cbnm_run_batch(const cbnm_run_args *args, cbnm_outputs *outs, int n_groups, int *statuses);

/* Timings of the last cbnm_run_simulations[_device] / cbnm_run_batch /
 * cbnm_adjoint_* call (for a batch: wall time in total_ms, the longest group's
 * kernel times, summed transfer sizes and launches). */
int cbnm_last_timing(cbnm_timing *timing);

/* Drops the cached session (device buffers and noise); core.cpp keeps it for
 * the process lifetime, this lets a host free the memory early. */
int cbnm_reset(void);

/* Human-readable description of the last error (empty if none). */
const char *cbnm_last_error(void);

/* Integrator of the last run on this thread: "fp64", or for precision "fp32"
 * "tc2" (two-tile tensor-core kernel), "tc1" (single-tile tensor-core kernel),
 * "lanes" / "lanes512" (simulations on the lanes, 1024 / 512 threads a CTA) or
 * "simt" (one CTA per simulation).  No reference counterpart (diagnostic). */
const char *cbnm_last_integrator(void);

/* FP32 fused-multiply-add throughput of the current device in TFLOP/s (two flops
 * a lane per FMA), scalar and packed two-wide: the measured denominator of the
 * integrators' FP32 roofline.  Takes about a quarter of a second.  No reference
 * counterpart (diagnostic). */
int cbnm_measure_fp32_peak(double *ffma_tflops, double *ffma2_tflops);

/* Forgets the autotuner's choices (model_config "autotune" = "1" or
 * CBNM_AUTOTUNE=1: the first run of each workload -- model, nodes, largest
 * delay, number of SCs -- times a short probe of every applicable FP32
 * integrator on up to 2,368 of its simulations and keeps the fastest; with
 * CBNM_TUNE_FILE set the choices are also appended to and read from that file).
 * Forced variants for testing: CBNM_FP32_KERNEL / CBNM_FP32_TC.  No reference
 * counterpart: the reference has one kernel. */
int cbnm_tune_reset(void);

/* Goodness-of-fit seam (src/cubnm/utils.py:416-507 fc_corr_device and
 * :306-414 fcd_ks_device; src/cubnm/sim/base.py:1165-1189 for fc_diff and
 * fc_normec).  Host arrays; all outputs [n_sims].
 *   fc_corr  : Pearson r between each sim_fc row and emp_fc
 *   fc_diff  : |mean(sim_fc) - mean(emp_fc)|
 *   fc_normec: ||sim_fc - emp_fc||_2 / (2 sqrt(n_pairs))
 *   fcd_ks   : two-sample Kolmogorov-Smirnov distance between each sim_fcd row and emp_fcd
 * Any output pointer may be NULL to skip that term. */
int cbnm_gof(const double *sim_fc, int n_sims, int n_pairs, const double *emp_fc,
             const double *sim_fcd, int n_window_pairs, const double *emp_fcd, int n_emp_fcd,
             double *fc_corr, double *fc_diff, double *fc_normec, double *fcd_ks);

/* Gradients (reverse mode) of a loss on BOLD with respect to the rWW parameters,
 * noise held fixed.  No counterpart in the reference, which fits parameters by
 * grid search and gradient-free optimisers only (src/cubnm/optimize.py); it
 * integrates the same model (src/ext/models/rww.cpp:194-232, bnm.cu:117-505).
 * Scope: model "rWW", no delays, do_fic = 0; the node state is FP32, the
 * Balloon-Windkessel state FP64 (the "fp32" precision of cbnm_run_simulations,
 * per-simulation kernel, so the forward BOLD equals that run's BOLD).
 * All array pointers of args are DEVICE pointers (as cbnm_run_simulations_device).
 *
 * 1. cbnm_adjoint_query: sizes of the caller-allocated device buffers.
 *    segment_steps: integration steps between checkpoints (a multiple of
 *    bw_dt / dt; 1000 = 0.1 s at dt = 0.1 ms).
 * 2. cbnm_adjoint_forward: BOLD [n_sims][bold_len][nodes] + checkpoints.
 * 3. the caller forms dL/dBOLD (same layout) on the device.
 * 4. cbnm_adjoint_backward: dL/dG -> grad_global [1][n_sims];
 *    dL/d(w_p, J_N, wIE, sigma) per node -> grad_regional [4][n_sims*nodes].
 *    Recomputes each segment from its checkpoint into the scratch.
 * Inputs (SC, parameters, seed, sizes) must be the same in 2 and 4. */
typedef struct cbnm_adjoint_sizes {
    int64_t n_segments;               /* checkpoints per simulation */
    int64_t checkpoint_bytes;         /* device bytes for the checkpoints of all simulations */
    int64_t scratch_bytes;            /* device bytes of backward scratch */
    int64_t bold_len;                 /* BOLD volumes per simulation */
    int64_t sims_per_backward_launch; /* simulations the scratch holds at once */
} cbnm_adjoint_sizes;

int cbnm_adjoint_query(const cbnm_run_args *args, int segment_steps, cbnm_adjoint_sizes *sizes);
int cbnm_adjoint_forward(const cbnm_run_args *args, int segment_steps, double *bold, void *checkpoints);
int cbnm_adjoint_backward(const cbnm_run_args *args, int segment_steps, const double *dbold,
                          const void *checkpoints, void *scratch, double *grad_global,
                          double *grad_regional);

/* Loss of the gradient fit and its gradient with respect to BOLD, for simulated
 * BOLD in device memory.  No counterpart in the reference, whose optimisers score
 * simulations by GOF terms without derivatives (src/cubnm/sim/base.py:1084-1207,
 * src/cubnm/optimize.py); the terms are those scores made differentiable:
 *   loss_fc[s]  = 1 - Pearson r(FC lower triangle of s, emp_fc)
 *   loss_fcd[s] = W1 between the FCD values of s and emp_fcd: mean over the m
 *                 sorted simulated values of |sorted_i - Q_emp((i + 1/2) / m)|,
 *                 Q_emp(p) = sorted emp_fcd[floor(p n_emp_fcd)]  (0 with < 2 windows)
 * FC / FCD as run_simulations computes them (volumes [n_vols_remove, bold_len),
 * windows of window_size / window_step / drop_edges, src/ext/utils.cpp:21-52).
 *   bold   [n_sims][bold_len][nodes] device; emp_fc [n_pairs] and emp_fcd host;
 *   loss_fc, loss_fcd [n_sims] device; dbold [n_sims][bold_len][nodes] device =
 *   d(loss_fc + loss_fcd)/dBOLD per simulation, or NULL for the loss only.
 * FP64 throughout; the call returns when the results are written. */
int cbnm_fit_loss(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                  int window_step, int drop_edges, const double *emp_fc, const double *emp_fcd, int n_emp_fcd,
                  double *loss_fc, double *loss_fcd, double *dbold);

/* FC and FCD of simulated BOLD already in device memory, allocating no device
 * memory.  No counterpart in the reference: there, FC and FCD are computed only
 * inside run_simulations (src/ext/bnm.cu:809-942).  It is for callers that
 * cannot allocate on the device: a host whose pooling allocator already holds
 * the free device memory, or a loop that keeps integration running on other
 * streams, which the implicit device-wide synchronisation of cudaFree would
 * stall.
 *   bold  [n_sims][bold_len*nodes] (device), volume-major per simulation
 *   fc    [n_sims][n_pairs] (device) -- same values and order as sim_fc_trils
 *   fcd   [n_sims][n_window_pairs] (device) or NULL for FC only -- as sim_fcd_trils
 *   n_vols_remove: volumes dropped before FC (bold_remove_s * 1000 / BOLD_TR);
 *   window_size, window_step, drop_edges, exc_interhemispheric: as in model_config.
 *   stream: a cudaStream_t (NULL = the default stream); the call only enqueues.
 * The window FCs of each chunk of simulations go to one fixed device array of
 * CBNM_NOALLOC_SCRATCH_BYTES per device (32 MiB); a batch whose single
 * simulation needs more (n_windows * n_pairs * 8 bytes) is rejected with
 * CBNM_ERR_ARG.  No buffer has to start zeroed.  The scratch is shared, so
 * calls whose kernels overlap on one device race: serialise them (one stream,
 * or events).  The first call on each device looks up the scratch address
 * (cudaGetSymbolAddress, with that device current), which can load the module
 * that holds it; make that first call before any stream capture begins. */
#define CBNM_NOALLOC_SCRATCH_BYTES (32u << 20)
int cbnm_fc_fcd_noalloc(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove,
                        int window_size, int window_step, int drop_edges, int exc_interhemispheric,
                        double *fc, double *fcd, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CUBNM_B200_H */
