// Internal interface between the host session (session.cpp) and the kernels.
// Not part of the public C ABI (include/cubnm_b200.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cbnm {

enum ModelId { MODEL_RWW = 0, MODEL_WC = 1, MODEL_JR = 2, MODEL_KURAMOTO = 3, MODEL_RWWEX = 4 };

// Raises `kernel`'s dynamic shared-memory limit to all the device allows (the
// opt-in maximum less the kernel's static shared memory).  The limit belongs to
// the function, process-wide, and the groups of a batch launch from several host
// threads at once: a limit set to each launch's own size could be lowered by
// another thread between its set and its launch.  Every caller sets this same
// value, so none can.  The launch's own size is checked by its caller.
template <class K>
inline cudaError_t allow_dynamic_smem(K kernel) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

// Balloon-Windkessel constants (reference: src/ext/models/bw.cpp:4-22).
struct BWConst {
    double dt, rho, alpha, tau, y, kappa, V_0, k1, k2, k3;
    double ialpha, itau, oneminrho, dt_itau, V_0_k1, V_0_k2, V_0_k3;
};

// Balloon-Windkessel constants in the form the FP32 tensor-core kernels use (FP64
// step with series for the powers, tc_common.cuh): filled on the host.
struct BWFast {
    double dt, kappa, y, dt_itau, ialpha, irho, log2_omr, ln_omr, omr, V0k1, V0k2, V0k3;
    double binom[13];            // C(1/alpha, k), k = 0..12
};

// Model constants, computed on the host exactly as the reference's
// init_constants(dt) does (src/ext/models/<model>.cpp).
struct RWWK {
    double dt, sqrt_dt, a_E, b_E, d_E, a_I, b_I, d_I, w_II, w_E__I_0, w_I__I_0, b_a_ratio_E;
    double dt_itau_E, dt_gamma_E, dt_itau_I, dt_gamma_I;
    // analytical-FIC constants (rww.cpp:42-53)
    double I_0, w_E, w_I, I_ext, tau_I_s, gamma_I_s, I_E_ss, S_E_ss;
};
struct WCK { double dt, sqrt_dt, itau_E, itau_I, a_E, a_I, mu_E, mu_I; };
struct JRK { double dt, sqrt_dt, A, B, a, b, v0, nu_max, r, mu, cmin, cmax, midpoint, a_sq, b_sq; };
struct KurK { double dt, sqrt_dt, twopi; };
struct RWWExK { double dt, sqrt_dt, J_N, a, b, d, dt_itau, dt_gamma; };
union ModelK {
    RWWK rww;
    WCK wc;
    JRK jr;
    KurK kur;
    RWWExK rwwex;
};

// Static description of each model (include/cubnm/models/<model>.hpp).
struct ModelDesc {
    const char *name;
    int id, n_state, n_inter, n_noise, n_global, n_regional, conn_idx, bold_idx, n_gout_bool, n_gout_int;
    bool osc, post_bw, modifies_params;
};
const ModelDesc *find_model(const char *name);

// Arguments of the integrator kernels (one persistent time loop per simulation).
struct IntegrateArgs {
    int nodes, n_sims, bw_it, inner_it, bold_tr_iters, states_sampling_iters, n_states_samples_remove;
    int noise_bw_it, bold_len, states_len, ext_out, states_ts;
    const double *sc;            // [n_scs][nodes*nodes] (FP64 kernel)
    const float *sc_f32;         // [n_scs][nodes*nodes] (FP32 kernel)
    const int *sc_idx;           // [n_sims]
    const double *gparams;       // [n_global][n_sims]
    const double *rparams;       // [n_regional][n_sims*nodes]
    double *rparams_out;         // wIE write-back (rWW FIC)
    const double *noise;         // [noise_size]
    const float *noise_f32;      // [noise_size] (FP32 kernel)
    const int *sh_nodes;         // [repeats][nodes]
    const int *sh_ts;            // [repeats][noise_bw_it]
    int has_delay;
    const int *delay;            // [n_tables][nodes*nodes] integration steps, row = source
    const int *delay_idx;        // [n_sims] table of each simulation
    const int *max_delay;        // [n_sims]
    const long long *hist_off;   // [n_sims] offset of each simulation's ring buffer
    double *hist;                // ring buffers (FP64 kernel)
    float *hist_f32;             // ring buffers (FP32 kernel)
    double *bold;                // [n_sims][bold_len*nodes]
    double *states;              // [n_state][n_sims][nodes or nodes*states_len]
    unsigned char *gbools;       // [n_gout_bool][n_sims]
    int *gints;                  // [n_gout_int][n_sims]
    int do_fic, max_fic_trials, I_start, I_end, I_dur;
    double init_delta;
    BWConst bw;
    ModelK K;
    int sim_begin;               // first simulation of this launch (FP64 kernel)
    int n_regional;              // regional parameters of the model
    const int *tiles;            // FP32 kernel: [n_tiles][1 + tile_width] = SC index, then simulation ids (-1 = empty)
    int n_tiles;
    int tile_width;              // FP32 kernel: simulations per tile (16 or 32)
    double bw_binom[13];         // FP32 kernel: binomial coefficients C(1/alpha, k), k = 0..12
    BWFast bwf;                  // two-tile kernel: Balloon-Windkessel constants
    alignas(8) float k32[24];    // two-tile kernel: the model's FP32 constants (M::K)
    int *status;                 // device status word (0 = ok)
    double *bw_scratch;          // two-tile kernel: per-CTA Balloon-Windkessel state (pp_bw_scratch_bytes)
    int pp_grid;                 // two-tile kernel: CTAs launched (the scratch holds this many)
    int pp_ws;                   // two-tile kernel: 1 = warp-specialised halves (1024 threads), 0 = 544 threads
    // lane kernel (integrate_lanes.cu): groups of 16 simulations sharing SC and delay table
    const int *ln_groups;        // [ln_n_groups][3 + 16] = SC index, delay table, max delay (1 without delays), simulations
    int ln_n_groups;
    int ln_grid;                 // CTAs launched (the ring-buffer and Balloon-Windkessel scratch hold this many)
    int ln_threads;              // 1024 (64 node rows a CTA, one CTA an SM) or 512 (32 rows, two an SM; <= 128 nodes)
    float *ln_params;            // [ln_n_groups][nodes][n_regional][16]  (written by the launcher)
    float *ln_hist;              // [ln_grid][ln_hist_per_cta]  ring buffers [slot][node][16]
    long long ln_hist_per_cta;   // floats per CTA: (largest max delay + 1) * nodes * 16
    double *ln_bw;               // [ln_grid][nodes][4 or 8][16]  Balloon-Windkessel state (+ its tangent)
    double *tan_bold;            // non-null: the lane kernel also integrates d/dG, dBOLD/dG here [n_sims][bold_len][nodes]
    // Sparse coupling (per-simulation kernels), ELLPACK by target node: entry q of
    // node j at [q * nodes + j]; ell_k entries per node, zero-weight padding last.
    // One entry = the SC weight packed with the source's offset into the ring
    // buffer, d * nodes + k (d = delay in steps of the pair k -> j; without
    // delays d = 0 and the offset is the source node k), read by one vector load.
    int ell_k;                   // 0 = dense coupling
    int ell_tables;              // delay tables packed per SC (1 without delays)
    const int2 *ell_pk32;        // [n_scs][ell_tables][ell_k][nodes] {offset, float weight bits} (FP32 kernel)
    const int4 *ell_pk64;        // [n_scs][ell_tables][ell_k][nodes] {weight lo, weight hi, offset, 0} (FP64 kernel)
};

// FC / FCD (reference: src/ext/fc.cu, src/ext/fc.cpp).
struct FcArgs {
    int nodes, bold_len, n_vols_remove, n_pairs, n_windows, n_window_pairs;
    int max_T;                   // longest volume range of the static FC and the windows
    int sim_begin, sim_count;
    const int *w_start, *w_end;  // [n_windows] inclusive volume ranges
    const int *pair_i, *pair_j;  // [n_pairs] node pair of each FC entry
    const double *bold;          // [n_sims][bold_len*nodes]
    double *fc;                  // [n_sims][n_pairs]
    double *fcd;                 // [n_sims][n_window_pairs]
    double *wfc;                 // scratch [sim_count][n_windows][n_pairs]
    double *wstat;               // scratch [sim_count][n_windows][2] (mean, ssd)
    int *status_fc;              // tensor-core FC: set to 1 if a bounded wait gave up
};

// Goodness of fit.
struct GofArgs {
    int n_sims, n_pairs, n_wp, n_emp_fcd;
    const double *sim_fc, *emp_fc, *sim_fcd, *emp_fcd_sorted;
    double emp_fc_mean, emp_fc_ssd;  // mean and sqrt(sum (x - mean)^2) of emp_fc
    double *fc_corr, *fc_diff, *fc_normec, *fcd_ks;
};

// launchers (return cudaGetLastError() of the launch)
cudaError_t launch_integrate_fp64(int model, const IntegrateArgs &a, cudaStream_t st);
cudaError_t launch_integrate_fp32(int model, const IntegrateArgs &a, cudaStream_t st, int *launches);
cudaError_t launch_integrate_simt32(int model, const IntegrateArgs &a, cudaStream_t st);  // FP32, one CTA per simulation
// FP32 with 16 simulations on the lanes (integrate_lanes.cu): delays and/or > 128 nodes.
bool lanes_supported(int model, int nodes, bool numerical_fic);
bool lanes_tangent_supported(int model);
int lanes_rows(int nodes, int threads);
cudaError_t launch_integrate_lanes(int model, const IntegrateArgs &a, cudaStream_t st);
// The parameter layout of a run (first half of launch_integrate_lanes), and one
// persistent launch over the 16-simulation groups of several runs of one model:
// items [n_items] = (run, group), longest first; scratch per CTA for the largest run.
cudaError_t launch_integrate_lanes_params(int model, const IntegrateArgs &a, cudaStream_t st);
cudaError_t launch_integrate_lanes_multi(int model, const IntegrateArgs *runs, const int2 *items, int n_items,
                                         int *counter, int mn, int grid, float *hist, long long hist_per_cta,
                                         double *bw, long long bw_per_cta, cudaStream_t st);
bool fp32_supported(int model, int nodes, bool has_delay);
// Two-tile tensor-core kernel (integrate_pp.cu): rWW, no delays, <= 128 nodes.
// Work items: [n_tiles][1 + 64] = SC index, then 32 simulation ids per half (-1 = empty).
bool pp_supported(int model, int nodes, bool has_delay);
size_t pp_bw_scratch_bytes(int nodes, int grid);
cudaError_t launch_integrate_pp(int model, const IntegrateArgs &a, cudaStream_t st, int *launches);
int fp32_tile_for(int nodes);  // simulations per FP32 tile for a node count
// rWW analytical FIC (fic.cu): wIE written into regional row 2 in place.
struct FicArgs {
    int nodes, n_sims;
    const double *sc;            // [n_scs][nodes*nodes]
    const int *sc_idx;           // [n_sims]
    const double *gparams;       // [1][n_sims] G
    double *regional;            // [n_regional][n_sims*nodes] (w_p, J_N read; wIE written)
    unsigned char *unstable;     // [n_sims] 1 where FIC failed (wIE set to 1)
    RWWK K;
};
cudaError_t launch_rww_fic(const FicArgs &a, cudaStream_t st);
// Normal noise from Philox4x32-10 + Box-Muller (noise.cu); out32 may be null.
cudaError_t launch_philox_normals(uint32_t seed, double *out, float *out32, size_t count, cudaStream_t st);
cudaError_t launch_fc(const FcArgs &a, cudaStream_t st, int *launches);
cudaError_t launch_fcd_only(const FcArgs &a, cudaStream_t st, int *launches);  // FCD of window FCs already in a.wfc
// FC / window FCs on the tensor cores (fc_tc.cu; FP32 mode); pidx [nodes*nodes]: pair index of (i > j) or -1.
cudaError_t launch_fc_tc(const FcArgs &a, const int *pidx, cudaStream_t st, int *launches);
cudaError_t launch_gof(const GofArgs &a, cudaStream_t st, int *launches);
size_t gof_ks_smem_limit();

// Loss of the gradient fit, (1 - r(FC)) + W1(FCD), and dL/dBOLD (fit_loss.cu).
struct FitLossArgs {
    int nodes, bold_len, n_vols_remove, n_pairs, n_windows, n_window_pairs;
    int sim_begin, sim_count, want_grad;
    const int *w_start, *w_end;  // [n_windows] inclusive volume ranges
    const double *bold;          // [n_sims][bold_len][nodes]
    const double *emp_c;         // [n_pairs] empirical FC minus its mean
    double emp_norm;             // |emp_c|
    const double *emp_q;         // [n_window_pairs] empirical FCD quantile at each simulated rank
    double *loss_fc, *loss_fcd;  // [n_sims]
    double *dbold;               // [n_sims][bold_len][nodes]
    // scratch of the chunk [sim_count]...
    double *fc, *wfc, *fcd, *wstat, *stats, *g_fc, *g_fcd, *g_wfc;
};
cudaError_t launch_fit_loss(const FitLossArgs &a, cudaStream_t st, int *launches);
// FP32 FMA throughput of the current device (peak.cu), TFLOP/s, scalar and packed.
cudaError_t measure_fp32_peak(double *ffma_tflops, double *ffma2_tflops);
size_t fit_loss_sort_smem(int n_window_pairs);

// Adjoint (reverse-mode) pass of the FP32 rWW integrator + FP64 Balloon-Windkessel
// model with the noise held fixed (adjoint.cu).  Checkpoints of the state every
// seg_bw Balloon-Windkessel steps; the backward pass recomputes each segment
// into a scratch and runs it in reverse.
struct AdjArgs {
    IntegrateArgs ia;            // forward arguments (FP32 SC, FP32 noise, BOLD, constants)
    const float *sct_f32;        // [n_scs][nodes*nodes] transposed SC: sct[a][b] = SC[b][a]
    int seg_bw, n_seg;           // Balloon-Windkessel steps per segment, segments per simulation
    float *ck_s;                 // [n_sims][n_seg][2][nodes]  S_E, S_I at each segment start
    double *ck_bw;               // [n_sims][n_seg][4][nodes]  x, f, nu, q at each segment start
    const double *dbold;         // [n_sims][bold_len][nodes]  dL/dBOLD
    float *scr_s;                // [chunk][seg_bw*inner_it][3][nodes]  S_E, S_I, input before each step
    float *scr_z;                // [chunk][seg_bw][nodes]  Balloon-Windkessel input of each step
    double *scr_bw;              // [chunk][seg_bw][4][nodes]  Balloon-Windkessel state before each step
    double *grad_g;              // [1][n_sims]   dL/dG
    double *grad_r;              // [4][n_sims*nodes]  dL/d(w_p, J_N, wIE, sigma)
    int sim_begin, sim_count;    // simulations of this launch (backward: the scratch chunk)
};
cudaError_t launch_adjoint_forward(const AdjArgs &a, cudaStream_t st);
cudaError_t launch_adjoint_backward(const AdjArgs &a, cudaStream_t st);
cudaError_t launch_transpose_sc(const double *sc, float *sc_f32, float *sct_f32, int n_scs, int nodes, cudaStream_t st);

// FC / FCD of device BOLD with the window FCs in a fixed file-scope device
// array of NOALLOC_SCRATCH_BYTES (fc_noalloc.cu); allocates no device memory.
// Returns a C-ABI status code and writes a message into msg[cap].
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;
int fc_fcd_noalloc(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                   int window_step, int drop_edges, int exc_inter, double *fc, double *fcd, cudaStream_t st,
                   char *msg, size_t cap);

}  // namespace cbnm
