// Host side of the cubnm_b200 C ABI (include/cubnm_b200.h).
//
// Replaces the reference's CPython boundary and session logic:
//   run_simulations / init / set_const   src/ext/core.cpp:147-504
//   model object sizes and config        include/cubnm/models/base.hpp:51-124, 271-297
//   session init (noise, windows, pairs) src/ext/bnm.cu:990-1265
//   run (params, delays, kernels, copy)  src/ext/bnm.cu:507-988
//   rWW analytical FIC                   src/ext/models/rww.cpp:73-146, rww_fic.cpp:62-231
// Design differences: plain device allocations (no managed memory), one
// stream, CUDA-event timings, status codes instead of exceptions, a cached
// session keyed on everything that changes the noise (as bnm.cu:1207-1215).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <condition_variable>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#include <thread>
#include <atomic>

#include <cuda_runtime.h>

#include "../../include/cubnm_b200.h"
#include "engine.h"
#include "tc_common.cuh"

namespace cbnm {

// ---------------------------------------------------------------- models
static const ModelDesc kModels[] = {
    // name, id, states, inter, noise, global, regional, conn, bold, gout_bool, gout_int, osc, post_bw, modifies
    {"rWW", MODEL_RWW, 6, 7, 2, 1, 4, 4, 4, 2, 1, false, true, true},
    {"WC", MODEL_WC, 2, 4, 2, 1, 8, 0, 0, 0, 0, false, false, false},
    {"JR", MODEL_JR, 8, 9, 1, 1, 6, 7, 6, 0, 0, false, false, false},
    {"Kuramoto", MODEL_KURAMOTO, 1, 1, 1, 1, 3, 0, 0, 0, 0, true, false, false},
    {"rWWEx", MODEL_RWWEX, 3, 2, 1, 1, 3, 2, 2, 0, 0, false, false, false},
};

const ModelDesc *find_model(const char *name) {
    if (!name) return nullptr;
    for (const auto &m : kModels)
        if (std::strcmp(m.name, name) == 0) return &m;
    return nullptr;
}

struct Err : std::runtime_error {
    int code;
    Err(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            throw Err(CBNM_ERR_CUDA, std::string("CUDA Error: ") + cudaGetErrorString(e_) + " at " +    \
                                         __FILE__ + ":" + std::to_string(__LINE__));                    \
    } while (0)

// ---------------------------------------------------------------- constants
static BWConst bw_defaults(double dt_s) {  // bw.cpp:4-22
    BWConst c;
    c.dt = dt_s; c.rho = 0.34; c.alpha = 0.32; c.tau = 0.98; c.y = 1.0 / 0.41; c.kappa = 1.0 / 0.65;
    c.V_0 = 0.02 * 100; c.k1 = 7 * c.rho; c.k2 = 2.0; c.k3 = 2 * c.rho - 0.2;
    c.ialpha = 1.0 / c.alpha; c.itau = 1.0 / c.tau; c.oneminrho = (1.0 - c.rho); c.dt_itau = c.dt * c.itau;
    c.V_0_k1 = c.V_0 * c.k1; c.V_0_k2 = c.V_0 * c.k2; c.V_0_k3 = c.V_0 * c.k3;
    return c;
}
static BWConst g_bw = bw_defaults(0.001);
static std::string g_err;

static ModelK make_constants(int model, double dt) {
    ModelK K;
    std::memset(&K, 0, sizeof(K));
    switch (model) {
        case MODEL_RWW: {  // rww.cpp:8-53
            RWWK &m = K.rww;
            m.dt = dt; m.sqrt_dt = std::sqrt(m.dt);
            m.a_E = 310; m.b_E = 125; m.d_E = 0.16; m.a_I = 615; m.b_I = 177; m.d_I = 0.087;
            const double gamma_E = (double)0.641 / (double)1000.0, gamma_I = (double)1.0 / (double)1000.0;
            const double tau_E = 100, tau_I = 10;
            m.I_0 = 0.382; m.w_E = 1.0; m.w_I = 0.7; m.w_II = 1.0; m.I_ext = 0.0;
            m.w_E__I_0 = m.w_E * m.I_0; m.w_I__I_0 = m.w_I * m.I_0; m.b_a_ratio_E = m.b_E / m.a_E;
            const double itau_E = 1.0 / tau_E, itau_I = 1.0 / tau_I;
            m.dt_itau_E = m.dt * itau_E; m.dt_gamma_E = m.dt * gamma_E;
            m.dt_itau_I = m.dt * itau_I; m.dt_gamma_I = m.dt * gamma_I;
            m.tau_I_s = 0.01; m.gamma_I_s = 1.0; m.I_E_ss = 0.3773805650; m.S_E_ss = 0.1647572075;
            break;
        }
        case MODEL_WC: {  // wc.cpp:14-25
            WCK &m = K.wc;
            m.dt = dt; m.sqrt_dt = std::sqrt(m.dt);
            const double tau_E = 2.5, tau_I = 3.75;
            m.itau_E = 1.0 / tau_E; m.itau_I = 1.0 / tau_I; m.a_E = 1.5; m.a_I = 1.5; m.mu_E = 3.0; m.mu_I = 3.0;
            break;
        }
        case MODEL_JR: {  // jr.cpp:14-30
            JRK &m = K.jr;
            m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.A = 3.25; m.B = 22.0; m.a = 0.1; m.b = 0.05; m.v0 = 6.0;
            m.nu_max = 0.0025; m.r = 0.56; m.mu = 0.22; m.cmin = 0.0; m.cmax = 0.005; m.midpoint = 6.0;
            m.a_sq = std::pow(m.a, 2); m.b_sq = std::pow(m.b, 2);
            break;
        }
        case MODEL_KURAMOTO: {  // kuramoto.cpp:14-18
            KurK &m = K.kur;
            m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.twopi = 2.0 * M_PI;
            break;
        }
        case MODEL_RWWEX: {  // rwwex.cpp:14-26
            RWWExK &m = K.rwwex;
            m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.J_N = 0.2609; m.a = 270; m.b = 108; m.d = 0.154;
            const double gamma = (double)0.641 / (double)1000.0, tau = 100, itau = 1.0 / tau;
            m.dt_itau = m.dt * itau; m.dt_gamma = m.dt * gamma;
            break;
        }
    }
    return K;
}

// ---------------------------------------------------------------- config
struct Cfg {
    bool verbose = false, do_fc = true, do_fcd = true;
    int bold_remove_s = 30;
    bool exc_inter = true;
    int window_size = 10, window_step = 2;
    bool drop_edges = true, ext_out = true, states_ts = false;
    int noise_time_steps = 30000;
    bool do_fic = true;
    int max_fic_trials = 0;
    int I_start = 1000, I_end = 10000, I_dur = 10000 - 1000 + 1;
    double init_delta = 0.02;
    bool fp32 = false;
    bool philox = false;  // noise segment from Philox on the GPU instead of the host mt19937
    bool autotune = false;  // pick the FP32 integrator by timing short probe runs (model_config "autotune")
    bool fc_tc = false;     // FP32 mode: FC / window FCs on the tensor cores (model_config "fc" = "tc")
    int nodes = 0, n_sims = 0, time_steps = 0, bold_tr = 0, states_sampling = 0, sim_seed = 0;
    double dt = 0.1, bw_dt = 0.001;
    int bold_len = 0, bold_tr_iters = 0, states_len = 0, states_sampling_iters = 0, bw_it = 0, inner_it = 0;
    int n_vols_remove = 0, n_states_samples_remove = 0, corr_len = 0;
    int n_pairs = 0, n_windows = 0, n_window_pairs = 0;
    std::vector<int> w_start, w_end;
    int noise_bw_it = 0, noise_repeats = 0;
    int64_t noise_size = 0;
};

static int to_int(const std::string &k, const std::string &v) {
    try {
        size_t pos = 0;
        int x = std::stoi(v, &pos);
        return x;
    } catch (...) {
        throw Err(CBNM_ERR_CONFIG, "invalid integer for config key '" + k + "': '" + v + "'");
    }
}

static void build_cfg(Cfg &c, const cbnm_run_args *a, const ModelDesc &md) {
    c.nodes = a->nodes; c.n_sims = a->n_sims; c.time_steps = a->time_steps; c.bold_tr = a->bold_tr;
    c.states_sampling = a->states_sampling; c.sim_seed = a->sim_seed; c.dt = a->dt; c.bw_dt = a->bw_dt / 1000.0;
    c.ext_out = a->ext_out != 0; c.states_ts = a->states_ts != 0;
    for (int i = 0; i < a->n_config; ++i) {  // base.hpp:271-297, rww.cpp:54-71
        if (!a->config_keys || !a->config_values || !a->config_keys[i] || !a->config_values[i])
            throw Err(CBNM_ERR_ARG, "null config key or value");
        const std::string k = a->config_keys[i], v = a->config_values[i];
        if (k == "verbose") c.verbose = to_int(k, v) != 0;
        else if (k == "do_fc") c.do_fc = to_int(k, v) != 0;
        else if (k == "do_fcd") c.do_fcd = to_int(k, v) != 0;
        else if (k == "bold_remove_s") c.bold_remove_s = to_int(k, v);
        else if (k == "exc_interhemispheric") c.exc_inter = to_int(k, v) != 0;
        else if (k == "window_size") c.window_size = to_int(k, v);
        else if (k == "window_step") c.window_step = to_int(k, v);
        else if (k == "drop_edges") c.drop_edges = to_int(k, v) != 0;
        else if (k == "noise_time_steps") c.noise_time_steps = to_int(k, v);
        else if (k == "precision") {
            if (v == "fp32") c.fp32 = true;
            else if (v == "fp64") c.fp32 = false;
            else throw Err(CBNM_ERR_CONFIG, "precision must be 'fp64' or 'fp32', got '" + v + "'");
        } else if (k == "autotune") {
            c.autotune = to_int(k, v) != 0;
        } else if (k == "fc") {
            if (v == "tc") c.fc_tc = true;
            else if (v == "fp64") c.fc_tc = false;
            else throw Err(CBNM_ERR_CONFIG, "fc must be 'fp64' or 'tc', got '" + v + "'");
        } else if (k == "noise") {
            if (v == "philox") c.philox = true;
            else if (v == "mt19937") c.philox = false;
            else throw Err(CBNM_ERR_CONFIG, "noise must be 'mt19937' or 'philox', got '" + v + "'");
        }
        if (md.id == MODEL_RWW) {
            if (k == "do_fic") c.do_fic = to_int(k, v) != 0;
            else if (k == "max_fic_trials") c.max_fic_trials = to_int(k, v);
            else if (k == "I_SAMPLING_START") c.I_start = (int)((to_int(k, v) / 1000) / c.bw_dt);
            else if (k == "I_SAMPLING_END") c.I_end = (int)((to_int(k, v) / 1000) / c.bw_dt);
            else if (k == "init_delta") c.init_delta = std::stod(v);
        }
    }
    c.I_dur = c.I_end - c.I_start + 1;
    if (md.id != MODEL_RWW) c.do_fic = false;
    if (c.nodes <= 0 || c.n_sims <= 0) throw Err(CBNM_ERR_ARG, "nodes and N_SIMS must be positive");
    if (c.bold_tr <= 0 || c.states_sampling <= 0 || c.time_steps <= 0 || c.dt <= 0 || c.bw_dt <= 0)
        throw Err(CBNM_ERR_ARG, "time_steps, BOLD_TR, states_sampling, dt and bw_dt must be positive");
    // base.hpp:51-68 (truncating conversions kept)
    c.bold_len = c.time_steps / c.bold_tr;
    c.bold_tr_iters = (int)(((double)c.bold_tr / 1000.0) / c.bw_dt);
    c.states_len = c.time_steps / c.states_sampling;
    c.states_sampling_iters = (int)(((double)c.states_sampling / 1000.0) / c.bw_dt);
    c.bw_it = (int)(((double)c.time_steps / 1000.0) / c.bw_dt);
    c.inner_it = (int)((c.bw_dt * 1000) / c.dt);
    if (c.bold_tr_iters <= 0 || c.states_sampling_iters <= 0 || c.bw_it <= 0 || c.inner_it <= 0)
        throw Err(CBNM_ERR_ARG, "BOLD_TR, states_sampling and duration must be multiples of bw_dt, bw_dt of dt");
    c.n_states_samples_remove = c.bold_remove_s * 1000 / c.states_sampling;
    if (c.do_fc) {  // bnm.cu:1078-1182
        c.n_vols_remove = c.bold_remove_s * 1000 / c.bold_tr;
        c.corr_len = c.bold_len - c.n_vols_remove;
        if (c.corr_len < 2)
            throw Err(CBNM_ERR_CONFIG, "Number of BOLD volumes (after removing " + std::to_string(c.n_vols_remove) +
                                           " initial volumes) is " + std::to_string(c.corr_len) +
                                           " which is too low for FC calculations");
        c.n_pairs = c.nodes * (c.nodes - 1) / 2;
        if (c.exc_inter) {
            if (c.nodes % 2 != 0) throw Err(CBNM_ERR_CONFIG, "exc_interhemispheric is set but number of nodes is not even");
            c.n_pairs -= (c.nodes / 2) * (c.nodes / 2);
        }
        if (c.n_pairs < 1)  // one node, or two with exc_interhemispheric: nothing to correlate
            throw Err(CBNM_ERR_CONFIG, "no node pairs for FC (" + std::to_string(c.nodes) + " nodes" +
                                           (c.exc_inter ? ", exc_interhemispheric)" : ")"));
        if (c.do_fcd) {  // utils.cpp:21-52
            int first = c.drop_edges ? c.window_size / 2 : 0;
            int last = c.drop_edges ? c.corr_len - 1 - c.window_size / 2 : c.corr_len - 1;
            first += c.n_vols_remove;
            last += c.n_vols_remove;
            if (c.window_step <= 0) throw Err(CBNM_ERR_CONFIG, "window_step must be positive");
            for (int ctr = first; ctr <= last; ctr += c.window_step) {
                int s = std::max(0, ctr - c.window_size / 2);
                int e = std::min(c.bold_len - 1, ctr + c.window_size / 2);
                c.w_start.push_back(s);
                c.w_end.push_back(e);
            }
            c.n_windows = (int)c.w_start.size();
            if (c.n_windows == 0) throw Err(CBNM_ERR_CONFIG, "Number of dynamic FC windows is 0");
            c.n_window_pairs = c.n_windows * (c.n_windows - 1) / 2;
        }
    } else {
        c.do_fcd = false;
    }
    c.noise_bw_it = (int)(((double)(c.noise_time_steps) / 1000.0) / c.bw_dt);  // bnm.cu:1229-1231
    if (c.noise_bw_it <= 0) throw Err(CBNM_ERR_CONFIG, "noise_time_steps must cover at least one bw_dt");
    c.noise_repeats = (int)std::ceil((double)(c.bw_it) / (double)(c.noise_bw_it));
    c.noise_size = (int64_t)c.nodes * c.noise_bw_it * c.inner_it * md.n_noise;
}

// ---------------------------------------------------------------- noise
// bnm.cu:1240-1256 + utils.cpp:74-95.  The values come from std::mt19937 and
// libstdc++'s std::normal_distribution<double>; the node and time shuffles are
// restated explicitly: the bounded draw is the division-based rejection method
// and, while n^2 fits in the generator's 32-bit range, two swap positions come
// from one draw in [0, (i+1)(i+2)) (otherwise one draw in [0, i] per element),
// which is what the libstdc++ that produced the reference's stored outputs does.
static uint64_t bounded_draw(std::mt19937 &g, uint64_t range_max) {
    const uint64_t urng_range = 0xffffffffULL;
    const uint64_t span = range_max + 1, scaling = urng_range / span, past = span * scaling;
    uint64_t r;
    do { r = (uint64_t)g(); } while (r >= past);
    return r / scaling;
}
static void shuffle_positions(std::vector<int> &v, std::mt19937 &g) {
    const size_t n = v.size();
    if (n < 2) return;
    if (0xffffffffULL / n < n) {  // n^2 exceeds the generator's range: one draw in [0, i] per element
        for (size_t i = 1; i < n; ++i) std::swap(v[i], v[bounded_draw(g, i)]);
        return;
    }
    size_t i = 1;
    if (n % 2 == 0) { std::swap(v[i], v[bounded_draw(g, 1)]); ++i; }
    while (i != n) {
        const uint64_t b0 = i + 1, b1 = i + 2, x = bounded_draw(g, b0 * b1 - 1);
        std::swap(v[i], v[x / b1]); ++i;
        std::swap(v[i], v[x % b1]); ++i;
    }
}

// ---------------------------------------------------------------- device buffers
struct DBuf {
    void *p = nullptr;
    size_t cap = 0;
    void *ensure(size_t bytes) {
        if (bytes == 0) bytes = 16;
        if (bytes > cap) {
            if (p) CK(cudaFree(p));
            p = nullptr;
            cap = 0;
            CK(cudaMalloc(&p, bytes));
            cap = bytes;
        }
        return p;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() { return static_cast<T *>(p); }
};

struct Session {
    bool ready = false;
    int dev = -1;                // the device the stream, events and buffers belong to
    cudaStream_t st = nullptr;
    cudaEvent_t ev[8];
    // noise cache (bnm.cu:1207-1215 key)
    bool noise_valid = false, noise_f32_valid = false;
    int k_seed = 0, k_time = 0, k_nodes = 0, k_nts = 0, k_nnoise = 0;
    bool k_philox = false;
    size_t noise_n = 0;  // values in the noise segment (on the host too unless Philox)
    double k_bwdt = 0, k_dt = 0;
    std::vector<double> noise;
    std::vector<int> sh_nodes, sh_ts;
    DBuf d_noise, d_noise_f32, d_sh_nodes, d_sh_ts;
    // run buffers
    DBuf d_sc, d_sc_f32, d_sc_idx, d_g, d_r, d_v, d_delay, d_delay_idx, d_max_delay, d_hist_off, d_hist, d_hist_f32;
    DBuf d_bold, d_states, d_gbools, d_gints, d_fc, d_fcd, d_wfc, d_pairs_i, d_pairs_j, d_wstart, d_wend, d_status;
    DBuf d_tiles, d_sct_f32, d_ell_pk, d_bw_scr, d_ln_groups, d_ln_params, d_ln_hist, d_ln_bw;
    DBuf fl_ec, fl_q, fl_win, fl_scr;  // fit loss
    DBuf d_pidx, d_wstat;              // tensor-core FC: pair index of (i, j); window-FC statistics
    // gof
    DBuf g_simfc, g_empfc, g_simfcd, g_empfcd, g_out;
    cbnm_timing timing{};
    ~Session() {}
};
static Session *g_sess = nullptr;
static std::vector<Session *> g_batch;  // one per concurrent worker of cbnm_run_batch
static cbnm_timing g_last_timing{};     // timings of the last run call (single, batch or adjoint)

// A session belongs to the device that was current when it opened: one device
// per process, as the reference's process-global model object.  A call made
// while another device is current fails instead of launching on a foreign
// stream or reusing another device's buffers; cbnm_reset() releases the session
// so that the next call opens one on the new device.
static void open_session(Session &S) {
    int cur = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (S.ready) {
        if (e != cudaSuccess) throw Err(CBNM_ERR_CUDA, std::string("CUDA Error: ") + cudaGetErrorString(e));
        if (cur != S.dev)
            throw Err(CBNM_ERR_CUDA, "CUDA Error: the session was opened on device " + std::to_string(S.dev) +
                                         " but device " + std::to_string(cur) +
                                         " is current; call cbnm_reset() before switching devices");
        return;
    }
    int ndev = 0;
    if (e == cudaSuccess) e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        throw Err(CBNM_ERR_CUDA, std::string("CUDA Error: no CUDA device available (") + cudaGetErrorString(e) + ")");
    S.dev = cur;
    CK(cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking));
    for (auto &ev : S.ev) CK(cudaEventCreate(&ev));
    S.ready = true;
}

static Session &session() {
    if (!g_sess) g_sess = new Session();
    open_session(*g_sess);
    return *g_sess;
}

static void close_session(Session *&p) {
    if (!p) return;
    Session &S = *p;
    if (S.ready) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != S.dev) cudaSetDevice(S.dev);  // free on the device that owns the buffers
        cudaStreamSynchronize(S.st);
        for (DBuf *b : {&S.d_noise, &S.d_noise_f32, &S.d_sh_nodes, &S.d_sh_ts, &S.d_sc, &S.d_sc_f32, &S.d_sc_idx,
                        &S.d_g, &S.d_r, &S.d_v, &S.d_delay, &S.d_delay_idx, &S.d_max_delay, &S.d_hist_off,
                        &S.d_hist, &S.d_hist_f32, &S.d_bold, &S.d_states, &S.d_gbools, &S.d_gints, &S.d_fc,
                        &S.d_fcd, &S.d_wfc, &S.d_pairs_i, &S.d_pairs_j, &S.d_wstart, &S.d_wend, &S.d_status, &S.d_tiles,
                        &S.d_sct_f32, &S.d_ell_pk, &S.d_bw_scr, &S.d_ln_groups, &S.d_ln_params, &S.d_ln_hist, &S.d_ln_bw, &S.fl_ec, &S.fl_q, &S.fl_win, &S.fl_scr, &S.d_pidx, &S.d_wstat,
                        &S.g_simfc, &S.g_empfc, &S.g_simfcd, &S.g_empfcd, &S.g_out})
            b->release();
        for (auto &ev : S.ev) cudaEventDestroy(ev);
        cudaStreamDestroy(S.st);
        if (cur >= 0 && cur != S.dev) cudaSetDevice(cur);
    }
    delete p;
    p = nullptr;
}

static void release_batch_launch();  // below, with the batch machinery

static void release_session() {
    release_batch_launch();
    close_session(g_sess);
    for (Session *&b : g_batch) close_session(b);
    g_batch.clear();
}

static void ensure_noise(Session &S, const Cfg &c, const ModelDesc &md, bool force) {
    const bool same = S.noise_valid && S.k_seed == c.sim_seed && S.k_time == c.time_steps && S.k_nodes == c.nodes &&
                      S.k_nts == c.noise_time_steps && S.k_nnoise == md.n_noise && S.k_bwdt == c.bw_dt &&
                      S.k_dt == c.dt && S.k_philox == c.philox;
    if (!same || force) {
        std::mt19937 gen(c.sim_seed);
        S.noise_n = (size_t)c.noise_size;
        if (c.philox) {  // the segment is drawn on the GPU below; the shuffles from mt19937(seed)
            S.noise.clear();
            S.noise.shrink_to_fit();
        } else {
            std::normal_distribution<double> nd(0, 1);
            S.noise.resize(S.noise_n);
            for (int64_t i = 0; i < c.noise_size; ++i) S.noise[i] = nd(gen);
        }
        std::vector<int> idx(c.nodes);
        S.sh_nodes.resize((size_t)c.noise_repeats * c.nodes);
        std::iota(idx.begin(), idx.end(), 0);
        for (int r = 0; r < c.noise_repeats; ++r) {
            shuffle_positions(idx, gen);
            std::copy(idx.begin(), idx.end(), S.sh_nodes.begin() + (size_t)r * c.nodes);
        }
        std::vector<int> ts(c.noise_bw_it);
        S.sh_ts.resize((size_t)c.noise_repeats * c.noise_bw_it);
        std::iota(ts.begin(), ts.end(), 0);
        for (int r = 0; r < c.noise_repeats; ++r) {
            shuffle_positions(ts, gen);
            std::copy(ts.begin(), ts.end(), S.sh_ts.begin() + (size_t)r * c.noise_bw_it);
        }
        S.d_noise.ensure(sizeof(double) * S.noise_n);
        if (c.philox)
            CK(launch_philox_normals((uint32_t)c.sim_seed, S.d_noise.as<double>(), nullptr, S.noise_n, S.st));
        else
            CK(cudaMemcpyAsync(S.d_noise.p, S.noise.data(), sizeof(double) * S.noise_n, cudaMemcpyHostToDevice, S.st));
        S.d_sh_nodes.ensure(sizeof(int) * S.sh_nodes.size());
        CK(cudaMemcpyAsync(S.d_sh_nodes.p, S.sh_nodes.data(), sizeof(int) * S.sh_nodes.size(), cudaMemcpyHostToDevice, S.st));
        S.d_sh_ts.ensure(sizeof(int) * S.sh_ts.size());
        CK(cudaMemcpyAsync(S.d_sh_ts.p, S.sh_ts.data(), sizeof(int) * S.sh_ts.size(), cudaMemcpyHostToDevice, S.st));
        CK(cudaStreamSynchronize(S.st));
        S.noise_valid = true;
        S.noise_f32_valid = false;
        S.k_seed = c.sim_seed; S.k_time = c.time_steps; S.k_nodes = c.nodes; S.k_nts = c.noise_time_steps;
        S.k_nnoise = md.n_noise; S.k_bwdt = c.bw_dt; S.k_dt = c.dt; S.k_philox = c.philox;
    }
    if (c.fp32 && !S.noise_f32_valid && c.philox) {  // regenerate, writing both copies
        S.d_noise_f32.ensure(sizeof(float) * S.noise_n);
        CK(launch_philox_normals((uint32_t)c.sim_seed, S.d_noise.as<double>(), S.d_noise_f32.as<float>(), S.noise_n,
                                 S.st));
        CK(cudaStreamSynchronize(S.st));
        S.noise_f32_valid = true;
    }
    if (c.fp32 && !S.noise_f32_valid) {
        std::vector<float> f(S.noise.begin(), S.noise.end());
        S.d_noise_f32.ensure(sizeof(float) * f.size());
        CK(cudaMemcpyAsync(S.d_noise_f32.p, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice, S.st));
        CK(cudaStreamSynchronize(S.st));
        S.noise_f32_valid = true;
    }
}

// ---------------------------------------------------------------- helpers
static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void check_args(const cbnm_run_args *a) {
    if (!a) throw Err(CBNM_ERR_ARG, "null arguments");
    if (!a->sc || !a->sc_indices || !a->sc_dist || !a->global_params || !a->regional_params || !a->v_list)
        throw Err(CBNM_ERR_ARG, "null input array");
    if (a->n_scs <= 0) throw Err(CBNM_ERR_ARG, "n_scs must be positive");
}

static void fill_sizes(const Cfg &c, const ModelDesc &md, cbnm_sizes *sz) {
    std::memset(sz, 0, sizeof(*sz));
    sz->n_global_params = md.n_global; sz->n_regional_params = md.n_regional; sz->n_state_vars = md.n_state;
    sz->n_global_out_bool = md.n_gout_bool; sz->n_global_out_int = md.n_gout_int;
    sz->bold_len = c.bold_len; sz->n_pairs = c.n_pairs; sz->n_windows = c.n_windows;
    sz->n_window_pairs = c.n_window_pairs; sz->states_len = c.states_len; sz->do_fc = c.do_fc; sz->do_fcd = c.do_fcd;
    sz->modifies_params = md.modifies_params && c.do_fic;
    sz->noise_repeats = c.noise_repeats; sz->noise_bw_it = c.noise_bw_it; sz->noise_size = c.noise_size;
}

// ---------------------------------------------------------------- run
// sp: the session to run on; null = the process's default session, opened once
// the arguments have been validated (so argument errors come before device errors)
// Touches one byte per 4 KB page of a host output buffer so that its pages are
// mapped (and zeroed by the OS) now, while the GPU is still computing, rather
// than inside the device-to-host copy into it.  The copy overwrites every byte.
static void prefault_host(void *p, size_t bytes) {
    volatile unsigned char *c = static_cast<volatile unsigned char *>(p);
    for (size_t i = 0; i < bytes; i += 4096) c[i] = 0;
}

static int sm_count() {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

// Work items of the two-tile kernel from 32-simulation tiles ([n][33]: SC index,
// simulation ids): items [m][65] = SC index, half 0, half 1 (-1 = empty).  Tiles
// of one SC are paired; an odd tile of an SC runs as a single.  The items are
// spread over `sms` CTAs in rounds (item w runs in round w / grid); while a round
// would be partly empty, pairs are split into singles (one half idle, a shorter
// step) until every round is full or no pair is left, singles last.
static std::vector<int> pair_tiles(const std::vector<int> &tiles, int n_tiles, int sms, int *n_items, int *grid) {
    constexpr int W = 33;
    std::vector<std::array<int, 2>> pairs, singles;
    for (int t = 0; t < n_tiles;) {
        if (t + 1 < n_tiles && tiles[(size_t)t * W] == tiles[(size_t)(t + 1) * W]) {
            pairs.push_back({t, t + 1});
            t += 2;
        } else {
            singles.push_back({t, -1});
            t += 1;
        }
    }
    auto count = [&] { return (int)(pairs.size() + singles.size()); };
    const int g = std::max(1, sms);
    while (!pairs.empty() && (count() < g || count() % g != 0)) {  // every CTA busy in every round
        const auto pq = pairs.back();
        pairs.pop_back();
        singles.insert(singles.begin(), {{pq[0], -1}, {pq[1], -1}});
    }
    std::vector<int> out;
    out.reserve((size_t)count() * 65);
    for (const auto *v : {&pairs, &singles})
        for (const auto &pq : *v) {
            out.push_back(tiles[(size_t)pq[0] * W]);
            for (int h = 0; h < 2; ++h)
                for (int i = 0; i < 32; ++i) out.push_back(pq[h] >= 0 ? tiles[(size_t)pq[h] * W + 1 + i] : -1);
        }
    *n_items = count();
    *grid = std::max(1, std::min(sms, count()));
    return out;
}

// ---------------------------------------------------------------- one launch for a batch's lane groups
// cbnm_run_batch runs up to 16 groups at a time ("a round"), each in a worker
// thread with its own session.  Groups that take the lane kernel (FP32, delays or
// > 128 nodes) do not launch it themselves: each prepares its inputs, lays out
// its parameters on its own stream and joins the round; when every group of the
// round has joined or declined (taken another integrator, or failed), the last
// one launches a single persistent work-queue kernel over all joined groups'
// 16-simulation items, longest first, and the joined groups then continue with
// their FC / FCD and copies once that kernel is done.
struct BatchRound {
    std::mutex mu;
    std::condition_variable cv;
    int expected = 0, resolved = 0;
    bool launched = false;
    std::string err;
    struct Join {
        IntegrateArgs ia;
        int model;
        cudaEvent_t ready;
    };
    std::vector<Join> joins;
};
struct BatchLaunch {  // state shared by the rounds of one cbnm_run_batch call (they run in order)
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr, t0 = nullptr, t1 = nullptr;
    DBuf runs, items, counter, hist, bw;
    std::vector<std::vector<IntegrateArgs>> host_runs;   // kept alive for the asynchronous copies
    std::vector<std::vector<int2>> host_items;
    float kernel_ms = 0.0f;
    int launches = 0;
};
static thread_local BatchRound *t_round = nullptr;
static thread_local bool t_round_resolved = false;
static BatchLaunch *g_batch_launch = nullptr;

// Launches the round's combined kernel(s), one per model (called with the round's lock held).
static void round_launch(BatchRound &R) {
    BatchLaunch &B = *g_batch_launch;
    try {
        std::map<int, std::vector<int>> by_model;
        for (int i = 0; i < (int)R.joins.size(); ++i) by_model[R.joins[i].model].push_back(i);
        for (const auto &kv : by_model) {
            std::vector<IntegrateArgs> runs;
            std::vector<std::pair<double, int2>> work;
            long long hist_per = 0, bw_per = 0;
            int mn = 1;
            for (int i : kv.second) {
                const IntegrateArgs &ia = R.joins[i].ia;
                CK(cudaStreamWaitEvent(B.st, R.joins[i].ready, 0));
                const int r = (int)runs.size();
                runs.push_back(ia);
                const double cost = (double)ia.nodes * std::max(1, ia.ell_k) * ia.bw_it * ia.inner_it;
                for (int gi = 0; gi < ia.ln_n_groups; ++gi) work.push_back({cost, make_int2(r, gi)});
                hist_per = std::max(hist_per, ia.ln_hist_per_cta);
                bw_per = std::max(bw_per, (long long)ia.nodes * 4 * 16);
                mn = std::max(mn, lanes_rows(ia.nodes, 1024));
            }
            std::stable_sort(work.begin(), work.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
            std::vector<int2> items;
            for (const auto &w : work) items.push_back(w.second);
            const int grid = std::min((int)items.size(), sm_count());
            B.host_runs.push_back(std::move(runs));
            B.host_items.push_back(std::move(items));
            const auto &hr = B.host_runs.back();
            const auto &hi = B.host_items.back();
            CK(cudaStreamSynchronize(B.st));  // the scratch of the previous launch is free
            IntegrateArgs *d_runs = (IntegrateArgs *)B.runs.ensure(sizeof(IntegrateArgs) * hr.size());
            int2 *d_items = (int2 *)B.items.ensure(sizeof(int2) * hi.size());
            int *d_counter = (int *)B.counter.ensure(sizeof(int));
            float *d_hist = (float *)B.hist.ensure(sizeof(float) * (size_t)grid * hist_per);
            double *d_bw = (double *)B.bw.ensure(sizeof(double) * (size_t)grid * bw_per);
            CK(cudaMemcpyAsync(d_runs, hr.data(), sizeof(IntegrateArgs) * hr.size(), cudaMemcpyHostToDevice, B.st));
            CK(cudaMemcpyAsync(d_items, hi.data(), sizeof(int2) * hi.size(), cudaMemcpyHostToDevice, B.st));
            CK(cudaMemsetAsync(d_counter, 0, sizeof(int), B.st));
            CK(cudaEventRecord(B.t0, B.st));
            CK(launch_integrate_lanes_multi(kv.first, d_runs, d_items, (int)hi.size(), d_counter, mn, grid, d_hist,
                                            hist_per, d_bw, bw_per, B.st));
            CK(cudaEventRecord(B.t1, B.st));
            CK(cudaEventSynchronize(B.t1));
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, B.t0, B.t1));
            B.kernel_ms += ms;
            ++B.launches;
        }
        CK(cudaEventRecord(B.done, B.st));
    } catch (const Err &e) {
        R.err = e.what();
    }
    R.launched = true;
    R.cv.notify_all();
}

static void release_batch_launch() {
    if (!g_batch_launch) return;
    BatchLaunch &B = *g_batch_launch;
    cudaStreamSynchronize(B.st);
    for (DBuf *b : {&B.runs, &B.items, &B.counter, &B.hist, &B.bw}) b->release();
    cudaEventDestroy(B.done);
    cudaEventDestroy(B.t0);
    cudaEventDestroy(B.t1);
    cudaStreamDestroy(B.st);
    delete g_batch_launch;
    g_batch_launch = nullptr;
}

// A group of the round takes part in the combined launch; returns once it is enqueued.
static void round_join(BatchRound &R, const IntegrateArgs &ia, int model, cudaEvent_t ready) {
    std::unique_lock<std::mutex> lk(R.mu);
    R.joins.push_back({ia, model, ready});
    if (++R.resolved == R.expected) round_launch(R);
    else R.cv.wait(lk, [&] { return R.launched; });
    if (!R.err.empty()) throw Err(CBNM_ERR_CUDA, R.err);
}

// A group of the round that does not take part (another integrator, or an error).
static void round_decline(BatchRound &R) {
    std::unique_lock<std::mutex> lk(R.mu);
    if (++R.resolved == R.expected) round_launch(R);
}

// ---------------------------------------------------------------- FP32 integrator variants
// The FP32 path has several integrators for the same arithmetic; which is fastest
// depends on the node count, the delays and the SC's sparsity.  The default
// choice follows fixed rules (run_impl); with model_config "autotune" = "1" (or
// CBNM_AUTOTUNE=1) the first run of each workload key times a short probe of
// every applicable variant on a slice of the batch and keeps the fastest for the
// process (and in CBNM_TUNE_FILE when set, one "key variant" line each).
enum Variant { V_DEFAULT = 0, V_PP, V_V5, V_LANES, V_LANES512, V_SIMT, V_PPWS, V_COUNT };
static const char *const kVariantName[V_COUNT] = {"default", "tc2", "tc1", "lanes", "lanes512", "simt", "tc2ws"};
static thread_local int t_force_variant = V_DEFAULT;  // set while a probe runs
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tuned;
static bool g_tune_loaded = false;
static Session *g_tune = nullptr;                     // probes run on a session of their own
static thread_local std::string t_last_variant = "";

static int variant_of(const std::string &name) {
    for (int v = 0; v < V_COUNT; ++v)
        if (name == kVariantName[v]) return v;
    return -1;
}

static void tune_load() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = std::getenv("CBNM_TUNE_FILE");
    if (!path) return;
    FILE *f = std::fopen(path, "r");
    if (!f) return;
    char key[512], name[64];
    while (std::fscanf(f, "%511s %63s", key, name) == 2) {
        const int v = variant_of(name);
        if (v > 0) g_tuned[key] = v;
    }
    std::fclose(f);
}

static void tune_store(const std::string &key, int v) {
    g_tuned[key] = v;
    const char *path = std::getenv("CBNM_TUNE_FILE");
    if (!path) return;
    if (FILE *f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %s\n", key.c_str(), kVariantName[v]);
        std::fclose(f);
    }
}

static void run_impl(Session *sp, const cbnm_run_args *a, cbnm_outputs *o, bool device_io, double *tan_bold = nullptr);

// Times one variant on `probe` (host buffers); returns milliseconds of the integrator or -1.
static double probe_variant(const cbnm_run_args &probe, int v) {
    const int P = probe.n_sims;
    cbnm_sizes z;
    {
        Cfg c;
        build_cfg(c, &probe, *find_model(probe.model_name));
        fill_sizes(c, *find_model(probe.model_name), &z);
    }
    std::vector<double> bold((size_t)P * z.bold_len * probe.nodes);
    std::vector<unsigned char> gb((size_t)std::max(1, z.n_global_out_bool) * P);
    std::vector<int> gi((size_t)std::max(1, z.n_global_out_int) * P);
    cbnm_outputs out{};
    out.sim_bold = bold.data();
    out.global_bools = gb.data();
    out.global_ints = gi.data();
    if (!g_tune) g_tune = new Session();
    open_session(*g_tune);
    t_force_variant = v;
    double best = -1.0;
    try {
        for (int rep = 0; rep < 2; ++rep) {  // the first run loads modules and draws the probe's noise
            run_impl(g_tune, &probe, &out, false);
            best = g_tune->timing.integrate_ms;
        }
    } catch (const Err &) {
        best = -1.0;  // not applicable to this workload
    }
    t_force_variant = V_DEFAULT;
    return best;
}

// The tuned variant for this run (probing on first sight of its key).
static int tuned_variant(const cbnm_run_args *a, const Cfg &c, const std::string &key, const std::vector<int> &cands) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_load();
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return it->second;
    // probe: the first <= 2368 simulations (16 per SM-resident group x 148), <= 1 s, no FC / FCD / states
    const int P = std::min(c.n_sims, 2368);
    const int md_g = find_model(a->model_name)->n_global, md_r = find_model(a->model_name)->n_regional;
    std::vector<double> g((size_t)md_g * P), r((size_t)md_r * P * c.nodes), v(a->v_list, a->v_list + P);
    for (int q = 0; q < md_g; ++q)
        std::copy(a->global_params + (size_t)q * c.n_sims, a->global_params + (size_t)q * c.n_sims + P, g.begin() + (size_t)q * P);
    for (int q = 0; q < md_r; ++q)
        std::copy(a->regional_params + (size_t)q * c.n_sims * c.nodes,
                  a->regional_params + (size_t)q * c.n_sims * c.nodes + (size_t)P * c.nodes,
                  r.begin() + (size_t)q * P * c.nodes);
    std::vector<std::string> keys, vals;
    for (int i = 0; i < a->n_config; ++i) {
        const std::string k = a->config_keys[i];
        if (k == "do_fc" || k == "do_fcd" || k == "autotune") continue;
        keys.push_back(k);
        vals.push_back(a->config_values[i]);
    }
    keys.push_back("do_fc"); vals.push_back("0");
    keys.push_back("do_fcd"); vals.push_back("0");
    std::vector<const char *> kp, vp;
    for (size_t i = 0; i < keys.size(); ++i) { kp.push_back(keys[i].c_str()); vp.push_back(vals[i].c_str()); }
    cbnm_run_args probe = *a;
    probe.n_sims = P;
    probe.global_params = g.data();
    probe.regional_params = r.data();
    probe.v_list = v.data();
    probe.config_keys = kp.data();
    probe.config_values = vp.data();
    probe.n_config = (int)kp.size();
    probe.ext_out = 0;
    probe.states_ts = 0;
    probe.noise_out = 0;
    probe.force_reinit = 0;
    const int tr = std::max(1, a->bold_tr);
    probe.time_steps = std::min(a->time_steps, std::max(tr, (1000 / tr) * tr));
    int best_v = V_DEFAULT;
    double best_ms = 0.0;
    for (int cand : cands) {
        const double ms = probe_variant(probe, cand);
        if (ms > 0.0 && (best_v == V_DEFAULT || ms < best_ms)) { best_v = cand; best_ms = ms; }
    }
    if (best_v != V_DEFAULT) tune_store(key, best_v);
    return best_v;
}

// tan_bold (device, [N][bold_len][nodes]) non-null: also integrate the tangent along
// G and write dBOLD/dG there (lane kernel, FP32 precision, rWW or WC).
static void run_impl(Session *sp, const cbnm_run_args *a, cbnm_outputs *o, bool device_io, double *tan_bold) {
    const double t_begin = now_s();
    check_args(a);
    if (!o || !o->sim_bold) throw Err(CBNM_ERR_ARG, "null output arrays");
    const ModelDesc *mdp = find_model(a->model_name);
    if (!mdp) throw Err(CBNM_ERR_MODEL, std::string("Model ") + (a->model_name ? a->model_name : "(null)") + " not found");
    const ModelDesc &md = *mdp;
    if (a->use_cpu)
        throw Err(CBNM_ERR_UNSUPPORTED, "use_cpu is not supported: this library runs the simulations on the GPU only");
    Cfg c;
    build_cfg(c, a, md);
    if (c.nodes > 1024) throw Err(CBNM_ERR_UNSUPPORTED, "more than 1024 nodes is not supported by this library");
    if (c.do_fc && !o->sim_fc_trils) throw Err(CBNM_ERR_ARG, "do_fc is set but sim_fc_trils is null");
    if (c.do_fcd && !o->sim_fcd_trils) throw Err(CBNM_ERR_ARG, "do_fcd is set but sim_fcd_trils is null");
    if (c.ext_out && !o->sim_states) throw Err(CBNM_ERR_ARG, "ext_out is set but sim_states is null");
    if (a->noise_out && (!o->noise || !o->shuffled_nodes || !o->shuffled_ts))
        throw Err(CBNM_ERR_ARG, "noise_out is set but noise outputs are null");
    for (int s = 0; s < c.n_sims && !device_io; ++s)
        if (a->sc_indices[s] < 0 || a->sc_indices[s] >= a->n_scs) throw Err(CBNM_ERR_ARG, "SC index out of range");

    Session &S = sp ? *sp : session();
    cbnm_timing tm{};
    const int N = c.n_sims, n = c.nodes;
    const size_t nn = (size_t)n * n, gsize = (size_t)md.n_global * N, rsize = (size_t)md.n_regional * N * n;

    // ---- init phase: noise (session cache), as init_gpu
    const double t_init0 = now_s();
    ensure_noise(S, c, md, a->force_reinit != 0);
    const double init_time = now_s() - t_init0;

    // ---- inputs
    CK(cudaEventRecord(S.ev[0], S.st));
    const double *d_sc = nullptr;
    const int *d_sc_idx = nullptr;
    const double *d_g = nullptr;
    double *d_r = nullptr;
    std::vector<double> h_g, h_r;
    std::vector<uint8_t> h_gbools((size_t)md.n_gout_bool * N, 0);
    std::vector<int32_t> h_sc_idx;
    const double *h_sc = a->sc;
    if (device_io) {
        d_sc = a->sc; d_sc_idx = a->sc_indices; d_g = a->global_params; d_r = a->regional_params;
        if (c.do_fic || c.fp32) {  // host copies needed for FIC / SC conversion
            h_g.resize(gsize); h_r.resize(rsize);
            CK(cudaMemcpyAsync(h_g.data(), a->global_params, sizeof(double) * gsize, cudaMemcpyDeviceToHost, S.st));
            CK(cudaMemcpyAsync(h_r.data(), a->regional_params, sizeof(double) * rsize, cudaMemcpyDeviceToHost, S.st));
            h_sc_idx.resize(N);
            CK(cudaMemcpyAsync(h_sc_idx.data(), a->sc_indices, sizeof(int) * N, cudaMemcpyDeviceToHost, S.st));
            CK(cudaStreamSynchronize(S.st));
        }
    } else {
        S.d_sc.ensure(sizeof(double) * nn * a->n_scs);
        CK(cudaMemcpyAsync(S.d_sc.p, a->sc, sizeof(double) * nn * a->n_scs, cudaMemcpyHostToDevice, S.st));
        S.d_sc_idx.ensure(sizeof(int) * N);
        CK(cudaMemcpyAsync(S.d_sc_idx.p, a->sc_indices, sizeof(int) * N, cudaMemcpyHostToDevice, S.st));
        d_sc = S.d_sc.as<double>(); d_sc_idx = S.d_sc_idx.as<int>();
        tm.h2d_bytes += sizeof(double) * nn * a->n_scs + sizeof(int) * N;
        h_g.assign(a->global_params, a->global_params + gsize);
        h_r.assign(a->regional_params, a->regional_params + rsize);
    }
    if (!device_io) {
        S.d_g.ensure(sizeof(double) * gsize);
        S.d_r.ensure(sizeof(double) * rsize);
        CK(cudaMemcpyAsync(S.d_g.p, h_g.data(), sizeof(double) * gsize, cudaMemcpyHostToDevice, S.st));
        CK(cudaMemcpyAsync(S.d_r.p, h_r.data(), sizeof(double) * rsize, cudaMemcpyHostToDevice, S.st));
        d_g = S.d_g.as<double>(); d_r = S.d_r.as<double>();
        tm.h2d_bytes += sizeof(double) * (gsize + rsize);
    }

    // ---- delays (bnm.cpp:146-202: per-pair steps from the lower triangle, diagonal 1)
    std::vector<double> h_v;
    int has_delay = 0;
    std::vector<int> h_delay, h_delay_idx(N, 0), h_max_delay(N, 0);
    std::vector<long long> h_hist_off(N, 0);
    long long hist_total = 0;
    if (a->do_delay) {
        h_v.resize(N);
        std::vector<double> h_dist(nn);
        if (device_io) {
            CK(cudaMemcpy(h_v.data(), a->v_list, sizeof(double) * N, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(h_dist.data(), a->sc_dist, sizeof(double) * nn, cudaMemcpyDeviceToHost));
        } else {
            h_v.assign(a->v_list, a->v_list + N);
            h_dist.assign(a->sc_dist, a->sc_dist + nn);
        }
        std::map<double, int> table_of;
        std::vector<int> table_max;
        for (int s = 0; s < N; ++s) {
            const double vel = h_v[s] * c.dt;
            auto it = table_of.find(vel);
            if (it == table_of.end()) {
                const int t = (int)table_max.size();
                table_of[vel] = t;
                h_delay.resize((size_t)(t + 1) * nn, 0);
                int *dl = h_delay.data() + (size_t)t * nn;
                int mx = 0;
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j <= i; ++j) {
                        if (i > j) {
                            int dd = (int)rintf(h_dist[(size_t)i * n + j] / vel);
                            dd = std::max(dd, 1);
                            dl[(size_t)i * n + j] = dd;
                            dl[(size_t)j * n + i] = dd;
                            mx = std::max(mx, dd);
                        } else {
                            dl[(size_t)i * n + j] = 1;
                        }
                    }
                table_max.push_back(mx);
                it = table_of.find(vel);
            }
            h_delay_idx[s] = it->second;
            h_max_delay[s] = table_max[it->second];
        }
        for (int s = 0; s < N; ++s) {
            h_hist_off[s] = hist_total;
            hist_total += (long long)h_max_delay[s] * n;
        }
        has_delay = *std::max_element(h_max_delay.begin(), h_max_delay.end()) > 0;
    }
    // FP32 kernels: the tensor-core tiles take shared-SC batches without delays or
    // numerical FIC at <= 128 nodes.  Delayed networks of more than 512 nodes, with
    // at least half as many 16-simulation groups as SMs, take the lane kernel
    // (1,000-node WC, 2,048 sims: 440 vs 343 sims x sim-s / s); everything else runs
    // on the per-simulation kernel, which measured faster there (400-node rWW with
    // delays: 1,103 vs 435; 200-node rWW without, 512 sims: 11,645 vs 1,593).  The
    // lane kernel also runs the G tangent, and when CBNM_FP32_KERNEL=lanes or the
    // tuner picks it; CBNM_FP32_KERNEL=simt forces the per-simulation kernel.
    const char *fp32_kernel = std::getenv("CBNM_FP32_KERNEL");
    const bool force_simt = fp32_kernel && std::string(fp32_kernel) == "simt";
    const bool force_lanes = fp32_kernel && std::string(fp32_kernel) == "lanes";
    const bool num_fic = c.do_fic && c.max_fic_trials > 0;
    if (tan_bold && (!c.fp32 || !lanes_tangent_supported(md.id) || num_fic || !lanes_supported(md.id, n, num_fic)))
        throw Err(CBNM_ERR_UNSUPPORTED, "the G tangent needs precision fp32, model rWW or WC, at most 1024 nodes and "
                                        "no numerical FIC");
    const bool tc_ok = c.fp32 && fp32_supported(md.id, n, has_delay) && !num_fic;
    const bool lanes_ok = c.fp32 && lanes_supported(md.id, n, num_fic) &&
                          (has_delay ? *std::max_element(h_max_delay.begin(), h_max_delay.end()) + 1 : 2) * (long long)n <
                              (1LL << 30);
    int variant = t_force_variant;
    if (variant == V_DEFAULT && !tan_bold && c.fp32 && !force_simt && !device_io &&
        (c.autotune || (std::getenv("CBNM_AUTOTUNE") && std::string(std::getenv("CBNM_AUTOTUNE")) == "1"))) {
        std::vector<int> cands;
        if (tc_ok && pp_supported(md.id, n, has_delay)) {
            cands.push_back(V_PP);
            cands.push_back(V_PPWS);
        }
        if (tc_ok) cands.push_back(V_V5);
        if (lanes_ok) cands.push_back(V_LANES);
        if (lanes_ok && n <= 128) cands.push_back(V_LANES512);
        cands.push_back(V_SIMT);
        const int Dmax = has_delay ? *std::max_element(h_max_delay.begin(), h_max_delay.end()) : 0;
        const std::string key = std::string(md.name) + "|n" + std::to_string(n) + "|D" + std::to_string(Dmax) +
                                "|scs" + std::to_string(a->n_scs) + "|nfic" + std::to_string((int)num_fic);
        variant = tuned_variant(a, c, key, cands);
    }
    if (variant != V_DEFAULT) {  // a forced or tuned variant must apply to this run
        const bool ok = c.fp32 && !tan_bold &&
                        (((variant == V_PP || variant == V_PPWS) && tc_ok && pp_supported(md.id, n, has_delay)) ||
                         (variant == V_V5 && tc_ok) ||
                         (variant == V_LANES && lanes_ok) || (variant == V_LANES512 && lanes_ok && n <= 128) ||
                         variant == V_SIMT);
        if (!ok) throw Err(CBNM_ERR_UNSUPPORTED, std::string("integrator variant ") + kVariantName[variant] +
                                                     " does not apply to this run");
    }
    const bool use_tc = variant == V_DEFAULT ? (!tan_bold && !force_simt && tc_ok)
                                             : (variant == V_PP || variant == V_PPWS || variant == V_V5);
    const bool lanes_default = has_delay && n > 512 && 2 * ((N + 15) / 16) >= sm_count() && !force_simt;
    bool use_lanes = variant == V_DEFAULT ? (lanes_ok && (tan_bold || ((force_lanes || lanes_default) && !use_tc)))
                                          : (variant == V_LANES || variant == V_LANES512);
    const int lanes_threads = variant == V_LANES512 ? 512 : 1024;
    if (t_round && !t_round_resolved && !(use_lanes && lanes_threads == 1024 && !tan_bold && g_batch_launch)) {
        t_round_resolved = true;  // this group runs its own integrator: the round need not wait for it
        round_decline(*t_round);
    }
    if (has_delay) {
        S.d_delay.ensure(sizeof(int) * h_delay.size());
        CK(cudaMemcpyAsync(S.d_delay.p, h_delay.data(), sizeof(int) * h_delay.size(), cudaMemcpyHostToDevice, S.st));
        S.d_delay_idx.ensure(sizeof(int) * N);
        CK(cudaMemcpyAsync(S.d_delay_idx.p, h_delay_idx.data(), sizeof(int) * N, cudaMemcpyHostToDevice, S.st));
        S.d_max_delay.ensure(sizeof(int) * N);
        CK(cudaMemcpyAsync(S.d_max_delay.p, h_max_delay.data(), sizeof(int) * N, cudaMemcpyHostToDevice, S.st));
        S.d_hist_off.ensure(sizeof(long long) * N);
        CK(cudaMemcpyAsync(S.d_hist_off.p, h_hist_off.data(), sizeof(long long) * N, cudaMemcpyHostToDevice, S.st));
        // FP32 mode keeps FP32 ring buffers, except for the Kuramoto phase (double)
        if (c.fp32 && !md.osc) {
            if (!use_lanes) S.d_hist_f32.ensure(sizeof(float) * hist_total);
        } else {
            S.d_hist.ensure(sizeof(double) * hist_total);
        }
    }

    // ---- outputs on the device
    const size_t bold_n = (size_t)N * c.bold_len * n;
    const size_t ext = c.states_ts ? (size_t)n * c.states_len : (size_t)n;
    const size_t states_n = c.ext_out ? (size_t)md.n_state * N * ext : 0;
    double *d_bold = device_io ? o->sim_bold : (double *)S.d_bold.ensure(sizeof(double) * bold_n);
    double *d_states = device_io ? o->sim_states : (double *)S.d_states.ensure(sizeof(double) * std::max<size_t>(states_n, 1));
    uint8_t *d_gbools = (uint8_t *)S.d_gbools.ensure(std::max<size_t>(1, (size_t)md.n_gout_bool * N));
    int *d_gints = (int *)S.d_gints.ensure(sizeof(int) * std::max<size_t>(1, (size_t)md.n_gout_int * N));
    if (md.n_gout_bool)
        CK(cudaMemcpyAsync(d_gbools, h_gbools.data(), h_gbools.size(), cudaMemcpyHostToDevice, S.st));
    if (md.n_gout_int) CK(cudaMemsetAsync(d_gints, 0, sizeof(int) * md.n_gout_int * N, S.st));
    int *d_status = (int *)S.d_status.ensure(sizeof(int));
    CK(cudaMemsetAsync(d_status, 0, sizeof(int), S.st));
    CK(cudaEventRecord(S.ev[1], S.st));

    // ---- analytical FIC on the GPU (rww.cpp:73-146): wIE into the regional
    // parameters in place, failure flags into global_bools[0]
    if (c.do_fic) {
        FicArgs fa;
        fa.nodes = n; fa.n_sims = N; fa.sc = d_sc; fa.sc_idx = d_sc_idx; fa.gparams = d_g; fa.regional = d_r;
        fa.unstable = d_gbools; fa.K = make_constants(MODEL_RWW, c.dt).rww;
        CK(launch_rww_fic(fa, S.st));
    }

    // ---- integrate
    IntegrateArgs ia;
    std::memset(&ia, 0, sizeof(ia));
    ia.nodes = n; ia.n_sims = N; ia.bw_it = c.bw_it; ia.inner_it = c.inner_it; ia.bold_tr_iters = c.bold_tr_iters;
    ia.states_sampling_iters = c.states_sampling_iters; ia.n_states_samples_remove = c.n_states_samples_remove;
    ia.noise_bw_it = c.noise_bw_it; ia.bold_len = c.bold_len; ia.states_len = c.states_len;
    ia.ext_out = c.ext_out; ia.states_ts = c.states_ts;
    ia.sc = d_sc; ia.sc_idx = d_sc_idx; ia.gparams = d_g; ia.rparams = d_r; ia.rparams_out = d_r;
    ia.noise = S.d_noise.as<double>(); ia.noise_f32 = S.d_noise_f32.as<float>();
    ia.sh_nodes = S.d_sh_nodes.as<int>(); ia.sh_ts = S.d_sh_ts.as<int>();
    ia.has_delay = has_delay;
    ia.delay = S.d_delay.as<int>(); ia.delay_idx = S.d_delay_idx.as<int>(); ia.max_delay = S.d_max_delay.as<int>();
    ia.hist_off = S.d_hist_off.as<long long>(); ia.hist = S.d_hist.as<double>(); ia.hist_f32 = S.d_hist_f32.as<float>();
    ia.bold = d_bold; ia.states = d_states; ia.gbools = d_gbools; ia.gints = d_gints;
    ia.do_fic = c.do_fic; ia.max_fic_trials = c.max_fic_trials; ia.I_start = c.I_start; ia.I_end = c.I_end;
    ia.I_dur = c.I_dur; ia.init_delta = c.init_delta;
    ia.bw = g_bw; ia.bw.dt = c.bw_dt; ia.bw.dt_itau = ia.bw.dt * ia.bw.itau;  // core.cpp:291-292
    {  // C(1/alpha, k) for the FP32 kernel's binomial form of nu^(1/alpha)
        long double v = 1.0L;
        ia.bw_binom[0] = 1.0;
        for (int k = 1; k <= 12; ++k) {
            v = v * ((long double)ia.bw.ialpha - (k - 1)) / k;
            ia.bw_binom[k] = (double)v;
        }
    }
    ia.K = make_constants(md.id, c.dt);
    {  // the two-tile kernel reads these from its parameter space
        BWFast &f = ia.bwf;
        f.dt = ia.bw.dt; f.kappa = ia.bw.kappa; f.y = ia.bw.y; f.dt_itau = ia.bw.dt_itau; f.ialpha = ia.bw.ialpha;
        f.irho = 1.0 / ia.bw.rho; f.log2_omr = std::log2(ia.bw.oneminrho); f.ln_omr = std::log(ia.bw.oneminrho);
        f.omr = ia.bw.oneminrho;
        f.V0k1 = ia.bw.V_0 * ia.bw.k1; f.V0k2 = ia.bw.V_0 * ia.bw.k2; f.V0k3 = ia.bw.V_0 * ia.bw.k3;
        std::copy(ia.bw_binom, ia.bw_binom + 13, f.binom);
        if (md.id == MODEL_RWW) {
            const RWW32::K k = RWW32::make(ia.K);
            static_assert(sizeof(k) <= sizeof(ia.k32), "FP32 constants");
            std::memcpy(ia.k32, &k, sizeof(k));
        }
    }
    ia.sim_begin = 0;
    ia.n_regional = md.n_regional;
    ia.status = d_status;
    int launches = 0;
    if (c.fp32) {  // FP32 SC copy (converted once per run)
        std::vector<float> f;
        std::vector<double> tmp;
        const double *src = h_sc;
        if (device_io) {
            tmp.resize(nn * a->n_scs);
            CK(cudaMemcpy(tmp.data(), a->sc, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost));
            src = tmp.data();
        }
        f.assign(src, src + nn * a->n_scs);
        S.d_sc_f32.ensure(sizeof(float) * f.size());
        CK(cudaMemcpyAsync(S.d_sc_f32.p, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice, S.st));
        ia.sc_f32 = S.d_sc_f32.as<float>();
    }
    if (!use_tc) {
        // Sparse coupling for the per-simulation kernels (ELLPACK by target node):
        // used when the densest column of every SC holds at most half the nodes
        // (CBNM_COUPLING=sparse|dense overrides).  Zero weights are skipped and the
        // nonzeros summed in ascending source order, so FP64 sums are unchanged.
        // The packed ring-buffer offsets are 32-bit: every simulation's buffer must
        // hold fewer than 2^30 values, else the dense loop runs.
        std::vector<double> sc_host;
        const double *src = h_sc;
        if (device_io) {
            sc_host.resize(nn * a->n_scs);
            CK(cudaMemcpy(sc_host.data(), a->sc, sizeof(double) * sc_host.size(), cudaMemcpyDeviceToHost));
            src = sc_host.data();
        }
        int kmax = 0;
        for (int sc = 0; sc < a->n_scs; ++sc)
            for (int j = 0; j < n; ++j) {
                int cnt = 0;
                for (int k = 0; k < n; ++k) cnt += src[(size_t)sc * nn + (size_t)k * n + j] != 0.0;
                kmax = std::max(kmax, cnt);
            }
        const char *cpl = std::getenv("CBNM_COUPLING");
        const std::string mode = cpl ? cpl : "";
        const long long max_hist = has_delay ? (long long)*std::max_element(h_max_delay.begin(), h_max_delay.end()) * n : 0;
        const bool fits = max_hist < (1LL << 30);
        const bool sparse =
            fits && (use_lanes || mode == "sparse" || (mode != "dense" && n >= 32 && 2 * kmax <= n));
        if (!fits) use_lanes = false;
        if (sparse) {
            const int K = std::max(kmax, 1);
            const int tabs = has_delay ? (int)(h_delay.size() / nn) : 1;
            const size_t per_tab = (size_t)K * n;
            const size_t total = per_tab * tabs * a->n_scs;
            std::vector<int2> pk32(c.fp32 ? total : 0);
            std::vector<int4> pk64(c.fp32 ? 0 : total);
            // padding: source j (delay 1 with delays), weight 0
            auto put = [&](size_t e, int off, double v) {
                if (c.fp32) {
                    const float f = (float)v;
                    int bits;
                    std::memcpy(&bits, &f, sizeof(bits));
                    pk32[e] = make_int2(off, bits);
                } else {
                    uint64_t u;
                    std::memcpy(&u, &v, sizeof(u));
                    pk64[e] = make_int4((int)(uint32_t)u, (int)(uint32_t)(u >> 32), off, 0);
                }
            };
            for (int sc = 0; sc < a->n_scs; ++sc)
                for (int t = 0; t < tabs; ++t) {
                    const int *dl = has_delay ? h_delay.data() + (size_t)t * nn : nullptr;
                    const size_t base = ((size_t)sc * tabs + t) * per_tab;
                    for (int j = 0; j < n; ++j) {
                        int q = 0;
                        for (int k = 0; k < n; ++k) {
                            const double v = src[(size_t)sc * nn + (size_t)k * n + j];
                            if (v == 0.0) continue;
                            const int d = dl ? dl[(size_t)k * n + j] : 0;
                            put(base + (size_t)q * n + j, d * n + k, v);
                            ++q;
                        }
                        for (; q < K; ++q) put(base + (size_t)q * n + j, (dl ? n : 0) + j, 0.0);
                    }
                }
            const size_t bytes = c.fp32 ? sizeof(int2) * total : sizeof(int4) * total;
            S.d_ell_pk.ensure(bytes);
            CK(cudaMemcpyAsync(S.d_ell_pk.p, c.fp32 ? (const void *)pk32.data() : (const void *)pk64.data(), bytes,
                               cudaMemcpyHostToDevice, S.st));
            if (c.fp32) ia.ell_pk32 = S.d_ell_pk.as<int2>();
            else ia.ell_pk64 = S.d_ell_pk.as<int4>();
            ia.ell_k = K;
            ia.ell_tables = tabs;
            CK(cudaStreamSynchronize(S.st));  // host vectors go out of scope
        }
    }
    // rWW on the tensor cores: the single-tile kernel (measured faster on the
    // 100-node workload: 210k vs 195k sims x sim-s / s) unless CBNM_FP32_TC=pp or ws
    // selects the two-tile one (or the tuner picks it)
    const char *tc_kind = std::getenv("CBNM_FP32_TC");
    const bool pp_env = tc_kind && (std::string(tc_kind) == "pp" || std::string(tc_kind) == "ws");
    const bool use_pp = use_tc && pp_supported(md.id, n, has_delay) &&
                        (variant == V_DEFAULT ? pp_env : (variant == V_PP || variant == V_PPWS));
    // the warp-specialised two-tile form: CBNM_FP32_TC=ws, or the tuned variant
    const bool pp_ws = use_pp && (variant == V_DEFAULT ? (tc_kind && std::string(tc_kind) == "ws") : variant == V_PPWS);
    if (use_tc) {
        // tiles of simulations that share one SC
        const int TN = use_pp ? 32 : fp32_tile_for(n);
        ia.tile_width = TN;
        std::vector<int> sc_of(N);
        if (device_io) {
            if (h_sc_idx.size() != (size_t)N) {
                h_sc_idx.resize(N);
                CK(cudaMemcpy(h_sc_idx.data(), a->sc_indices, sizeof(int) * N, cudaMemcpyDeviceToHost));
            }
            sc_of.assign(h_sc_idx.begin(), h_sc_idx.end());
        } else {
            sc_of.assign(a->sc_indices, a->sc_indices + N);
        }
        std::vector<int> order(N);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sc_of[x] < sc_of[y]; });
        std::vector<int> tiles;
        for (size_t i = 0; i < order.size();) {
            const int sc = sc_of[order[i]];
            tiles.push_back(sc);
            int cnt = 0;
            while (cnt < TN && i < order.size() && sc_of[order[i]] == sc) { tiles.push_back(order[i]); ++i; ++cnt; }
            for (; cnt < TN; ++cnt) tiles.push_back(-1);
        }
        ia.n_tiles = (int)(tiles.size() / (TN + 1));
        if (use_pp) tiles = pair_tiles(tiles, ia.n_tiles, sm_count(), &ia.n_tiles, &ia.pp_grid);
        ia.pp_ws = pp_ws ? 1 : 0;
        S.d_tiles.ensure(sizeof(int) * tiles.size());
        CK(cudaMemcpyAsync(S.d_tiles.p, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, S.st));
        ia.tiles = S.d_tiles.as<int>();
        if (use_pp) ia.bw_scratch = (double *)S.d_bw_scr.ensure(pp_bw_scratch_bytes(n, ia.pp_grid));
        CK(cudaStreamSynchronize(S.st));
        CK(cudaEventRecord(S.ev[1], S.st));
        if (use_pp) CK(launch_integrate_pp(md.id, ia, S.st, &launches));
        else CK(launch_integrate_fp32(md.id, ia, S.st, &launches));
    } else if (use_lanes) {
        // groups of 16 simulations sharing SC and delay table (bnm.cu runs one
        // CTA per simulation; here one CTA integrates a group)
        std::vector<int> sc_of(N);
        if (device_io) {
            if (h_sc_idx.size() != (size_t)N) {
                h_sc_idx.resize(N);
                CK(cudaMemcpy(h_sc_idx.data(), a->sc_indices, sizeof(int) * N, cudaMemcpyDeviceToHost));
            }
            sc_of.assign(h_sc_idx.begin(), h_sc_idx.end());
        } else {
            sc_of.assign(a->sc_indices, a->sc_indices + N);
        }
        std::vector<int> order(N);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return std::make_pair(sc_of[x], h_delay_idx[x]) < std::make_pair(sc_of[y], h_delay_idx[y]);
        });
        constexpr int G = 16;
        std::vector<int> groups;
        int max_slots = 2;
        for (size_t i = 0; i < order.size();) {
            const int sc = sc_of[order[i]], tab = h_delay_idx[order[i]];
            const int D = has_delay ? std::max(1, h_max_delay[order[i]]) : 1;
            max_slots = std::max(max_slots, D + 1);
            groups.push_back(sc);
            groups.push_back(has_delay ? tab : 0);
            groups.push_back(D);
            int cnt = 0;
            while (cnt < G && i < order.size() && sc_of[order[i]] == sc && h_delay_idx[order[i]] == tab) {
                groups.push_back(order[i]);
                ++i;
                ++cnt;
            }
            for (; cnt < G; ++cnt) groups.push_back(-1);
        }
        ia.ln_n_groups = (int)(groups.size() / (3 + G));
        ia.ln_threads = lanes_threads;
        ia.ln_grid = std::min(ia.ln_n_groups, sm_count() * (1024 / lanes_threads));
        S.d_ln_groups.ensure(sizeof(int) * groups.size());
        CK(cudaMemcpyAsync(S.d_ln_groups.p, groups.data(), sizeof(int) * groups.size(), cudaMemcpyHostToDevice, S.st));
        ia.ln_groups = S.d_ln_groups.as<int>();
        ia.ln_params = (float *)S.d_ln_params.ensure(sizeof(float) * (size_t)ia.ln_n_groups * n * md.n_regional * G);
        ia.ln_hist_per_cta = (long long)max_slots * n * G * (tan_bold ? 2 : 1);  // (x, dx/dG) pairs with the tangent
        ia.tan_bold = tan_bold;
        const bool join = t_round && !t_round_resolved && !tan_bold && lanes_threads == 1024 && g_batch_launch;
        if (join) {  // one launch for the lane groups of the batch round
            CK(cudaStreamSynchronize(S.st));
            CK(cudaEventRecord(S.ev[1], S.st));
            CK(launch_integrate_lanes_params(md.id, ia, S.st));
            CK(cudaEventRecord(S.ev[5], S.st));
            t_round_resolved = true;
            round_join(*t_round, ia, md.id, S.ev[5]);
            CK(cudaStreamWaitEvent(S.st, g_batch_launch->done, 0));
            launches += 1;  // parameter layout; the combined integrator launch is counted by the batch
        } else {
            ia.ln_hist = (float *)S.d_ln_hist.ensure(sizeof(float) * (size_t)ia.ln_grid * ia.ln_hist_per_cta);
            ia.ln_bw = (double *)S.d_ln_bw.ensure(sizeof(double) * (size_t)ia.ln_grid * n * (tan_bold ? 8 : 4) * G);
            CK(cudaStreamSynchronize(S.st));
            CK(cudaEventRecord(S.ev[1], S.st));
            CK(launch_integrate_lanes(md.id, ia, S.st));
            launches += 2;  // parameter layout + integrator
        }
    } else if (c.fp32) {
        CK(cudaStreamSynchronize(S.st));
        CK(cudaEventRecord(S.ev[1], S.st));
        CK(launch_integrate_simt32(md.id, ia, S.st));
        ++launches;
    } else {
        CK(launch_integrate_fp64(md.id, ia, S.st));
        ++launches;
    }
    t_last_variant = !c.fp32 ? "fp64" : use_pp ? (pp_ws ? "tc2ws" : "tc2") : use_tc ? "tc1" : use_lanes ? (lanes_threads == 512 ? "lanes512" : "lanes") : "simt";
    CK(cudaEventRecord(S.ev[2], S.st));
    if (!device_io) {  // the integrator runs asynchronously: map the host output pages meanwhile
        prefault_host(o->sim_bold, sizeof(double) * bold_n);
        if (c.do_fc) prefault_host(o->sim_fc_trils, sizeof(double) * (size_t)N * c.n_pairs);
        if (c.do_fc && c.do_fcd) prefault_host(o->sim_fcd_trils, sizeof(double) * (size_t)N * c.n_window_pairs);
        if (c.ext_out) prefault_host(o->sim_states, sizeof(double) * states_n);
    }

    // ---- FC / FCD (bnm.cu:809-942), in chunks that bound the window-FC scratch
    double *d_fc = nullptr, *d_fcd = nullptr;
    if (c.do_fc) {
        d_fc = device_io ? o->sim_fc_trils : (double *)S.d_fc.ensure(sizeof(double) * (size_t)N * c.n_pairs);
        if (c.do_fcd) d_fcd = device_io ? o->sim_fcd_trils : (double *)S.d_fcd.ensure(sizeof(double) * std::max<size_t>(1, (size_t)N * c.n_window_pairs));
        std::vector<int> pi, pj;
        const int rh = n / 2;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < i; ++j) {
                if (c.exc_inter && ((i < rh) ^ (j < rh))) continue;
                pi.push_back(i);
                pj.push_back(j);
            }
        S.d_pairs_i.ensure(sizeof(int) * pi.size());
        S.d_pairs_j.ensure(sizeof(int) * pj.size());
        CK(cudaMemcpyAsync(S.d_pairs_i.p, pi.data(), sizeof(int) * pi.size(), cudaMemcpyHostToDevice, S.st));
        CK(cudaMemcpyAsync(S.d_pairs_j.p, pj.data(), sizeof(int) * pj.size(), cudaMemcpyHostToDevice, S.st));
        int max_T = c.corr_len;
        if (c.do_fcd) {
            S.d_wstart.ensure(sizeof(int) * c.n_windows);
            S.d_wend.ensure(sizeof(int) * c.n_windows);
            CK(cudaMemcpyAsync(S.d_wstart.p, c.w_start.data(), sizeof(int) * c.n_windows, cudaMemcpyHostToDevice, S.st));
            CK(cudaMemcpyAsync(S.d_wend.p, c.w_end.data(), sizeof(int) * c.n_windows, cudaMemcpyHostToDevice, S.st));
            for (int w = 0; w < c.n_windows; ++w) max_T = std::max(max_T, c.w_end[w] - c.w_start[w] + 1);
        }
        const size_t per_sim = sizeof(double) * (size_t)std::max(1, c.n_windows) * c.n_pairs;
        const size_t budget = (size_t)1 << 30;
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>(N, budget / per_sim));
        if (c.do_fcd) S.d_wfc.ensure(per_sim * chunk);
        FcArgs fa;
        std::memset(&fa, 0, sizeof(fa));
        fa.nodes = n; fa.bold_len = c.bold_len; fa.n_vols_remove = c.n_vols_remove; fa.n_pairs = c.n_pairs;
        fa.n_windows = c.do_fcd ? c.n_windows : 0; fa.n_window_pairs = c.n_window_pairs; fa.max_T = max_T;
        fa.w_start = S.d_wstart.as<int>(); fa.w_end = S.d_wend.as<int>();
        fa.pair_i = S.d_pairs_i.as<int>(); fa.pair_j = S.d_pairs_j.as<int>();
        fa.bold = d_bold; fa.fc = d_fc; fa.fcd = d_fcd; fa.wfc = S.d_wfc.as<double>();
        fa.status_fc = d_status;
        // tensor-core FC in FP32 mode when asked for (model_config "fc" = "tc" or CBNM_FC=tc)
        const char *fce = std::getenv("CBNM_FC");
        const bool fc_tc = c.fp32 && (c.fc_tc || (fce && std::string(fce) == "tc"));
        if (fc_tc) {
            if (c.do_fcd) fa.wstat = (double *)S.d_wstat.ensure(sizeof(double) * 2 * (size_t)chunk * std::max(1, c.n_windows));
            std::vector<int> pidx(nn, -1);
            for (size_t q = 0; q < pi.size(); ++q) pidx[(size_t)pi[q] * n + pj[q]] = (int)q;
            S.d_pidx.ensure(sizeof(int) * nn);
            CK(cudaMemcpyAsync(S.d_pidx.p, pidx.data(), sizeof(int) * nn, cudaMemcpyHostToDevice, S.st));
            CK(cudaStreamSynchronize(S.st));
        }
        for (int s0 = 0; s0 < N; s0 += chunk) {
            fa.sim_begin = s0;
            fa.sim_count = std::min(chunk, N - s0);
            if (fc_tc) CK(launch_fc_tc(fa, S.d_pidx.as<int>(), S.st, &launches));
            else CK(launch_fc(fa, S.st, &launches));
        }
    }
    CK(cudaEventRecord(S.ev[3], S.st));

    // ---- outputs back to the host (bnm.cu:951-971) and parameter write-back
    if (!device_io) {
        CK(cudaMemcpyAsync(o->sim_bold, d_bold, sizeof(double) * bold_n, cudaMemcpyDeviceToHost, S.st));
        tm.d2h_bytes += sizeof(double) * bold_n;
        if (c.do_fc) {
            CK(cudaMemcpyAsync(o->sim_fc_trils, d_fc, sizeof(double) * (size_t)N * c.n_pairs, cudaMemcpyDeviceToHost, S.st));
            tm.d2h_bytes += sizeof(double) * (size_t)N * c.n_pairs;
            if (c.do_fcd) {
                CK(cudaMemcpyAsync(o->sim_fcd_trils, d_fcd, sizeof(double) * (size_t)N * c.n_window_pairs, cudaMemcpyDeviceToHost, S.st));
                tm.d2h_bytes += sizeof(double) * (size_t)N * c.n_window_pairs;
            }
        }
        if (c.ext_out) {
            CK(cudaMemcpyAsync(o->sim_states, d_states, sizeof(double) * states_n, cudaMemcpyDeviceToHost, S.st));
            tm.d2h_bytes += sizeof(double) * states_n;
        }
        if (md.modifies_params && c.do_fic) {  // core.cpp:437-450
            CK(cudaMemcpyAsync(a->regional_params, d_r, sizeof(double) * rsize, cudaMemcpyDeviceToHost, S.st));
            tm.d2h_bytes += sizeof(double) * rsize;
        }
    }
    if (md.n_gout_bool && o->global_bools) {
        CK(cudaMemcpyAsync(o->global_bools, d_gbools, (size_t)md.n_gout_bool * N,
                           device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, S.st));
    }
    if (md.n_gout_int && o->global_ints) {
        CK(cudaMemcpyAsync(o->global_ints, d_gints, sizeof(int) * md.n_gout_int * N,
                           device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, S.st));
    }
    int h_status = 0;
    CK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, S.st));
    CK(cudaEventRecord(S.ev[4], S.st));
    CK(cudaStreamSynchronize(S.st));
    if (h_status != 0)
        throw Err(CBNM_ERR_TIMEOUT, "a device-side wait in the integrator gave up (status " + std::to_string(h_status) + ")");
    if (c.do_fic) {  // report every simulation whose analytical FIC failed, as prep_params does (rww.cpp:73-146)
        std::vector<uint8_t> flags(N);
        CK(cudaMemcpy(flags.data(), d_gbools, N, cudaMemcpyDeviceToHost));
        for (int s2 = 0; s2 < N; ++s2)
            if (flags[s2]) std::fprintf(stderr, "In simulation #%d analytical FIC failed. Setting wIE to 1 in all nodes\n", s2);
    }
    if (a->noise_out) {  // core.cpp:429-435
        if (device_io) {
            CK(cudaMemcpy(o->noise, S.d_noise.p, sizeof(double) * S.noise_n, cudaMemcpyDeviceToDevice));
            CK(cudaMemcpy(o->shuffled_nodes, S.d_sh_nodes.p, sizeof(int) * S.sh_nodes.size(), cudaMemcpyDeviceToDevice));
            CK(cudaMemcpy(o->shuffled_ts, S.d_sh_ts.p, sizeof(int) * S.sh_ts.size(), cudaMemcpyDeviceToDevice));
        } else {
            if (S.noise.size() == S.noise_n) std::memcpy(o->noise, S.noise.data(), sizeof(double) * S.noise_n);
            else CK(cudaMemcpy(o->noise, S.d_noise.p, sizeof(double) * S.noise_n, cudaMemcpyDeviceToHost));
            std::memcpy(o->shuffled_nodes, S.sh_nodes.data(), sizeof(int) * S.sh_nodes.size());
            std::memcpy(o->shuffled_ts, S.sh_ts.data(), sizeof(int) * S.sh_ts.size());
        }
    }
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, S.ev[0], S.ev[1])); tm.h2d_ms = ms;
    CK(cudaEventElapsedTime(&ms, S.ev[1], S.ev[2])); tm.integrate_ms = ms;
    CK(cudaEventElapsedTime(&ms, S.ev[2], S.ev[3])); tm.fc_ms = ms;
    CK(cudaEventElapsedTime(&ms, S.ev[3], S.ev[4])); tm.d2h_ms = ms;
    CK(cudaEventElapsedTime(&ms, S.ev[0], S.ev[4])); tm.total_ms = ms;
    tm.kernel_launches = launches;
    S.timing = tm;
    g_last_timing = tm;
    o->init_time = init_time;
    o->run_time = now_s() - t_begin - init_time;
}

// ---------------------------------------------------------------- GOF
// ---------------------------------------------------------------- adjoint (gradients)
// Reverse-mode gradient of an FP32 rWW batch (adjoint.cu).  Inputs are device
// arrays, as cbnm_run_simulations_device; noise and shuffles come from the
// session cache exactly as for a run with the same seed, nodes and duration.
struct AdjPlan {
    Cfg c;
    const ModelDesc *md = nullptr;
    int seg_bw = 0, n_seg = 0, chunk = 0;
    size_t ck_s_bytes = 0, ck_bytes = 0, scr_bw_bytes = 0, scr_s_bytes = 0, scr_z_bytes = 0, scratch_bytes = 0;
};

static AdjPlan adjoint_plan(const cbnm_run_args *a, int segment_steps) {
    check_args(a);
    AdjPlan P;
    P.md = find_model(a->model_name);
    if (!P.md) throw Err(CBNM_ERR_MODEL, std::string("Model ") + (a->model_name ? a->model_name : "(null)") + " not found");
    if (P.md->id != MODEL_RWW) throw Err(CBNM_ERR_UNSUPPORTED, "gradients are implemented for the rWW model only");
    if (a->do_delay) throw Err(CBNM_ERR_UNSUPPORTED, "gradients with conduction delays are not implemented");
    if (a->use_cpu) throw Err(CBNM_ERR_UNSUPPORTED, "use_cpu is not supported");
    build_cfg(P.c, a, *P.md);
    P.c.fp32 = true;
    if (P.c.do_fic) throw Err(CBNM_ERR_UNSUPPORTED, "gradients need do_fic = 0 (wIE given)");
    if (P.c.nodes > 1024) throw Err(CBNM_ERR_UNSUPPORTED, "more than 1024 nodes is not supported by this library");
    if (segment_steps <= 0 || segment_steps % P.c.inner_it != 0)
        throw Err(CBNM_ERR_ARG, "segment_steps must be a positive multiple of bw_dt / dt = " + std::to_string(P.c.inner_it));
    const int N = P.c.n_sims, n = P.c.nodes;
    P.seg_bw = segment_steps / P.c.inner_it;
    P.n_seg = (P.c.bw_it + P.seg_bw - 1) / P.seg_bw;
    P.ck_s_bytes = sizeof(float) * (size_t)N * P.n_seg * 2 * n;
    P.ck_bytes = P.ck_s_bytes + sizeof(double) * (size_t)N * P.n_seg * 4 * n;
    const size_t bw_per = sizeof(double) * (size_t)P.seg_bw * 4 * n;
    const size_t s_per = sizeof(float) * (size_t)P.seg_bw * P.c.inner_it * 3 * n;
    const size_t z_per = sizeof(float) * (size_t)P.seg_bw * n;
    const size_t per_sim = bw_per + s_per + z_per;
    const size_t budget = (size_t)2 << 30;
    P.chunk = (int)std::max<size_t>(1, std::min<size_t>(N, budget / per_sim));
    P.scr_bw_bytes = bw_per * P.chunk;
    P.scr_s_bytes = s_per * P.chunk;
    P.scr_z_bytes = z_per * P.chunk;
    P.scratch_bytes = P.scr_bw_bytes + P.scr_s_bytes + P.scr_z_bytes;
    return P;
}

static AdjArgs adjoint_args(Session &S, AdjPlan &P, const cbnm_run_args *a) {
    const Cfg &c = P.c;
    ensure_noise(S, c, *P.md, a->force_reinit != 0);
    const size_t nn = (size_t)c.nodes * c.nodes;
    S.d_sc_f32.ensure(sizeof(float) * nn * a->n_scs);
    S.d_sct_f32.ensure(sizeof(float) * nn * a->n_scs);
    CK(launch_transpose_sc(a->sc, S.d_sc_f32.as<float>(), S.d_sct_f32.as<float>(), a->n_scs, c.nodes, S.st));
    AdjArgs A;
    std::memset(&A, 0, sizeof(A));
    IntegrateArgs &ia = A.ia;
    ia.nodes = c.nodes; ia.n_sims = c.n_sims; ia.bw_it = c.bw_it; ia.inner_it = c.inner_it;
    ia.bold_tr_iters = c.bold_tr_iters; ia.noise_bw_it = c.noise_bw_it; ia.bold_len = c.bold_len;
    ia.sc_f32 = S.d_sc_f32.as<float>(); ia.sc_idx = a->sc_indices;
    ia.gparams = a->global_params; ia.rparams = a->regional_params;
    ia.noise_f32 = S.d_noise_f32.as<float>(); ia.sh_nodes = S.d_sh_nodes.as<int>(); ia.sh_ts = S.d_sh_ts.as<int>();
    ia.bw = g_bw; ia.bw.dt = c.bw_dt; ia.bw.dt_itau = ia.bw.dt * ia.bw.itau;  // core.cpp:291-292
    ia.K = make_constants(MODEL_RWW, c.dt);
    A.sct_f32 = S.d_sct_f32.as<float>();
    A.seg_bw = P.seg_bw; A.n_seg = P.n_seg;
    return A;
}

static void adjoint_forward_impl(const cbnm_run_args *a, int segment_steps, double *bold, void *ckpt) {
    if (!bold || !ckpt) throw Err(CBNM_ERR_ARG, "null bold or checkpoint buffer");
    AdjPlan P = adjoint_plan(a, segment_steps);
    Session &S = session();
    AdjArgs A = adjoint_args(S, P, a);
    A.ia.bold = bold;
    A.ck_s = static_cast<float *>(ckpt);
    A.ck_bw = reinterpret_cast<double *>(static_cast<char *>(ckpt) + P.ck_s_bytes);
    A.sim_begin = 0; A.sim_count = P.c.n_sims;
    cbnm_timing tm{};
    CK(cudaEventRecord(S.ev[0], S.st));
    CK(launch_adjoint_forward(A, S.st));
    CK(cudaEventRecord(S.ev[1], S.st));
    CK(cudaEventSynchronize(S.ev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, S.ev[0], S.ev[1]));
    tm.integrate_ms = ms; tm.total_ms = ms; tm.kernel_launches = 2;
    S.timing = tm;
    g_last_timing = tm;
}

static void adjoint_backward_impl(const cbnm_run_args *a, int segment_steps, const double *dbold, const void *ckpt,
                                  void *scratch, double *grad_global, double *grad_regional) {
    if (!dbold || !ckpt || !scratch || !grad_global || !grad_regional) throw Err(CBNM_ERR_ARG, "null buffer");
    AdjPlan P = adjoint_plan(a, segment_steps);
    Session &S = session();
    AdjArgs A = adjoint_args(S, P, a);
    A.ck_s = const_cast<float *>(static_cast<const float *>(ckpt));
    A.ck_bw = reinterpret_cast<double *>(const_cast<char *>(static_cast<const char *>(ckpt)) + P.ck_s_bytes);
    A.dbold = dbold;
    A.scr_bw = static_cast<double *>(scratch);
    A.scr_s = reinterpret_cast<float *>(static_cast<char *>(scratch) + P.scr_bw_bytes);
    A.scr_z = reinterpret_cast<float *>(static_cast<char *>(scratch) + P.scr_bw_bytes + P.scr_s_bytes);
    A.grad_g = grad_global; A.grad_r = grad_regional;
    cbnm_timing tm{};
    int launches = 1;
    CK(cudaEventRecord(S.ev[0], S.st));
    for (int s0 = 0; s0 < P.c.n_sims; s0 += P.chunk) {
        A.sim_begin = s0;
        A.sim_count = std::min(P.chunk, P.c.n_sims - s0);
        CK(launch_adjoint_backward(A, S.st));
        ++launches;
    }
    CK(cudaEventRecord(S.ev[1], S.st));
    CK(cudaEventSynchronize(S.ev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, S.ev[0], S.ev[1]));
    tm.integrate_ms = ms; tm.total_ms = ms; tm.kernel_launches = launches;
    S.timing = tm;
    g_last_timing = tm;
}

static void gof_impl(const double *sim_fc, int n_sims, int n_pairs, const double *emp_fc, const double *sim_fcd,
                     int n_wp, const double *emp_fcd, int n_emp_fcd, double *fc_corr, double *fc_diff,
                     double *fc_normec, double *fcd_ks) {
    if (n_sims <= 0) return;
    const bool want_fc = sim_fc && emp_fc && n_pairs > 0 && (fc_corr || fc_diff || fc_normec);
    const bool want_ks = sim_fcd && emp_fcd && n_wp > 0 && n_emp_fcd > 0 && fcd_ks;
    if (want_ks) {
        size_t m1p = 1;  // the KS kernel sorts one simulation's FCD, padded to a power of two, in shared memory
        while (m1p < (size_t)n_wp) m1p <<= 1;
        if (sizeof(double) * m1p > gof_ks_smem_limit()) {
            size_t max_pairs = 1;
            while (sizeof(double) * (max_pairs << 1) <= gof_ks_smem_limit()) max_pairs <<= 1;
            throw Err(CBNM_ERR_UNSUPPORTED, "FCD too long for the KS kernel: " + std::to_string(n_wp) +
                                                " window pairs per simulation (at most " + std::to_string(max_pairs) + ")");
        }
    }
    Session &S = session();
    GofArgs g;
    std::memset(&g, 0, sizeof(g));
    g.n_sims = n_sims; g.n_pairs = n_pairs; g.n_wp = n_wp; g.n_emp_fcd = n_emp_fcd;
    double *d_out = (double *)S.g_out.ensure(sizeof(double) * 4 * n_sims);
    if (want_fc) {
        double m = 0;
        for (int p = 0; p < n_pairs; ++p) m += emp_fc[p];
        m /= n_pairs;
        double q = 0;
        for (int p = 0; p < n_pairs; ++p) q += (emp_fc[p] - m) * (emp_fc[p] - m);
        g.emp_fc_mean = m; g.emp_fc_ssd = std::sqrt(q);
        S.g_simfc.ensure(sizeof(double) * (size_t)n_sims * n_pairs);
        S.g_empfc.ensure(sizeof(double) * n_pairs);
        CK(cudaMemcpyAsync(S.g_simfc.p, sim_fc, sizeof(double) * (size_t)n_sims * n_pairs, cudaMemcpyHostToDevice, S.st));
        CK(cudaMemcpyAsync(S.g_empfc.p, emp_fc, sizeof(double) * n_pairs, cudaMemcpyHostToDevice, S.st));
        g.sim_fc = S.g_simfc.as<double>(); g.emp_fc = S.g_empfc.as<double>();
        if (fc_corr) g.fc_corr = d_out;
        if (fc_diff) g.fc_diff = d_out + n_sims;
        if (fc_normec) g.fc_normec = d_out + 2 * n_sims;
    }
    std::vector<double> emp_sorted;
    if (want_ks) {
        emp_sorted.assign(emp_fcd, emp_fcd + n_emp_fcd);
        std::sort(emp_sorted.begin(), emp_sorted.end());
        S.g_simfcd.ensure(sizeof(double) * (size_t)n_sims * n_wp);
        S.g_empfcd.ensure(sizeof(double) * n_emp_fcd);
        CK(cudaMemcpyAsync(S.g_simfcd.p, sim_fcd, sizeof(double) * (size_t)n_sims * n_wp, cudaMemcpyHostToDevice, S.st));
        CK(cudaMemcpyAsync(S.g_empfcd.p, emp_sorted.data(), sizeof(double) * n_emp_fcd, cudaMemcpyHostToDevice, S.st));
        g.sim_fcd = S.g_simfcd.as<double>(); g.emp_fcd_sorted = S.g_empfcd.as<double>();
        g.fcd_ks = d_out + 3 * n_sims;
    }
    int launches = 0;
    CK(launch_gof(g, S.st, &launches));
    std::vector<double> h((size_t)4 * n_sims);
    CK(cudaMemcpyAsync(h.data(), d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, S.st));
    CK(cudaStreamSynchronize(S.st));
    if (want_fc && fc_corr) std::memcpy(fc_corr, h.data(), sizeof(double) * n_sims);
    if (want_fc && fc_diff) std::memcpy(fc_diff, h.data() + n_sims, sizeof(double) * n_sims);
    if (want_fc && fc_normec) std::memcpy(fc_normec, h.data() + 2 * n_sims, sizeof(double) * n_sims);
    if (want_ks) {
        std::memcpy(fcd_ks, h.data() + 3 * n_sims, sizeof(double) * n_sims);
        for (int s = 0; s < n_sims; ++s)  // a NaN in a row makes the statistic NaN
            for (int p = 0; p < n_wp; ++p)
                if (std::isnan(sim_fcd[(size_t)s * n_wp + p])) { fcd_ks[s] = NAN; break; }
    }
}

}  // namespace cbnm

// ---------------------------------------------------------------- C ABI
using namespace cbnm;

template <class F>
static int guarded(F f) {
    try {
        f();
        g_err.clear();
        return CBNM_OK;
    } catch (const Err &e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_err = e.what();
        return CBNM_ERR_CONFIG;
    }
}

extern "C" {

int cbnm_init(void) {
    g_bw = bw_defaults(0.001);
    return CBNM_OK;
}

int cbnm_set_const(const char *key, double value) {
    if (!key) { g_err = "null key"; return CBNM_ERR_ARG; }
    const std::string k = key;
    if (k == "k1") g_bw.k1 = value;
    else if (k == "k2") g_bw.k2 = value;
    else if (k == "k3") g_bw.k3 = value;
    else if (k == "V_0") g_bw.V_0 = value;
    g_bw.V_0_k1 = g_bw.V_0 * g_bw.k1;
    g_bw.V_0_k2 = g_bw.V_0 * g_bw.k2;
    g_bw.V_0_k3 = g_bw.V_0 * g_bw.k3;
    return CBNM_OK;
}

int cbnm_query_sizes(const cbnm_run_args *a, cbnm_sizes *sz) {
    return guarded([&] {
        if (!a || !sz) throw Err(CBNM_ERR_ARG, "null argument");
        const ModelDesc *md = find_model(a->model_name);
        if (!md) throw Err(CBNM_ERR_MODEL, std::string("Model ") + (a->model_name ? a->model_name : "(null)") + " not found");
        Cfg c;
        build_cfg(c, a, *md);
        fill_sizes(c, *md, sz);
    });
}

int cbnm_run_simulations(const cbnm_run_args *a, cbnm_outputs *o) {
    return guarded([&] { run_impl(nullptr, a, o, false); });
}

int cbnm_run_simulations_device(const cbnm_run_args *a, cbnm_outputs *o) {
    return guarded([&] { run_impl(nullptr, a, o, true); });
}

int cbnm_run_tangent_device(const cbnm_run_args *a, cbnm_outputs *o, double *dbold_dG) {
    return guarded([&] {
        if (!dbold_dG) throw Err(CBNM_ERR_ARG, "null dBOLD/dG output");
        run_impl(nullptr, a, o, true, dbold_dG);
    });
}

// Groups run concurrently, each worker on its own session (stream, buffers, noise
// cache): up to 16 host threads, worker w taking groups w, w + K, w + 2K, .. so a
// repeated batch finds each group's noise cached in the same session.
int cbnm_run_batch(const cbnm_run_args *args, cbnm_outputs *outs, int n_groups, int *statuses) {
    return guarded([&] {
        if (!args || !outs || n_groups < 1) throw Err(CBNM_ERR_ARG, "null batch or no groups");
        const int K = std::min(n_groups, 16);
        int dev = 0;
        CK(cudaGetDevice(&dev));
        while ((int)g_batch.size() < K) g_batch.push_back(new Session());
        for (int w = 0; w < K; ++w) open_session(*g_batch[w]);
        std::vector<int> codes(n_groups, CBNM_OK);
        std::vector<std::string> errs(n_groups);
        std::atomic<int> launches{0};
        std::atomic<long long> h2d{0}, d2h{0};
        // the lane groups of each round of K groups share one launch (CBNM_BATCH_LAUNCH=streams:
        // every group launches its own kernel on its own stream)
        const char *bl = std::getenv("CBNM_BATCH_LAUNCH");
        const bool combined = !(bl && std::string(bl) == "streams");
        const int n_rounds = (n_groups + K - 1) / K;
        std::vector<BatchRound> rounds(n_rounds);
        for (int r = 0; r < n_rounds; ++r) rounds[r].expected = std::min(K, n_groups - r * K);
        if (combined) {
            if (!g_batch_launch) {
                g_batch_launch = new BatchLaunch();
                CK(cudaStreamCreateWithFlags(&g_batch_launch->st, cudaStreamNonBlocking));
                CK(cudaEventCreateWithFlags(&g_batch_launch->done, cudaEventDisableTiming));
                CK(cudaEventCreate(&g_batch_launch->t0));
                CK(cudaEventCreate(&g_batch_launch->t1));
            }
            g_batch_launch->kernel_ms = 0.0f;
            g_batch_launch->launches = 0;
            g_batch_launch->host_runs.clear();
            g_batch_launch->host_items.clear();
        }
        const double t0 = now_s();
        auto worker = [&](int w) {
            const cudaError_t e = cudaSetDevice(dev);
            for (int g = w; g < n_groups; g += K) {
                t_round = combined ? &rounds[g / K] : nullptr;
                t_round_resolved = false;
                if (e != cudaSuccess) {
                    codes[g] = CBNM_ERR_CUDA;
                    errs[g] = std::string("CUDA Error: ") + cudaGetErrorString(e);
                    if (t_round) round_decline(*t_round);
                    continue;
                }
                try {
                    run_impl(g_batch[w], &args[g], &outs[g], false);
                    const cbnm_timing &t = g_batch[w]->timing;
                    launches += t.kernel_launches;
                    h2d += t.h2d_bytes;
                    d2h += t.d2h_bytes;
                } catch (const Err &x) {
                    codes[g] = x.code;
                    errs[g] = x.what();
                } catch (const std::exception &x) {
                    codes[g] = CBNM_ERR_CONFIG;
                    errs[g] = x.what();
                }
                if (t_round && !t_round_resolved) round_decline(*t_round);
                t_round = nullptr;
            }
        };
        std::vector<std::thread> pool;
        for (int w = 0; w < K; ++w) pool.emplace_back(worker, w);
        for (auto &t : pool) t.join();
        cbnm_timing tm{};
        tm.total_ms = (now_s() - t0) * 1e3;
        for (int w = 0; w < K; ++w) {
            tm.integrate_ms = std::max(tm.integrate_ms, g_batch[w]->timing.integrate_ms);
            tm.fc_ms = std::max(tm.fc_ms, g_batch[w]->timing.fc_ms);
        }
        tm.kernel_launches = launches.load();
        if (combined) {  // the combined integrator launches: their device time and count
            tm.kernel_launches += g_batch_launch->launches;
            if (g_batch_launch->launches) tm.integrate_ms = std::max(tm.integrate_ms, (double)g_batch_launch->kernel_ms);
        }
        tm.h2d_bytes = h2d.load();
        tm.d2h_bytes = d2h.load();
        g_last_timing = tm;
        if (statuses) std::copy(codes.begin(), codes.end(), statuses);
        for (int g = 0; g < n_groups; ++g)
            if (codes[g] != CBNM_OK) throw Err(codes[g], "group " + std::to_string(g) + ": " + errs[g]);
    });
}

int cbnm_last_timing(cbnm_timing *t) {
    if (!t) return CBNM_ERR_ARG;
    *t = g_last_timing;
    return CBNM_OK;
}

int cbnm_reset(void) {
    return guarded([&] { release_session(); });
}

const char *cbnm_last_error(void) { return g_err.c_str(); }

const char *cbnm_last_integrator(void) { return t_last_variant.c_str(); }

int cbnm_measure_fp32_peak(double *ffma_tflops, double *ffma2_tflops) {
    return guarded([&] {
        if (!ffma_tflops || !ffma2_tflops) throw Err(CBNM_ERR_ARG, "null output");
        CK(measure_fp32_peak(ffma_tflops, ffma2_tflops));
    });
}

int cbnm_tune_reset(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned.clear();
    g_tune_loaded = false;
    return CBNM_OK;
}

int cbnm_gof(const double *sim_fc, int n_sims, int n_pairs, const double *emp_fc, const double *sim_fcd,
             int n_window_pairs, const double *emp_fcd, int n_emp_fcd, double *fc_corr, double *fc_diff,
             double *fc_normec, double *fcd_ks) {
    return guarded([&] {
        gof_impl(sim_fc, n_sims, n_pairs, emp_fc, sim_fcd, n_window_pairs, emp_fcd, n_emp_fcd, fc_corr, fc_diff,
                 fc_normec, fcd_ks);
    });
}

int cbnm_adjoint_query(const cbnm_run_args *a, int segment_steps, cbnm_adjoint_sizes *sz) {
    return guarded([&] {
        if (!sz) throw Err(CBNM_ERR_ARG, "null sizes");
        AdjPlan P = adjoint_plan(a, segment_steps);
        sz->n_segments = P.n_seg;
        sz->checkpoint_bytes = (int64_t)P.ck_bytes;
        sz->scratch_bytes = (int64_t)P.scratch_bytes;
        sz->bold_len = P.c.bold_len;
        sz->sims_per_backward_launch = P.chunk;
    });
}

int cbnm_adjoint_forward(const cbnm_run_args *a, int segment_steps, double *bold, void *checkpoints) {
    return guarded([&] { adjoint_forward_impl(a, segment_steps, bold, checkpoints); });
}

int cbnm_adjoint_backward(const cbnm_run_args *a, int segment_steps, const double *dbold, const void *checkpoints,
                          void *scratch, double *grad_global, double *grad_regional) {
    return guarded([&] {
        adjoint_backward_impl(a, segment_steps, dbold, checkpoints, scratch, grad_global, grad_regional);
    });
}

// (1 - r(FC)) + W1(FCD) of device BOLD and its gradient (fit_loss.cu).
static void fit_loss_impl(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                          int window_step, int drop_edges, const double *emp_fc, const double *emp_fcd,
                          int n_emp_fcd, double *loss_fc, double *loss_fcd, double *dbold) {
    if (!bold || !emp_fc || !loss_fc || !loss_fcd) throw Err(CBNM_ERR_ARG, "null array");
    if (n_sims < 1 || nodes < 2 || bold_len < 2 || n_vols_remove < 0 || window_step < 1 || window_size < 0)
        throw Err(CBNM_ERR_ARG, "invalid sizes");
    const int corr_len = bold_len - n_vols_remove;
    if (corr_len < 2) throw Err(CBNM_ERR_CONFIG, "fewer than 2 BOLD volumes for FC");
    // windows as build_cfg (utils.cpp:21-52)
    std::vector<int> ws, we;
    {
        const int half = window_size / 2;
        const int first = (drop_edges ? half : 0) + n_vols_remove;
        const int last = (drop_edges ? corr_len - 1 - half : corr_len - 1) + n_vols_remove;
        for (int ctr = first; ctr <= last; ctr += window_step) {
            ws.push_back(std::max(0, ctr - half));
            we.push_back(std::min(bold_len - 1, ctr + half));
        }
    }
    const int W = (int)ws.size();
    const int P = nodes * (nodes - 1) / 2, M = W * (W - 1) / 2;
    if (W > 1024) throw Err(CBNM_ERR_UNSUPPORTED, "at most 1024 dynamic FC windows are supported");
    if (fit_loss_sort_smem(std::max(1, M)) > 200 * 1024)
        throw Err(CBNM_ERR_UNSUPPORTED, "too many FCD values for the in-block sort (" + std::to_string(M) + ")");
    if (M > 0 && (!emp_fcd || n_emp_fcd < 1)) throw Err(CBNM_ERR_ARG, "the FCD term needs the empirical FCD");
    // empirical FC centred; empirical FCD quantiles at the simulated ranks
    std::vector<double> ec(emp_fc, emp_fc + P), q(std::max(1, M), 0.0);
    double em = 0.0;
    for (double v : ec) em += v;
    em /= P;
    double en = 0.0;
    for (double &v : ec) { v -= em; en += v * v; }
    en = std::sqrt(en);
    if (M > 0) {
        std::vector<double> es(emp_fcd, emp_fcd + n_emp_fcd);
        std::sort(es.begin(), es.end());
        for (int i = 0; i < M; ++i) {
            // floor((i + 1/2) m2 / M) in integers (exact where the quotient is whole)
            const long long k = std::min<long long>(n_emp_fcd - 1, (2LL * i + 1) * n_emp_fcd / (2LL * M));
            q[i] = es[k];
        }
    }
    Session &S = session();
    S.fl_ec.ensure(sizeof(double) * P);
    S.fl_q.ensure(sizeof(double) * q.size());
    S.fl_win.ensure(sizeof(int) * 2 * std::max(1, W));
    CK(cudaMemcpyAsync(S.fl_ec.p, ec.data(), sizeof(double) * P, cudaMemcpyHostToDevice, S.st));
    CK(cudaMemcpyAsync(S.fl_q.p, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice, S.st));
    if (W > 0) {
        CK(cudaMemcpyAsync(S.fl_win.p, ws.data(), sizeof(int) * W, cudaMemcpyHostToDevice, S.st));
        CK(cudaMemcpyAsync(S.fl_win.as<int>() + W, we.data(), sizeof(int) * W, cudaMemcpyHostToDevice, S.st));
    }
    FitLossArgs f{};
    f.nodes = nodes; f.bold_len = bold_len; f.n_vols_remove = n_vols_remove; f.n_pairs = P; f.n_windows = W;
    f.n_window_pairs = M; f.want_grad = dbold != nullptr;
    f.w_start = S.fl_win.as<int>(); f.w_end = S.fl_win.as<int>() + W;
    f.bold = bold; f.emp_c = S.fl_ec.as<double>(); f.emp_norm = en; f.emp_q = S.fl_q.as<double>();
    f.loss_fc = loss_fc; f.loss_fcd = loss_fcd; f.dbold = dbold;
    // per-simulation scratch, chunked to <= 1 GiB
    const size_t per = sizeof(double) * ((size_t)2 * P + (size_t)2 * W * P + 2 * (size_t)std::max(1, M) + 2 * (size_t)W +
                                         (size_t)2 * nodes * (W + 1));
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(n_sims, ((size_t)1 << 30) / per));
    double *base = (double *)S.fl_scr.ensure(per * chunk);
    int launches = 0;
    CK(cudaEventRecord(S.ev[0], S.st));
    for (int s0 = 0; s0 < n_sims; s0 += chunk) {
        f.sim_begin = s0;
        f.sim_count = std::min(chunk, n_sims - s0);
        const size_t c = (size_t)chunk;
        double *p = base;
        f.fc = p; p += c * P;
        f.g_fc = p; p += c * P;
        f.wfc = p; p += c * W * P;
        f.g_wfc = p; p += c * W * P;
        f.fcd = p; p += c * std::max(1, M);
        f.g_fcd = p; p += c * std::max(1, M);
        f.wstat = p; p += c * 2 * W;
        f.stats = p;
        CK(launch_fit_loss(f, S.st, &launches));
    }
    CK(cudaEventRecord(S.ev[1], S.st));
    CK(cudaStreamSynchronize(S.st));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, S.ev[0], S.ev[1]);
    cbnm_timing tm{};
    tm.fc_ms = ms;
    tm.total_ms = ms;
    tm.kernel_launches = launches;
    g_last_timing = tm;
}

int cbnm_fit_loss(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                  int window_step, int drop_edges, const double *emp_fc, const double *emp_fcd, int n_emp_fcd,
                  double *loss_fc, double *loss_fcd, double *dbold) {
    return guarded([&] {
        fit_loss_impl(bold, n_sims, bold_len, nodes, n_vols_remove, window_size, window_step, drop_edges, emp_fc,
                      emp_fcd, n_emp_fcd, loss_fc, loss_fcd, dbold);
    });
}

int cbnm_fc_fcd_noalloc(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                        int window_step, int drop_edges, int exc_interhemispheric, double *fc, double *fcd,
                        void *stream) {
    char msg[256];
    const int rc = fc_fcd_noalloc(bold, n_sims, bold_len, nodes, n_vols_remove, window_size, window_step, drop_edges,
                                  exc_interhemispheric, fc, fcd, (cudaStream_t)stream, msg, sizeof(msg));
    g_err = rc ? msg : "";
    return rc;
}

}  // extern "C"
