/*
 * CPU oracle for the cubnm_b200 simulation path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's CPU engine, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  The
 * product library (cubnm_b200/csrc) never links or calls this file.
 *
 * What it follows (paths inside the reference project):
 *   per-simulation loop        src/ext/bnm.cpp:69-522
 *   OpenMP over simulations    src/ext/bnm.cpp:524-583
 *   session init / noise       src/ext/bnm.cpp:585-715, src/ext/utils.cpp:74-95
 *   windows / pair counts      src/ext/utils.cpp:6-72
 *   FC / FCD                   src/ext/fc.cpp:1-91 (Pearson r per pair; computed
 *                              two-pass as in src/ext/fc.cu:4-239)
 *   Balloon-Windkessel         src/ext/models/bw.cpp:4-35
 *   models                     src/ext/models/{rww,wc,jr,kuramoto,rwwex}.cpp
 *   rWW analytical FIC         src/ext/models/rww.cpp:73-146, rww_fic.cpp:62-231
 *   config parsing             include/cubnm/models/base.hpp:51-68, 271-297;
 *                              src/ext/models/rww.cpp:54-71
 *
 * Third-party arithmetic restated here: GSL 2.7's Brent root bracketing
 * (gsl_root_fsolver_brent + gsl_root_test_interval, rww_fic.cpp:62-102), whose
 * iteration brent_root follows step for step;
 * GSL's gsl_blas_ddot is a sequential dot product.  std::mt19937 and libstdc++'s
 * std::normal_distribution<double> produce the noise values as the reference
 * does (bnm.cpp:690-706); the node/time shuffles are restated (shuffle_ref).
 *
 * Pinned against the reference's own stored outputs in tests/expected/sim/ (one .pkl.gz per model)
 * (copied into tests/golden/sim_golden.npz by tests/golden/make_golden.py).
 *
 * Build: see oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/cubnm_b200.h"

namespace orc {

// ---------------------------------------------------------------- BW constants
// src/ext/models/bw.cpp:4-22; set_const core.cpp:157-192
struct BWConst {
    double dt, rho, alpha, tau, y, kappa, V_0, k1, k2, k3;
    double ialpha, itau, oneminrho, dt_itau, V_0_k1, V_0_k2, V_0_k3;
};
static BWConst bw_defaults(double dt_s) {
    BWConst c;
    c.dt = dt_s;
    c.rho = 0.34;
    c.alpha = 0.32;
    c.tau = 0.98;
    c.y = 1.0 / 0.41;
    c.kappa = 1.0 / 0.65;
    c.V_0 = 0.02 * 100;
    c.k1 = 7 * c.rho;
    c.k2 = 2.0;
    c.k3 = 2 * c.rho - 0.2;
    c.ialpha = 1.0 / c.alpha;
    c.itau = 1.0 / c.tau;
    c.oneminrho = (1.0 - c.rho);
    c.dt_itau = c.dt * c.itau;
    c.V_0_k1 = c.V_0 * c.k1;
    c.V_0_k2 = c.V_0 * c.k2;
    c.V_0_k3 = c.V_0 * c.k3;
    return c;
}
static BWConst g_bw = bw_defaults(0.001);
static std::string g_err;

// BW Euler step, bw.cpp:24-35 (note: the q update uses the already-updated nu)
static inline void bw_step(double &x, double &f, double &nu, double &q, double n_state, const BWConst &c) {
    x = x + c.dt * (n_state - c.kappa * x - c.y * (f - 1.0));
    double tmp_f = f + c.dt * x;
    nu = nu + c.dt_itau * (f - std::pow(nu, c.ialpha));
    q = q + c.dt_itau * (f * (1.0 - std::pow(c.oneminrho, (1.0 / f))) / c.rho - std::pow(nu, c.ialpha) * q / nu);
    f = tmp_f;
}

// ---------------------------------------------------------------- run config
struct RunCfg {
    // base config, base.hpp:111-124 defaults
    bool verbose = false, do_fc = true, do_fcd = true;
    int bold_remove_s = 30;
    bool exc_interhemispheric = true;
    int window_size = 10, window_step = 2;
    bool drop_edges = true, ext_out = true, states_ts = false;
    int noise_time_steps = 30000;
    // rWW config, rww.hpp:61-69 (I_SAMPLING_* converted to bw iterations)
    bool do_fic = true;
    int max_fic_trials = 0;
    int I_SAMPLING_START = 1000, I_SAMPLING_END = 10000, I_SAMPLING_DURATION = 10000 - 1000 + 1;
    double init_delta = 0.02;
    // sizes, base.hpp:51-68
    int nodes = 0, n_sims = 0, time_steps = 0, BOLD_TR = 0, states_sampling = 0, sim_seed = 0;
    double dt = 0.1, bw_dt = 0.001;  // dt in ms, bw_dt in s
    int bold_len = 0, BOLD_TR_iters = 0, states_len = 0, states_sampling_iters = 0;
    int bw_it = 0, inner_it = 0;
    int n_vols_remove = 0, n_states_samples_remove = 0, corr_len = 0;
    int n_pairs = 0, n_windows = 0, n_window_pairs = 0;
    std::vector<int> window_starts, window_ends;
    int noise_bw_it = 0, noise_repeats = 0;
    int64_t noise_size = 0;
    bool do_delay = false;
};

static void parse_config(RunCfg &c, const cbnm_run_args *a, bool is_rww) {
    // base.hpp:271-297 and rww.cpp:54-71
    for (int i = 0; i < a->n_config; ++i) {
        std::string k = a->config_keys[i], v = a->config_values[i];
        if (k == "verbose") c.verbose = std::stoi(v) != 0;
        else if (k == "do_fc") c.do_fc = std::stoi(v) != 0;
        else if (k == "do_fcd") c.do_fcd = std::stoi(v) != 0;
        else if (k == "bold_remove_s") c.bold_remove_s = std::stoi(v);
        else if (k == "exc_interhemispheric") c.exc_interhemispheric = std::stoi(v) != 0;
        else if (k == "window_size") c.window_size = std::stoi(v);
        else if (k == "window_step") c.window_step = std::stoi(v);
        else if (k == "drop_edges") c.drop_edges = std::stoi(v) != 0;
        else if (k == "noise_time_steps") c.noise_time_steps = std::stoi(v);
        if (is_rww) {
            if (k == "do_fic") c.do_fic = std::stoi(v) != 0;
            else if (k == "max_fic_trials") c.max_fic_trials = std::stoi(v);
            else if (k == "I_SAMPLING_START") c.I_SAMPLING_START = (int)((std::stoi(v) / 1000) / c.bw_dt);
            else if (k == "I_SAMPLING_END") c.I_SAMPLING_END = (int)((std::stoi(v) / 1000) / c.bw_dt);
            else if (k == "init_delta") c.init_delta = std::stod(v);
        }
    }
    // rww.cpp:65 recomputes the duration after each key
    c.I_SAMPLING_DURATION = c.I_SAMPLING_END - c.I_SAMPLING_START + 1;
}

// utils.cpp:6-19
static int fc_n_pairs(int nodes, bool exc_inter) {
    int n = nodes * (nodes - 1) / 2;
    if (exc_inter) {
        if (nodes % 2 != 0) throw std::runtime_error("exc_interhemispheric is set but number of nodes is not even");
        int rh = nodes / 2;
        n -= rh * rh;
    }
    return n;
}

// utils.cpp:21-52
static int dfc_windows(std::vector<int> &starts, std::vector<int> &ends, int corr_len, int bold_len,
                       int n_vols_remove, int step, int size, bool drop_edges) {
    int first = drop_edges ? size / 2 : 0;
    int last = drop_edges ? corr_len - 1 - size / 2 : corr_len - 1;
    first += n_vols_remove;
    last += n_vols_remove;
    for (int center = first; center <= last; center += step) {
        int s = center - size / 2;
        if (s < 0) s = 0;
        int e = center + size / 2;
        if (e >= bold_len) e = bold_len - 1;
        starts.push_back(s);
        ends.push_back(e);
    }
    if (starts.empty()) throw std::runtime_error("Number of dynamic FC windows is 0");
    return (int)starts.size();
}

static void setup_sizes(RunCfg &c, const cbnm_run_args *a) {
    c.nodes = a->nodes; c.n_sims = a->n_sims; c.time_steps = a->time_steps; c.BOLD_TR = a->bold_tr;
    c.states_sampling = a->states_sampling; c.sim_seed = a->sim_seed; c.dt = a->dt; c.bw_dt = a->bw_dt / 1000.0;
    c.do_delay = a->do_delay != 0;
    c.ext_out = a->ext_out != 0;
    c.states_ts = a->states_ts != 0;
    // base.hpp:51-68 (truncating int conversions kept)
    c.bold_len = c.time_steps / c.BOLD_TR;
    c.BOLD_TR_iters = (int)(((double)c.BOLD_TR / 1000.0) / c.bw_dt);
    c.states_len = c.time_steps / c.states_sampling;
    c.states_sampling_iters = (int)(((double)c.states_sampling / 1000.0) / c.bw_dt);
    c.bw_it = (int)(((double)c.time_steps / 1000.0) / c.bw_dt);
    c.inner_it = (int)((c.bw_dt * 1000) / c.dt);
    // bnm.cpp:630-657
    c.n_states_samples_remove = c.bold_remove_s * 1000 / c.states_sampling;
    if (c.do_fc) {
        c.n_vols_remove = c.bold_remove_s * 1000 / c.BOLD_TR;
        c.corr_len = c.bold_len - c.n_vols_remove;
        if (c.corr_len < 2) throw std::runtime_error("Number of BOLD volumes (after removing initial volumes) is too low for FC calculations");
        c.n_pairs = fc_n_pairs(c.nodes, c.exc_interhemispheric);
        if (c.do_fcd) {
            c.n_windows = dfc_windows(c.window_starts, c.window_ends, c.corr_len, c.bold_len, c.n_vols_remove,
                                      c.window_step, c.window_size, c.drop_edges);
            c.n_window_pairs = c.n_windows * (c.n_windows - 1) / 2;
        }
    } else {
        c.do_fcd = false;
    }
    // bnm.cpp:679-681 (segmented noise)
    c.noise_bw_it = (int)(((double)(c.noise_time_steps) / 1000.0) / c.bw_dt);
    c.noise_repeats = (int)std::ceil((double)(c.bw_it) / (double)(c.noise_bw_it));
}

// ---------------------------------------------------------------- models
// Each model restates src/ext/models/<model>.cpp init_constants / h_init / h_step.
struct ModelRWW {
    static constexpr int NS = 6, NI = 7, NN = 2, NG = 1, NR = 4, CONN = 4, BOLDV = 4, NGB = 2, NGI = 1;
    static constexpr bool OSC = false, POSTBW = true;
    struct K {
        double dt, sqrt_dt, a_E, b_E, d_E, a_I, b_I, d_I, gamma_E, gamma_I, tau_E, tau_I, I_0, w_E, w_I, w_II, I_ext;
        double w_E__I_0, w_I__I_0, b_a_ratio_E, itau_E, itau_I, dt_itau_E, dt_gamma_E, dt_itau_I, dt_gamma_I;
        double tau_E_s, tau_I_s, gamma_E_s, gamma_I_s, r_I_ss, r_E_ss, I_I_ss, I_E_ss, S_I_ss, S_E_ss;
    };
    static K make(double dt) {  // rww.cpp:8-53
        K m;
        m.dt = dt; m.sqrt_dt = std::sqrt(m.dt);
        m.a_E = 310; m.b_E = 125; m.d_E = 0.16; m.a_I = 615; m.b_I = 177; m.d_I = 0.087;
        m.gamma_E = (double)0.641 / (double)1000.0; m.gamma_I = (double)1.0 / (double)1000.0;
        m.tau_E = 100; m.tau_I = 10; m.I_0 = 0.382; m.w_E = 1.0; m.w_I = 0.7; m.w_II = 1.0; m.I_ext = 0.0;
        m.w_E__I_0 = m.w_E * m.I_0; m.w_I__I_0 = m.w_I * m.I_0; m.b_a_ratio_E = m.b_E / m.a_E;
        m.itau_E = 1.0 / m.tau_E; m.itau_I = 1.0 / m.tau_I;
        m.dt_itau_E = m.dt * m.itau_E; m.dt_gamma_E = m.dt * m.gamma_E;
        m.dt_itau_I = m.dt * m.itau_I; m.dt_gamma_I = m.dt * m.gamma_I;
        m.tau_E_s = 0.1; m.tau_I_s = 0.01; m.gamma_E_s = 0.641; m.gamma_I_s = 1.0;
        m.r_I_ss = 3.9218448633; m.r_E_ss = 3.0773270642; m.I_I_ss = 0.2528951325; m.I_E_ss = 0.3773805650;
        m.S_I_ss = 0.0392184486; m.S_E_ss = 0.1647572075;
        return m;
    }
    static void init(double *s, double *iv, const double *, const double *, const RunCfg &c) {  // rww.cpp:156-177
        s[4] = 0.001; s[5] = 0.001; iv[4] = 0.0; iv[5] = c.init_delta;
    }
    static void restart(double *s, double *iv, const double *, const double *) {  // rww.cpp:179-192
        s[4] = 0.001; s[5] = 0.001; iv[4] = 0.0;
    }
    static void step(double *s, double *iv, const double *g, const double *r, double in, const double *noise,
                     int64_t ni, const K &m) {  // rww.cpp:194-232
        s[0] = m.w_E__I_0 + r[0] * r[1] * s[4] + in * g[0] * r[1] - r[2] * s[5];
        s[1] = m.w_I__I_0 + r[1] * s[4] - m.w_II * s[5];
        iv[0] = m.a_E * s[0] - m.b_E;
        iv[1] = m.a_I * s[1] - m.b_I;
        s[2] = iv[0] / (1 - std::exp(-m.d_E * iv[0]));
        s[3] = iv[1] / (1 - std::exp(-m.d_I * iv[1]));
        iv[2] = noise[ni] * r[3] * m.sqrt_dt + m.dt_gamma_E * ((1 - s[4]) * s[2]) - m.dt_itau_E * s[4];
        iv[3] = noise[ni + 1] * r[3] * m.sqrt_dt + m.dt_gamma_I * s[3] - m.dt_itau_I * s[5];
        s[4] += iv[2];
        s[5] += iv[3];
        s[4] = std::max(0.0, std::min(1.0, s[4]));
        s[5] = std::max(0.0, std::min(1.0, s[5]));
    }
};

struct ModelWC {
    static constexpr int NS = 2, NI = 4, NN = 2, NG = 1, NR = 8, CONN = 0, BOLDV = 0, NGB = 0, NGI = 0;
    static constexpr bool OSC = false, POSTBW = false;
    struct K { double dt, sqrt_dt, tau_E, tau_I, itau_E, itau_I, a_E, a_I, mu_E, mu_I; };
    static K make(double dt) {  // wc.cpp:14-25
        K m;
        m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.tau_E = 2.5; m.tau_I = 3.75;
        m.itau_E = 1.0 / m.tau_E; m.itau_I = 1.0 / m.tau_I; m.a_E = 1.5; m.a_I = 1.5; m.mu_E = 3.0; m.mu_I = 3.0;
        return m;
    }
    static void init(double *s, double *, const double *, const double *, const RunCfg &) { s[0] = 0.001; s[1] = 0.001; }
    static void restart(double *s, double *, const double *, const double *) { s[0] = 0.001; s[1] = 0.001; }
    static void step(double *s, double *iv, const double *g, const double *r, double in, const double *noise,
                     int64_t ni, const K &m) {  // wc.cpp:51-80
        iv[0] = 1.0 / (1.0 + std::exp(-m.a_E * (r[0] * s[0] - r[1] * s[1] + g[0] * in + r[4] - m.mu_E)));
        iv[1] = 1.0 / (1.0 + std::exp(-m.a_I * (r[2] * s[0] - r[3] * s[1] + r[5] - m.mu_I)));
        iv[2] = (-s[0] + (1.0 - s[0]) * iv[0]) * m.itau_E;
        iv[3] = (-s[1] + (1.0 - s[1]) * iv[1]) * m.itau_I;
        s[0] += m.dt * iv[2] + m.sqrt_dt * noise[ni] * r[6];
        s[1] += m.dt * iv[3] + m.sqrt_dt * noise[ni + 1] * r[7];
        s[0] = std::max(0.0, std::min(1.0, s[0]));
        s[1] = std::max(0.0, std::min(1.0, s[1]));
    }
};

struct ModelJR {
    static constexpr int NS = 8, NI = 9, NN = 1, NG = 1, NR = 6, CONN = 7, BOLDV = 6, NGB = 0, NGI = 0;
    static constexpr bool OSC = false, POSTBW = false;
    struct K { double dt, sqrt_dt, A, B, a, b, v0, nu_max, r, p_min, p_max, mu, cmin, cmax, midpoint, a_sq, b_sq; };
    static K make(double dt) {  // jr.cpp:14-30
        K m;
        m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.A = 3.25; m.B = 22.0; m.a = 0.1; m.b = 0.05; m.v0 = 6.0;
        m.nu_max = 0.0025; m.r = 0.56; m.p_min = 0.12; m.p_max = 0.32; m.mu = 0.22; m.cmin = 0.0; m.cmax = 0.005;
        m.midpoint = 6.0;
        m.a_sq = std::pow(m.a, 2); m.b_sq = std::pow(m.b, 2);  // jr.cpp:101,105 pow(a,2), pow(b,2)
        return m;
    }
    static void init(double *s, double *, const double *, const double *, const RunCfg &) { for (int i = 0; i < 8; ++i) s[i] = 0.0; }
    static void restart(double *s, double *, const double *, const double *) { for (int i = 0; i < 8; ++i) s[i] = 0.0; }
    static void step(double *s, double *iv, const double *g, const double *r, double in, const double *noise,
                     int64_t ni, const K &m) {  // jr.cpp:80-133
        iv[0] = 2.0 * m.nu_max / (1.0 + std::exp(m.r * (m.v0 - (s[1] - s[2]))));
        iv[1] = 2.0 * m.nu_max / (1.0 + std::exp(m.r * (m.v0 - (r[1] * r[0] * s[0]))));
        iv[2] = 2.0 * m.nu_max / (1.0 + std::exp(m.r * (m.v0 - (r[3] * r[0] * s[0]))));
        iv[3] = s[3];
        iv[4] = s[4];
        iv[5] = s[5];
        iv[6] = m.A * m.a * iv[0] - 2.0 * m.a * s[3] - (m.a_sq) * s[0];
        iv[7] = m.A * m.a * (m.mu + r[2] * r[0] * iv[1] + g[0] * in) - 2.0 * m.a * s[4] - (m.a_sq) * s[1];
        iv[8] = m.B * m.b * (r[4] * r[0] * iv[2]) - 2.0 * m.b * s[5] - (m.b_sq) * s[2];
        s[0] += m.dt * iv[3];
        s[1] += m.dt * iv[4];
        s[2] += m.dt * iv[5];
        s[3] += m.dt * iv[6] + m.sqrt_dt * noise[ni] * r[5];
        s[4] += m.dt * iv[7];
        s[5] += m.dt * iv[8];
        s[6] = s[1] - s[2];
        s[7] = m.cmin + (m.cmax - m.cmin) / (1.0 + std::exp(m.r * (m.midpoint - (s[6]))));
    }
};

struct ModelKuramoto {
    static constexpr int NS = 1, NI = 1, NN = 1, NG = 1, NR = 3, CONN = 0, BOLDV = 0, NGB = 0, NGI = 0;
    static constexpr bool OSC = true, POSTBW = false;
    struct K { double dt, sqrt_dt, twopi; };
    static K make(double dt) {  // kuramoto.cpp:14-18
        K m;
        m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.twopi = 2.0 * M_PI;
        return m;
    }
    static void init(double *s, double *, const double *, const double *r, const RunCfg &) { s[0] = r[0]; }
    static void restart(double *s, double *, const double *, const double *r) { s[0] = r[0]; }
    static void step(double *s, double *iv, const double *g, const double *r, double in, const double *noise,
                     int64_t ni, const K &m) {  // kuramoto.cpp:48-61
        iv[0] = r[1] + g[0] * in;
        s[0] = s[0] + m.dt * iv[0] + m.sqrt_dt * noise[ni] * r[2];
        s[0] = std::fmod(s[0], m.twopi);
    }
};

struct ModelRWWEx {
    static constexpr int NS = 3, NI = 2, NN = 1, NG = 1, NR = 3, CONN = 2, BOLDV = 2, NGB = 0, NGI = 0;
    static constexpr bool OSC = false, POSTBW = false;
    struct K { double dt, sqrt_dt, J_N, a, b, d, gamma, tau, itau, dt_itau, dt_gamma; };
    static K make(double dt) {  // rwwex.cpp:14-26
        K m;
        m.dt = dt; m.sqrt_dt = std::sqrt(m.dt); m.J_N = 0.2609; m.a = 270; m.b = 108; m.d = 0.154;
        m.gamma = (double)0.641 / (double)1000.0; m.tau = 100; m.itau = 1.0 / m.tau;
        m.dt_itau = m.dt * m.itau; m.dt_gamma = m.dt * m.gamma;
        return m;
    }
    static void init(double *s, double *, const double *, const double *, const RunCfg &) { s[2] = 0.001; }
    static void restart(double *s, double *, const double *, const double *) { s[2] = 0.001; }
    static void step(double *s, double *iv, const double *g, const double *r, double in, const double *noise,
                     int64_t ni, const K &m) {  // rwwex.cpp:48-73
        s[0] = r[0] * m.J_N * s[2] + g[0] * m.J_N * in + r[1];
        iv[0] = m.a * s[0] - m.b;
        s[1] = iv[0] / (1 - std::exp(-m.d * iv[0]));
        iv[1] = m.dt_gamma * ((1 - s[2]) * s[1]) - m.dt_itau * s[2] + noise[ni] * m.sqrt_dt * r[2];
        s[2] += iv[1];
        s[2] = std::max(0.0, std::min(1.0, s[2]));
    }
};

// ---------------------------------------------------------------- analytical FIC
// Brent's method (R. P. Brent, "Algorithms for Minimization without
// Derivatives", 1973, ch. 4) with the iteration of GSL 2.7's brent fsolver
// (gsl_root_fsolver_brent, step for step, which FIC parity needs), driven the
// way GSL's fsolver interface drives it: every iteration reports the bracket
// [min(b,c), max(b,c)]; the caller stops when
//   |hi - lo| < epsabs + epsrel * min(|lo|,|hi|)   (min -> 0 if 0 is inside)
// with epsabs = 0, epsrel = 1e-3 and at most 100 iterations (rww_fic.cpp:62-102).
// Returns -1 when the endpoints do not straddle a root or it does not converge.
template <class F>
static double brent_root(F f, double x_lo, double x_hi) {
    const double eps = 2.2204460492503131e-16;
    double a = x_lo, b = x_hi;
    double fa = f(a), fb = f(b);
    if ((fa < 0.0 && fb < 0.0) || (fa > 0.0 && fb > 0.0)) return -1;
    double c = b, fc = fb;
    double d = b - a, e = b - a;
    double root = 0.5 * (x_lo + x_hi);
    for (int iter = 1; iter <= 100; ++iter) {
        bool lin = false;
        if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {  // keep the root between b and c
            lin = true;
            c = a; fc = fa;
            d = b - a; e = b - a;
        }
        if (std::fabs(fc) < std::fabs(fb)) {  // b is the best estimate
            lin = true;
            a = b; b = c; c = a;
            fa = fb; fb = fc; fc = fa;
        }
        double tol = 0.5 * eps * std::fabs(b);
        double m = 0.5 * (c - b);
        double lo, hi;
        if (fb == 0) {
            root = b; lo = b; hi = b;
        } else if (std::fabs(m) <= tol) {
            root = b; lo = std::min(b, c); hi = std::max(b, c);
        } else {
            if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
                d = m; e = m;  // bisection
            } else {
                double p, q, r, s = fb / fa;
                if (lin) {  // secant
                    p = 2 * m * s;
                    q = 1 - s;
                } else {  // inverse quadratic interpolation
                    q = fa / fc;
                    r = fb / fc;
                    p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
                    q = (q - 1) * (r - 1) * (s - 1);
                }
                if (p > 0) q = -q; else p = -p;
                if (2 * p < std::min(3 * m * q - std::fabs(tol * q), std::fabs(e * q))) {
                    e = d; d = p / q;
                } else {
                    d = m; e = m;
                }
            }
            a = b; fa = fb;
            if (std::fabs(d) > tol) b += d; else b += (m > 0 ? +tol : -tol);
            fb = f(b);
            root = b;
            double cc = c;
            if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) cc = a;
            if (b < cc) { lo = b; hi = cc; } else { lo = cc; hi = b; }
        }
        double alo = std::fabs(lo), ahi = std::fabs(hi);
        double min_abs = ((lo > 0 && hi > 0) || (lo < 0 && hi < 0)) ? std::min(alo, ahi) : 0.0;
        if (std::fabs(hi - lo) < 0.001 * min_abs) return root;
    }
    return -1;
}

// rww_fic.cpp:104-135 transfer function of the inhibitory pool
static inline double phi_I(double II, const ModelRWW::K &m) {
    return ((m.a_I * II) - m.b_I) / (1 - std::exp(-1 * m.d_I * ((m.a_I * II) - m.b_I)));
}

// rww_fic.cpp:138-231 (sc_t is the target-by-source matrix, i.e. SC transposed)
static bool analytical_fic(const std::vector<double> &sc_t, int n, double G, const double *w_EE, const double *w_EI,
                           double *w_IE_out, const ModelRWW::K &m) {
    const double I0_I = m.I_0 * m.w_I, I0_E = m.I_0 * m.w_E;
    for (int j = 0; j < n; ++j) {
        const double w_EI_j = w_EI[j], S_E_ss = m.S_E_ss, w_II = m.w_II;
        auto F = [&](double x) {
            return I0_I + w_EI_j * S_E_ss - w_II * m.gamma_I_s * m.tau_I_s * phi_I(x, m) - x;
        };
        double I_I = brent_root(F, 0.0, 2.0);
        if (I_I == -1) return true;
        double r_I = phi_I(I_I, m);
        double S_I_ss = r_I * m.tau_I_s * m.gamma_I_s;
        double dot = 0.0;  // gsl_blas_ddot(K_EE row j, S_E_ss)
        for (int k = 0; k < n; ++k) {
            double kee = (sc_t[(size_t)j * n + k] * G) * w_EI[j];
            if (k == j) kee = kee + w_EE[j];
            dot += kee * S_E_ss;
        }
        double w_IE = (-1 / S_I_ss) * (m.I_E_ss - m.I_ext - I0_E - dot);
        if (w_IE < 0) return true;
        w_IE_out[j] = w_IE;
    }
    return false;
}

// rww.cpp:73-146
static void rww_prep_params(const RunCfg &c, const cbnm_run_args *a, double *regional, uint8_t *unstable,
                            const ModelRWW::K &m) {
    const int n = c.nodes;
    std::vector<std::vector<double>> sc_t(a->n_scs, std::vector<double>((size_t)n * n));
    for (int s = 0; s < a->n_scs; ++s)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) sc_t[s][(size_t)j * n + k] = a->sc[(size_t)s * n * n + (size_t)k * n + j];
    std::vector<double> w_EE(n), w_EI(n), w_IE(n);
    const size_t stride = (size_t)c.n_sims * n;
    for (int sim = 0; sim < c.n_sims; ++sim) {
        for (int j = 0; j < n; ++j) {
            w_EI[j] = regional[1 * stride + (size_t)sim * n + j];
            w_EE[j] = regional[0 * stride + (size_t)sim * n + j] * w_EI[j];
        }
        bool bad = analytical_fic(sc_t[a->sc_indices[sim]], n, a->global_params[sim], w_EE.data(), w_EI.data(),
                                  w_IE.data(), m);
        unstable[sim] = bad ? 1 : 0;
        for (int j = 0; j < n; ++j) regional[2 * stride + (size_t)sim * n + j] = bad ? 1.0 : w_IE[j];
    }
}

// ---------------------------------------------------------------- FC / FCD
// Pearson r of columns i, j over rows [r0, r1) of a (rows x nodes) matrix;
// two-pass means and sums of squares as in fc.cu:4-125.
static void col_stats(const double *bold, int nodes, int r0, int r1, std::vector<double> &mean, std::vector<double> &ssd) {
    mean.assign(nodes, 0.0); ssd.assign(nodes, 0.0);
    for (int j = 0; j < nodes; ++j) {
        double s = 0;
        for (int t = r0; t < r1; ++t) s += bold[(size_t)t * nodes + j];
        s /= (r1 - r0);
        double q = 0;
        for (int t = r0; t < r1; ++t) { double dlt = bold[(size_t)t * nodes + j] - s; q += dlt * dlt; }
        mean[j] = s; ssd[j] = std::sqrt(q);
    }
}
static void fc_tril(const double *bold, int nodes, int r0, int r1, bool exc_inter, double *out) {
    std::vector<double> mean, ssd;
    col_stats(bold, nodes, r0, r1, mean, ssd);
    int rh = nodes / 2, p = 0;
    for (int i = 0; i < nodes; ++i)
        for (int j = 0; j < i; ++j) {
            if (exc_inter && ((i < rh) ^ (j < rh))) continue;
            double cov = 0;
            for (int t = r0; t < r1; ++t)
                cov += (bold[(size_t)t * nodes + i] - mean[i]) * (bold[(size_t)t * nodes + j] - mean[j]);
            out[p++] = cov / (ssd[i] * ssd[j]);
        }
}
static void fcd_tril(const double *bold, const RunCfg &c, double *out) {
    const int W = c.n_windows, P = c.n_pairs;
    std::vector<double> wfc((size_t)W * P);
    for (int w = 0; w < W; ++w)
        fc_tril(bold, c.nodes, c.window_starts[w], c.window_ends[w] + 1, c.exc_interhemispheric, &wfc[(size_t)w * P]);
    std::vector<double> mean(W), ssd(W);
    for (int w = 0; w < W; ++w) {
        double s = 0;
        for (int p = 0; p < P; ++p) s += wfc[(size_t)w * P + p];
        s /= P;
        double q = 0;
        for (int p = 0; p < P; ++p) { double dlt = wfc[(size_t)w * P + p] - s; q += dlt * dlt; }
        mean[w] = s; ssd[w] = std::sqrt(q);
    }
    int idx = 0;
    for (int wi = 0; wi < W; ++wi)
        for (int wj = 0; wj < wi; ++wj) {
            double cov = 0;
            for (int p = 0; p < P; ++p) cov += (wfc[(size_t)wi * P + p] - mean[wi]) * (wfc[(size_t)wj * P + p] - mean[wj]);
            out[idx++] = cov / (ssd[wi] * ssd[wj]);
        }
}

// ---------------------------------------------------------------- noise
// The reference shuffles with std::shuffle(first, last, mt19937&) (utils.cpp:74-95).
// Its stored outputs were produced by a libstdc++ whose bounded integer draw
// is the division-based rejection method, and whose shuffle draws two swap
// positions per random number when the generator's range allows (every case
// here).  Both are restated explicitly so the noise does not depend on the
// libstdc++ the host happens to have (newer releases draw bounded integers by
// multiply-shift, which permutes differently).
static uint64_t bounded_draw(std::mt19937 &g, uint64_t range_max) {  // uniform in [0, range_max]
    const uint64_t urng_range = 0xffffffffULL;
    const uint64_t span = range_max + 1, scaling = urng_range / span, past = span * scaling;
    uint64_t r;
    do { r = (uint64_t)g(); } while (r >= past);
    return r / scaling;
}
static void shuffle_ref(std::vector<int> &v, std::mt19937 &g) {
    const uint64_t n = v.size();
    if (n < 2) return;
    if (0xffffffffULL / n < n) {  // n^2 exceeds the generator's range: one draw in [0, i] per element
        for (size_t i = 1; i < n; ++i) std::swap(v[i], v[bounded_draw(g, i)]);
        return;
    }
    size_t i = 1;
    if (n % 2 == 0) { std::swap(v[i], v[bounded_draw(g, 1)]); ++i; }
    while (i != n) {  // positions for elements i and i+1 from one draw in [0, (i+1)(i+2))
        const uint64_t b0 = i + 1, b1 = i + 2;
        const uint64_t x = bounded_draw(g, b0 * b1 - 1);
        std::swap(v[i], v[x / b1]); ++i;
        std::swap(v[i], v[x % b1]); ++i;
    }
}
// bnm.cpp:690-706 and utils.cpp:74-95
struct Noise {
    std::vector<double> noise;
    std::vector<int32_t> sh_nodes, sh_ts;
    int64_t key_size = -1;
    int key_seed = 0, key_nodes = 0, key_time = 0, key_nts = 0;
};
static Noise g_noise;

static void make_noise(const RunCfg &c, int n_noise, bool force) {
    int64_t size = (int64_t)c.nodes * c.noise_bw_it * c.inner_it * n_noise;
    if (!force && g_noise.key_size == size && g_noise.key_seed == c.sim_seed && g_noise.key_nodes == c.nodes &&
        g_noise.key_time == c.time_steps && g_noise.key_nts == c.noise_time_steps)
        return;
    std::mt19937 gen(c.sim_seed);
    std::normal_distribution<double> nd(0, 1);
    g_noise.noise.resize(size);
    for (int64_t i = 0; i < size; ++i) g_noise.noise[i] = nd(gen);
    std::vector<int> idx(c.nodes);
    g_noise.sh_nodes.resize((size_t)c.noise_repeats * c.nodes);
    std::iota(idx.begin(), idx.end(), 0);
    for (int r = 0; r < c.noise_repeats; ++r) {
        shuffle_ref(idx, gen);
        std::copy(idx.begin(), idx.end(), g_noise.sh_nodes.begin() + (size_t)r * c.nodes);
    }
    std::vector<int> ts(c.noise_bw_it);
    g_noise.sh_ts.resize((size_t)c.noise_repeats * c.noise_bw_it);
    std::iota(ts.begin(), ts.end(), 0);
    for (int r = 0; r < c.noise_repeats; ++r) {
        shuffle_ref(ts, gen);
        std::copy(ts.begin(), ts.end(), g_noise.sh_ts.begin() + (size_t)r * c.noise_bw_it);
    }
    g_noise.key_size = size; g_noise.key_seed = c.sim_seed; g_noise.key_nodes = c.nodes;
    g_noise.key_time = c.time_steps; g_noise.key_nts = c.noise_time_steps;
}

// ---------------------------------------------------------------- one simulation
// bnm.cpp:69-522
template <class M>
static void simulate(int sim, const RunCfg &c, const cbnm_run_args *a, const double *regional_in, double *regional_out,
                     const typename M::K &m, const BWConst &bwc, double *bold_out, double *fc_out, double *fcd_out,
                     double *states_out, int32_t *gints, uint8_t *gbools) {
    const int n = c.nodes;
    const size_t rstride = (size_t)c.n_sims * n;
    const double *SC = a->sc + (size_t)a->sc_indices[sim] * n * n;
    double g[M::NG];
    for (int i = 0; i < M::NG; ++i) g[i] = a->global_params[(size_t)i * c.n_sims + sim];
    std::vector<double> r((size_t)n * M::NR), s((size_t)n * M::NS, 0.0), iv((size_t)n * M::NI, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < M::NR; ++i) r[(size_t)j * M::NR + i] = regional_in[i * rstride + (size_t)sim * n + j];
    const size_t ext = c.states_ts ? (size_t)n * c.states_len : (size_t)n;
    auto st = [&](int var) { return states_out + ((size_t)var * c.n_sims + sim) * ext; };
    if (c.ext_out && !c.states_ts)
        for (int v = 0; v < M::NS; ++v) std::fill(st(v), st(v) + n, 0.0);
    // model-wide shared flags (rWW: fic_trial, adjust_fic, fic_failed)
    int fic_trial = 0;
    bool adjust_fic = c.do_fic && (c.max_fic_trials > 0), fic_failed = false;
    for (int j = 0; j < n; ++j) M::init(&s[(size_t)j * M::NS], &iv[(size_t)j * M::NI], g, &r[(size_t)j * M::NR], c);
    std::vector<double> bx(n, 0.0), bf(n, 1.0), bnu(n, 1.0), bq(n, 1.0);
    // delays, bnm.cpp:146-202
    std::vector<int> delay;
    int max_delay = 0;
    const double vel = a->v_list[sim] * c.dt;
    if (c.do_delay) {
        delay.assign((size_t)n * n, 0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double len = a->sc_dist[(size_t)i * n + j];
                if (i > j) {
                    int d = (int)rintf(len / vel);
                    d = std::max(d, 1);
                    delay[(size_t)i * n + j] = d;
                    delay[(size_t)j * n + i] = d;
                    if (d > max_delay) max_delay = d;
                } else if (i == j) {
                    delay[(size_t)i * n + j] = 1;
                }
            }
    }
    const bool has_delay = max_delay > 0;
    int buff_idx = max_delay - 1;
    std::vector<double> hist, x1;
    if (has_delay) hist.resize((size_t)n * max_delay); else x1.resize(n);
    auto reset_conn = [&]() {
        for (int j = 0; j < n; ++j) {
            double v = s[(size_t)j * M::NS + M::CONN];
            if (has_delay) for (int b = 0; b < max_delay; ++b) hist[(size_t)b * n + j] = v;
            else x1[j] = v;
        }
    };
    reset_conn();
    std::vector<double> bold((size_t)c.bold_len * n);
    std::vector<double> in(n);
    const double *noise = g_noise.noise.data();
    int bw_i = 0, bold_i = 0, states_i = 0, repeat = 0;
    while (bw_i < c.bw_it) {
        const int sh_ts = g_noise.sh_ts[(size_t)(bw_i % c.noise_bw_it) + (size_t)repeat * c.noise_bw_it];
        for (int inner = 0; inner < c.inner_it; ++inner) {
            // global input, bnm.cpp:14-67
            for (int j = 0; j < n; ++j) {
                double acc = 0;
                if (has_delay) {
                    for (int k = 0; k < n; ++k) {
                        int kb = (buff_idx + delay[(size_t)k * n + j]) % max_delay;
                        if (M::OSC) acc += SC[(size_t)k * n + j] * std::sin(hist[(size_t)kb * n + k] - hist[(size_t)buff_idx * n + j]);
                        else acc += SC[(size_t)k * n + j] * hist[(size_t)kb * n + k];
                    }
                } else {
                    for (int k = 0; k < n; ++k) {
                        if (M::OSC) acc += SC[(size_t)k * n + j] * std::sin(x1[k] - x1[j]);
                        else acc += SC[(size_t)k * n + j] * x1[k];
                    }
                }
                in[j] = acc;
            }
            for (int j = 0; j < n; ++j) {
                int sh_j = g_noise.sh_nodes[(size_t)repeat * n + j];
                int64_t ni = (((int64_t)sh_ts * c.inner_it + inner) * n * M::NN) + (int64_t)sh_j * M::NN;
                M::step(&s[(size_t)j * M::NS], &iv[(size_t)j * M::NI], g, &r[(size_t)j * M::NR], in[j], noise, ni, m);
            }
            if (has_delay) {
                for (int j = 0; j < n; ++j) hist[(size_t)buff_idx * n + j] = s[(size_t)j * M::NS + M::CONN];
                buff_idx = (buff_idx + max_delay - 1) % max_delay;
            } else {
                for (int j = 0; j < n; ++j) x1[j] = s[(size_t)j * M::NS + M::CONN];
            }
        }
        for (int j = 0; j < n; ++j) bw_step(bx[j], bf[j], bnu[j], bq[j], s[(size_t)j * M::NS + M::BOLDV], bwc);
        if ((bw_i + 1) % c.BOLD_TR_iters == 0) {  // bnm.cpp:316-335
            // truncated iteration counts can give one sample past bold_len, which has no slot
            for (int j = 0; j < n && bold_i < c.bold_len; ++j)
                bold[(size_t)bold_i * n + j] = bwc.V_0 * (bwc.k1 * (1 - bq[j]) + bwc.k2 * (1 - bq[j] / bnu[j]) + bwc.k3 * (1 - bnu[j]));
            bold_i++;
        }
        if (c.ext_out && (bw_i + 1) % c.states_sampling_iters == 0) {  // bnm.cpp:337-355
            for (int j = 0; j < n; ++j) {
                if (c.states_ts) {
                    if (states_i < c.states_len)
                        for (int v = 0; v < M::NS; ++v) st(v)[(size_t)states_i * n + j] = s[(size_t)j * M::NS + v];
                } else if (states_i >= c.n_states_samples_remove) {
                    for (int v = 0; v < M::NS; ++v) st(v)[j] += s[(size_t)j * M::NS + v];
                }
            }
            states_i++;
        }
        if ((bw_i + 1) % c.noise_bw_it == 0 && bw_i + 1 < c.bw_it) repeat++;
        bool restart = false;
        if constexpr (M::POSTBW) if (adjust_fic) {  // rww.cpp:233-298 numerical FIC
            const typename M::K &rm = m;
            const int t = bw_i + 1;
            for (int j = 0; j < n; ++j) {
                double *sj = &s[(size_t)j * M::NS], *ivj = &iv[(size_t)j * M::NI], *rj = &r[(size_t)j * M::NR];
                if (t >= c.I_SAMPLING_START && t <= c.I_SAMPLING_END) ivj[4] += sj[0];
                if (t == c.I_SAMPLING_END) {
                    bool jr = false;
                    ivj[4] /= c.I_SAMPLING_DURATION;
                    ivj[6] = ivj[4] - rm.b_a_ratio_E;
                    if (std::fabs(ivj[6] + 0.026) > 0.005) {
                        jr = true;
                        if (fic_trial < c.max_fic_trials) {
                            if (ivj[6] < -0.026) {
                                rj[2] -= ivj[5];
                                ivj[5] -= 0.001;
                                ivj[5] = std::fmax(ivj[5], 0.001);
                            } else {
                                rj[2] += ivj[5];
                            }
                        }
                    }
                    restart = restart || jr;
                }
            }
            if (t == c.I_SAMPLING_END) {
                if (restart) {
                    if (fic_trial < c.max_fic_trials) fic_trial++;
                    else { restart = false; adjust_fic = false; fic_failed = true; }
                } else {
                    adjust_fic = false;
                }
            }
        }
        bw_i++;
        if (restart) {  // bnm.cpp:386-434
            for (int j = 0; j < n; ++j) M::restart(&s[(size_t)j * M::NS], &iv[(size_t)j * M::NI], g, &r[(size_t)j * M::NR]);
            for (int j = 0; j < n; ++j) { bx[j] = 0.0; bf[j] = 1.0; bnu[j] = 1.0; bq[j] = 1.0; }
            reset_conn();
            bold_i = 0; states_i = 0; bw_i = 0; buff_idx = max_delay - 1; repeat = 0;
        }
    }
    if (M::POSTBW && c.do_fic) {  // rww.cpp:300-314 post_integration (rWW only)
        for (int j = 0; j < n; ++j) regional_out[2 * rstride + (size_t)sim * n + j] = r[(size_t)j * M::NR + 2];
        gints[0 * (size_t)c.n_sims + sim] = fic_trial;
        gbools[1 * (size_t)c.n_sims + sim] = fic_failed ? 1 : 0;
    }
    if (c.ext_out && !c.states_ts) {
        int pts = states_i - c.n_states_samples_remove;
        for (int v = 0; v < M::NS; ++v)
            for (int j = 0; j < n; ++j) st(v)[j] /= pts;
    }
    std::memcpy(bold_out, bold.data(), sizeof(double) * bold.size());
    if (c.do_fc) {
        fc_tril(bold.data(), n, c.n_vols_remove, c.bold_len, c.exc_interhemispheric, fc_out);
        if (c.do_fcd) fcd_tril(bold.data(), c, fcd_out);
    }
}

template <class M>
static void run_model(RunCfg &c, const cbnm_run_args *a, cbnm_outputs *o) {
    typename M::K m = M::make(c.dt);
    BWConst bwc = g_bw;
    bwc.dt = c.bw_dt;
    bwc.dt_itau = bwc.dt * bwc.itau;  // core.cpp:291-292
    make_noise(c, M::NN, a->force_reinit != 0);
    const size_t rsize = (size_t)M::NR * c.n_sims * c.nodes;
    std::vector<double> regional_in(a->regional_params, a->regional_params + rsize);
    if (M::NGB) std::memset(o->global_bools, 0, (size_t)M::NGB * c.n_sims);
    if (M::NGI) std::memset(o->global_ints, 0, sizeof(int32_t) * (size_t)M::NGI * c.n_sims);
    if constexpr (M::POSTBW) if (c.do_fic) {
        rww_prep_params(c, a, regional_in.data(), o->global_bools, m);
        std::memcpy(a->regional_params, regional_in.data(), sizeof(double) * rsize);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int sim = 0; sim < c.n_sims; ++sim) {
        simulate<M>(sim, c, a, regional_in.data(), a->regional_params, m, bwc,
                    o->sim_bold + (size_t)sim * c.bold_len * c.nodes,
                    c.do_fc ? o->sim_fc_trils + (size_t)sim * c.n_pairs : nullptr,
                    c.do_fcd ? o->sim_fcd_trils + (size_t)sim * c.n_window_pairs : nullptr,
                    o->sim_states, o->global_ints, o->global_bools);
    }
    if (a->noise_out) {
        std::memcpy(o->noise, g_noise.noise.data(), sizeof(double) * g_noise.noise.size());
        std::memcpy(o->shuffled_nodes, g_noise.sh_nodes.data(), sizeof(int32_t) * g_noise.sh_nodes.size());
        std::memcpy(o->shuffled_ts, g_noise.sh_ts.data(), sizeof(int32_t) * g_noise.sh_ts.size());
    }
}

struct ModelInfo { int ns, ng, nr, nn, ngb, ngi; bool mod; };
static bool model_info(const std::string &name, ModelInfo &mi) {
    if (name == "rWW") mi = {6, 1, 4, 2, 2, 1, true};
    else if (name == "WC") mi = {2, 1, 8, 2, 0, 0, false};
    else if (name == "JR") mi = {8, 1, 6, 1, 0, 0, false};
    else if (name == "Kuramoto") mi = {1, 1, 3, 1, 0, 0, false};
    else if (name == "rWWEx") mi = {3, 1, 3, 1, 0, 0, false};
    else return false;
    return true;
}

static int fill_sizes(const cbnm_run_args *a, RunCfg &c, cbnm_sizes *sz) {
    ModelInfo mi;
    if (!a || !a->model_name || !model_info(a->model_name, mi)) { g_err = "unknown model"; return CBNM_ERR_MODEL; }
    c.bw_dt = a->bw_dt / 1000.0;
    parse_config(c, a, std::string(a->model_name) == "rWW");
    setup_sizes(c, a);
    if (sz) {
        std::memset(sz, 0, sizeof(*sz));
        sz->n_global_params = mi.ng; sz->n_regional_params = mi.nr; sz->n_state_vars = mi.ns;
        sz->n_global_out_bool = mi.ngb; sz->n_global_out_int = mi.ngi;
        sz->bold_len = c.bold_len; sz->n_pairs = c.n_pairs; sz->n_windows = c.n_windows;
        sz->n_window_pairs = c.n_window_pairs; sz->states_len = c.states_len; sz->do_fc = c.do_fc;
        sz->do_fcd = c.do_fcd; sz->modifies_params = mi.mod && c.do_fic;
        sz->noise_repeats = c.noise_repeats; sz->noise_bw_it = c.noise_bw_it;
        sz->noise_size = (int64_t)c.nodes * c.noise_bw_it * c.inner_it * mi.nn;
    }
    return CBNM_OK;
}

}  // namespace orc

extern "C" {

int oracle_init(void) { orc::g_bw = orc::bw_defaults(0.001); return CBNM_OK; }

int oracle_set_const(const char *key, double value) {  // core.cpp:157-192
    std::string k = key;
    if (k == "k1") orc::g_bw.k1 = value;
    else if (k == "k2") orc::g_bw.k2 = value;
    else if (k == "k3") orc::g_bw.k3 = value;
    else if (k == "V_0") orc::g_bw.V_0 = value;
    orc::g_bw.V_0_k1 = orc::g_bw.V_0 * orc::g_bw.k1;
    orc::g_bw.V_0_k2 = orc::g_bw.V_0 * orc::g_bw.k2;
    orc::g_bw.V_0_k3 = orc::g_bw.V_0 * orc::g_bw.k3;
    return CBNM_OK;
}

int oracle_query_sizes(const cbnm_run_args *a, cbnm_sizes *sz) {
    try {
        orc::RunCfg c;
        return orc::fill_sizes(a, c, sz);
    } catch (const std::exception &e) {
        orc::g_err = e.what();
        return CBNM_ERR_CONFIG;
    }
}

int oracle_run_simulations(const cbnm_run_args *a, cbnm_outputs *o) {
    try {
        orc::RunCfg c;
        int st = orc::fill_sizes(a, c, nullptr);
        if (st) return st;
        std::string name = a->model_name;
        if (name == "rWW") orc::run_model<orc::ModelRWW>(c, a, o);
        else if (name == "WC") orc::run_model<orc::ModelWC>(c, a, o);
        else if (name == "JR") orc::run_model<orc::ModelJR>(c, a, o);
        else if (name == "Kuramoto") orc::run_model<orc::ModelKuramoto>(c, a, o);
        else if (name == "rWWEx") orc::run_model<orc::ModelRWWEx>(c, a, o);
        return CBNM_OK;
    } catch (const std::exception &e) {
        orc::g_err = e.what();
        return CBNM_ERR_CONFIG;
    }
}

const char *oracle_last_error(void) { return orc::g_err.c_str(); }

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
