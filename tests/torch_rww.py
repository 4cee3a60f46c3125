"""FP64 torch restatement of the rWW + Balloon-Windkessel forward pass, for
checking the adjoint gradients with torch autograd (test infrastructure).

It follows the reference's CPU loop (src/ext/bnm.cpp:69-522: inner Euler steps
of the node model, one Balloon-Windkessel step per bw_dt, BOLD every TR) with
the model of src/ext/models/rww.cpp:194-232 and bw.cpp:24-35, vectorised over
simulations and nodes, with the noise of a given run (_noise, _shuffled_nodes,
_shuffled_ts) indexed as bnm.cu:311-316 does.  Small sizes only: every step is
a handful of torch ops.
"""
import numpy as np
import torch

RWW = dict(a_E=310.0, b_E=125.0, d_E=0.16, a_I=615.0, b_I=177.0, d_I=0.087, w_II=1.0,
           w_E__I_0=1.0 * 0.382, w_I__I_0=0.7 * 0.382, gamma_E=0.641 / 1000.0, gamma_I=1.0 / 1000.0,
           tau_E=100.0, tau_I=10.0)
BW = dict(rho=0.34, alpha=0.32, tau=0.98, y=1.0 / 0.41, kappa=1.0 / 0.65, V_0=2.0)


def noise_steps(noise, sh_nodes, sh_ts, nodes, bw_it, inner_it, n_noise=2):
    """Noise of every integration step: [bw_it * inner_it, nodes, n_noise]."""
    noise_bw_it = sh_ts.shape[1]
    out = np.empty((bw_it * inner_it, nodes, n_noise))
    j = np.arange(nodes)
    for bw_i in range(bw_it):
        rep = bw_i // noise_bw_it
        ts = sh_ts[rep, bw_i % noise_bw_it]
        sj = sh_nodes[rep, j]
        for inner in range(inner_it):
            base = ((ts * inner_it + inner) * nodes + sj) * n_noise
            for q in range(n_noise):
                out[bw_i * inner_it + inner, :, q] = noise[base + q]
    return out


def bold_rww(G, w_p, J_N, wIE, sigma, sc, noise, dt=0.1, bw_dt_s=0.001, bold_tr_iters=1000, inner_it=10):
    """BOLD [N, T, n] (float64) of rWW simulations; G [N], w_p, J_N, wIE, sigma [N, n];
    sc [n, n] (row = source); noise [steps, n, 2] (shared by all simulations)."""
    m = RWW
    sqrt_dt = float(np.sqrt(dt))
    dt_gE, dt_iE = dt * m["gamma_E"], dt / m["tau_E"]
    dt_gI, dt_iI = dt * m["gamma_I"], dt / m["tau_I"]
    sc = torch.as_tensor(sc, dtype=torch.float64)
    nz = torch.as_tensor(noise, dtype=torch.float64)
    N, n = w_p.shape
    SE = torch.full((N, n), 0.001, dtype=torch.float64)
    SI = torch.full((N, n), 0.001, dtype=torch.float64)
    x = torch.zeros((N, n), dtype=torch.float64)
    f = torch.ones((N, n), dtype=torch.float64)
    nu = torch.ones((N, n), dtype=torch.float64)
    q = torch.ones((N, n), dtype=torch.float64)
    b = BW
    ialpha, itau = 1.0 / b["alpha"], 1.0 / b["tau"]
    k1, k2, k3 = 7 * b["rho"], 2.0, 2 * b["rho"] - 0.2
    bw_it = nz.shape[0] // inner_it
    out = []

    def rate(xv, d):
        return xv / (1 - torch.exp(-d * xv))

    for bw_i in range(bw_it):
        for inner in range(inner_it):
            k = bw_i * inner_it + inner
            inp = SE @ sc  # in_j = sum_k SC[k][j] S_E,k
            IE = m["w_E__I_0"] + w_p * J_N * SE + inp * G[:, None] * J_N - wIE * SI
            II = m["w_I__I_0"] + J_N * SE - m["w_II"] * SI
            rE = rate(m["a_E"] * IE - m["b_E"], m["d_E"])
            rI = rate(m["a_I"] * II - m["b_I"], m["d_I"])
            SE = torch.clamp(SE + (nz[k, :, 0] * sigma * sqrt_dt + dt_gE * ((1 - SE) * rE) - dt_iE * SE), 0, 1)
            SI = torch.clamp(SI + (nz[k, :, 1] * sigma * sqrt_dt + dt_gI * rI - dt_iI * SI), 0, 1)
        x = x + bw_dt_s * (SE - b["kappa"] * x - b["y"] * (f - 1.0))
        f_new = f + bw_dt_s * x
        nu_new = nu + bw_dt_s * itau * (f - nu ** ialpha)
        q = q + bw_dt_s * itau * (f * (1.0 - (1.0 - b["rho"]) ** (1.0 / f)) / b["rho"] - nu_new ** ialpha * q / nu_new)
        nu, f = nu_new, f_new
        if (bw_i + 1) % bold_tr_iters == 0:
            out.append(b["V_0"] * (k1 * (1 - q) + k2 * (1 - q / nu) + k3 * (1 - nu)))
    return torch.stack(out, dim=1)
