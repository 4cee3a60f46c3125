"""Seeded synthetic inputs with the shapes of the reference's data
(src/cubnm/data/hcp: SC nodes x nodes, zero diagonal, symmetric; BOLD nodes x
volumes; tract lengths nodes x nodes in mm).  They stand in for the HCP data
the reference is measured on.

``synthetic_args`` builds the 22 positional arguments of
``run_simulations`` for a seeded batch (the benchmark workloads and the
parity cases use it): parameters after ``SimGroup.N`` + ``_set_default_params``
(src/cubnm/sim/base.py:532-575) and the model_config strings of
``SimGroup._model_config`` (base.py:635-657, rww.py:120-133).
"""
import numpy as np


def synthetic_sc(nodes, density, seed):
    """Symmetric, zero diagonal, upper triangle kept by a seeded Bernoulli draw,
    lognormal(0, 1) weights, scaled so that the mean row sum is 1."""
    rng = np.random.default_rng(seed)
    mask = np.triu(rng.random((nodes, nodes)) < density, 1)
    w = np.where(mask, rng.lognormal(0.0, 1.0, (nodes, nodes)), 0.0)
    sc = w + w.T
    sc /= sc.sum(axis=1).mean()
    return sc


def synthetic_emp_bold(nodes, volumes, seed, rank=5, phi=0.8, white=0.3):
    """Rank-5 Gaussian loading on AR(1) latents (phi 0.8) plus 0.3 white noise,
    z-scored per node.  Shape (nodes, volumes)."""
    rng = np.random.default_rng(seed)
    load = rng.standard_normal((nodes, rank))
    lat = np.zeros((rank, volumes))
    for t in range(1, volumes):
        lat[:, t] = phi * lat[:, t - 1] + rng.standard_normal(rank)
    bold = load @ lat + white * rng.standard_normal((nodes, volumes))
    bold = (bold - bold.mean(axis=1, keepdims=True)) / bold.std(axis=1, keepdims=True)
    return bold


def synthetic_lengths(nodes, seed, radius_mm=70.0, tortuosity=1.3):
    """Tract lengths (mm) between ``nodes`` points drawn uniformly in a sphere of
    ``radius_mm``: Euclidean distance x ``tortuosity``, symmetric, zero diagonal.
    At 6 m/s (6 mm/ms) the longest delays are about 30 ms."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((nodes, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = d * radius_mm * rng.random(nodes)[:, None] ** (1.0 / 3.0)
    dist = np.linalg.norm(pts[:, None, :] - pts[None, :, :], axis=2) * tortuosity
    np.fill_diagonal(dist, 0.0)
    return dist


MODELS = {
    # name: (global names, regional names with defaults, state names, selected state)
    "rWW": (["G"], [("w_p", 1.4), ("J_N", 0.15), ("wIE", 1.0), ("sigma", 0.01)],
            ["I_E", "I_I", "r_E", "r_I", "S_E", "S_I"], "r_E"),
    "WC": (["G"], [("c_EE", 16), ("c_IE", 12), ("c_EI", 15), ("c_II", 3), ("P_E", 0.5), ("P_I", 0.0),
                   ("sigma_E", 5e-05), ("sigma_I", 5e-05)], ["E", "I"], "E"),
    "JR": (["G"], [("J", 135.0), ("a_1", 1.0), ("a_2", 0.8), ("a_3", 0.25), ("a_4", 0.25), ("sigma", 0.0001)],
           ["y0", "y1", "y2", "y3", "y4", "y5", "y1_y2", "s_y1_y2"], "y1_y2"),
    "Kuramoto": (["G"], [("init_theta", None), ("omega", np.pi), ("sigma", 0.17)], ["theta"], "theta"),
    "rWWEx": (["G"], [("w", 0.9), ("I0", 0.3), ("sigma", 0.001)], ["x", "r", "S"], "r"),
}


def base_config(window_size=10, window_step=2, bold_remove_s=30, exc_inter=False, drop_edges=True,
                noise_segment_s=30, do_fc=True, do_fcd=True):
    """SimGroup._model_config (base.py:635-657)."""
    return {
        "do_fc": str(int(do_fc)),
        "do_fcd": str(int(do_fcd)),
        "bold_remove_s": str(bold_remove_s),
        "exc_interhemispheric": str(int(exc_inter)),
        "window_size": str(window_size),
        "window_step": str(window_step),
        "drop_edges": str(int(drop_edges)),
        "noise_time_steps": str(int(noise_segment_s * 1000)),
        "verbose": "0",
        "progress_interval": "500",
    }


def model_config(model, do_fic=0, **kw):
    cfg = base_config(**kw)
    if model == "rWW":
        cfg.update({
            "do_fic": str(int(do_fic > 0)),
            "max_fic_trials": str(5 if do_fic == 2 else 0),
            "I_SAMPLING_START": "1000",
            "I_SAMPLING_END": "10000",
            "init_delta": "0.02",
            "fic_penalty_scale": "0.5",
        })
    elif model == "Kuramoto":
        cfg["random_init_theta"] = "1"
    return cfg


def default_params(model, N, nodes, G, do_fic=0, sim_seed=0, overrides=None):
    """param_lists after SimGroup.N setter + _set_default_params (base.py:532-575)."""
    gnames, rparams, _, _ = MODELS[model]
    overrides = overrides or {}
    glob = np.vstack([np.ascontiguousarray(np.broadcast_to(np.asarray(G, dtype=float), (N,)))[None, :]])
    regs = []
    for name, default in rparams:
        if name in overrides:
            val = np.broadcast_to(np.asarray(overrides[name], dtype=float), (N, nodes))
        elif model == "rWW" and name == "wIE" and do_fic:
            val = np.zeros((N, nodes))
        elif model == "Kuramoto" and name == "init_theta":
            rng = np.random.default_rng(sim_seed)
            val = np.tile(rng.uniform(0, 2 * np.pi, nodes), (N, 1))
        else:
            val = np.full((N, nodes), default, dtype=float)
        regs.append(np.ascontiguousarray(np.asarray(val, dtype=float).flatten()))
    return glob, np.vstack(regs)


def rww_grid(n_g=4, n_wp=5, n_jn=5):
    """The README grid: G in [0.001, 10] x w_p in [0, 2] x J_N in [0.001, 0.5]."""
    G, wp, jn = np.meshgrid(np.linspace(0.001, 10, n_g), np.linspace(0, 2, n_wp), np.linspace(0.001, 0.5, n_jn),
                            indexing="ij")
    return G.ravel(), wp.ravel(), jn.ravel()


def synthetic_args(model="rWW", N=100, nodes=100, duration_s=60, dt=0.1, seed=0, density=0.3, G=None, w_p=None,
                   J_N=None, do_fic=0, precision="fp64", sigma=0.01, window_size=10, window_step=2,
                   bold_remove_s=30, sim_seed=0, do_fc=True, do_fcd=True, force_reinit=False):
    sc = synthetic_sc(nodes, density, seed)
    rng = np.random.default_rng(seed + 1)
    if G is None:
        G = rng.uniform(0.001, 10, N)
    overrides = {}
    if model == "rWW":
        overrides["w_p"] = (rng.uniform(0, 2, N) if w_p is None else np.asarray(w_p))[:, None]
        overrides["J_N"] = (rng.uniform(0.001, 0.5, N) if J_N is None else np.asarray(J_N))[:, None]
        overrides["sigma"] = sigma
    glob, reg = default_params(model, N, nodes, G, do_fic=do_fic, sim_seed=sim_seed, overrides=overrides)
    cfg = model_config(model, do_fic, window_size=window_size, window_step=window_step,
                       bold_remove_s=bold_remove_s, do_fc=do_fc, do_fcd=do_fcd)
    cfg["precision"] = precision
    return (
        model, np.ascontiguousarray(sc.flatten())[None, :], np.zeros(N, dtype=np.intc),
        np.zeros(nodes * nodes), glob, reg, np.zeros(N), cfg, True, False, False, False, force_reinit, False,
        N, nodes, int(duration_s * 1000), 1000, 1000, sim_seed, dt, 1.0,
    )
