"""Seeded synthetic inputs with the shapes of the reference's data
(src/cubnm/data/hcp: SC nodes x nodes, zero diagonal, symmetric; BOLD nodes x
volumes).  They stand in for the HCP data the reference is measured on."""
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
