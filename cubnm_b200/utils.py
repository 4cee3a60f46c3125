"""Empirical FC/FCD and goodness-of-fit helpers.

``calculate_fc`` / ``calculate_fcd`` restate the reference's empirical
helpers (src/cubnm/utils.py:162-304) in numpy: they run once per fit on the
host.  ``fc_corr_device`` / ``fcd_ks_device`` replace the reference's CuPy and
numba kernels (utils.py:306-507) with this library's CUDA kernels.
"""
import ctypes as C

import numpy as np
import scipy.stats

from ._lib import lib, check


def get_bw_params(src):
    """Balloon-Windkessel k1..k3 (src/cubnm/utils.py:130-160)."""
    if src == "friston2003":
        rho = 0.34
        return {"k1": 7 * rho, "k2": 2.0, "k3": 2 * rho - 0.2}
    if src == "heinzle2016-3T":
        return {"k1": 3.72, "k2": 0.527, "k3": 0.53}
    raise ValueError(f"Unknown BW parameters source: {src}")


def calculate_fc(bold, exc_interhemispheric=False, return_tril=True):
    """FC of an empirical BOLD array (nodes, volumes); utils.py:162-201."""
    bold = np.array(bold, dtype=float, copy=True)
    outlier_vols = bold.sum(axis=0) == 0
    bold[:, ~outlier_vols] = scipy.stats.zscore(bold[:, ~outlier_vols], axis=1)
    fc = np.corrcoef(bold)
    if exc_interhemispheric:
        rh = bold.shape[0] // 2
        fc[:rh, rh:] = np.nan
        fc[rh:, :rh] = np.nan
    if return_tril:
        fc = fc[np.tril_indices(fc.shape[0], -1)]
        fc = fc[~np.isnan(fc)]
    return fc


def calculate_fcd(bold, window_size, window_step, drop_edges=True, outlier_threshold=0.5,
                  exc_interhemispheric=False, return_tril=True, return_dfc=False):
    """FCD of an empirical BOLD array (nodes, volumes); utils.py:204-304."""
    assert window_size % 2 == 0, "Window size must be even"
    bold = np.array(bold, dtype=float, copy=True)
    outlier_vols = bold.sum(axis=0) == 0
    bold[:, ~outlier_vols] = scipy.stats.zscore(bold[:, ~outlier_vols], axis=1)
    nodes, n_vols = bold.shape
    if drop_edges:
        first_center = int(window_size / 2)
        last_center = n_vols - 1 - int(window_size / 2)
    else:
        first_center, last_center = 0, n_vols - 1
    window_fc_trils, window_fcs = [], []
    center = first_center
    while center <= last_center:
        start = max(0, center - int(window_size / 2))
        end = min(n_vols - 1, center + int(window_size / 2))
        wb = bold[:, start:end + 1]
        center += window_step
        if (wb.sum(axis=0) == 0).mean() > outlier_threshold:
            continue
        wfc = np.corrcoef(wb)
        if exc_interhemispheric:
            rh = nodes // 2
            wfc[:rh, rh:] = np.nan
            wfc[rh:, :rh] = np.nan
        window_fcs.append(wfc[:, :, None])
        t = wfc[np.tril_indices(nodes, -1)]
        window_fc_trils.append(t[~np.isnan(t)][:, None])
    window_fc_trils = np.concatenate(window_fc_trils, axis=1)
    fcd = np.corrcoef(window_fc_trils.T)
    if return_tril:
        fcd = fcd[np.tril_indices(fcd.shape[0], -1)]
    if return_dfc:
        return fcd, np.concatenate(window_fcs, axis=2)
    return fcd


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def gof(sim_fc_trils=None, emp_fc_tril=None, sim_fcd_trils=None, emp_fcd_tril=None, terms=None):
    """All goodness-of-fit terms for a batch in one call (GPU).

    Returns a dict with the positive distances/correlations
    ``fc_corr``, ``fc_diff``, ``fc_normec``, ``fcd_ks`` (each (N,)).
    """
    terms = set(terms or ["fc_corr", "fc_diff", "fc_normec", "fcd_ks"])
    out = {}
    sf = ef = sd = ed = None
    N, P, M1, M2 = 0, 0, 0, 0
    if sim_fc_trils is not None and emp_fc_tril is not None:
        sf = np.require(sim_fc_trils, np.float64, ["C"])
        ef = np.require(emp_fc_tril, np.float64, ["C"])
        N, P = sf.shape
    if sim_fcd_trils is not None and emp_fcd_tril is not None:
        sd = np.require(sim_fcd_trils, np.float64, ["C"])
        ed = np.require(emp_fcd_tril, np.float64, ["C"])
        N, M1 = sd.shape
        M2 = ed.shape[0]
    for t in ["fc_corr", "fc_diff", "fc_normec"]:
        if t in terms and sf is not None:
            out[t] = np.empty(N)
    if "fcd_ks" in terms and sd is not None:
        out["fcd_ks"] = np.empty(N)
    if N == 0:
        return out
    check(lib().cbnm_gof(_dp(sf), N, P, _dp(ef), _dp(sd), M1, _dp(ed), M2, _dp(out.get("fc_corr")),
                         _dp(out.get("fc_diff")), _dp(out.get("fc_normec")), _dp(out.get("fcd_ks"))))
    return out


def fc_corr_device(sim_fc_trils, emp_fc_tril, usable_mem=None):
    """Pearson r of each simulated FC row with the empirical FC (utils.py:416-507)."""
    return gof(sim_fc_trils=sim_fc_trils, emp_fc_tril=emp_fc_tril, terms=["fc_corr"])["fc_corr"]


def fcd_ks_device(sim_fcd_trils, emp_fcd_tril, usable_mem=None):
    """Two-sample KS distance of each simulated FCD row to the empirical FCD (utils.py:306-414)."""
    return gof(sim_fcd_trils=sim_fcd_trils, emp_fcd_tril=emp_fcd_tril, terms=["fcd_ks"])["fcd_ks"]
