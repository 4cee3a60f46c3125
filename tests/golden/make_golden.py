"""Builds the golden fixtures used by the parity tests.

Run once, in a checkout that has the reference next to it:

    python tests/golden/make_golden.py /path/to/cubnm

It reads, as data only (nothing of the reference is imported or executed):

* ``tests/expected/sim/{rWW,WC,JR,Kuramoto,rWWEx}.pkl.gz`` -- the reference's own
  stored single-simulation outputs (``tests/sim/gen_expected.py:18-56`` made them;
  ``tests/sim/test.py:64-111`` checks them at ``atol=1e-6``);
* ``src/cubnm/data/hcp/sc/group-train706/ctx_parc-schaefer-100_desc-{strength,length}.npz``
  -- the structural connectome those outputs were simulated on.

The strength matrix is normalised the way ``datasets.load_sc`` does it
(``src/cubnm/datasets.py:70-75``: divide by ``mean * 100``).  The run
configuration of every stored key is the one of ``SimGroup._get_test_instance``
(``src/cubnm/sim/base.py:1267-1301``): 60 s, TR 1 s, window 10 s, step 2 s,
G = 0.5, model defaults otherwise; dt = 0.1 ms without delay and 1.0 ms with
delay (velocity 0.5 m/s); rWW ``do_fic`` 0 = off, 1 = analytical, 2 = analytical
+ numerical with ``max_fic_trials = 5`` (``src/cubnm/sim/rww.py:323-345``).

Output: ``tests/golden/sim_golden.npz`` with arrays named
``<model>|<key>|<field>`` plus ``sc_strength`` and ``sc_length``.
"""
import gzip
import os
import pickle
import sys

import numpy as np

MODELS = ["rWW", "WC", "JR", "Kuramoto", "rWWEx"]
FIELDS = ["sim_bold", "sim_fc_trils", "sim_fcd_trils", "sim_sel_state"]


def main(ref_root):
    out = {}
    sc_dir = os.path.join(ref_root, "src", "cubnm", "data", "hcp", "sc", "group-train706")
    sc = np.load(os.path.join(sc_dir, "ctx_parc-schaefer-100_desc-strength.npz"))["arr_0"].astype(np.float64)
    sc /= sc.mean() * 100
    out["sc_strength"] = sc
    out["sc_length"] = np.load(os.path.join(sc_dir, "ctx_parc-schaefer-100_desc-length.npz"))["arr_0"].astype(np.float64)
    for model in MODELS:
        path = os.path.join(ref_root, "tests", "expected", "sim", f"{model}.pkl.gz")
        with gzip.open(path, "rb") as f:
            data = pickle.load(f)
        for key, fields in data.items():
            for field in FIELDS:
                out[f"{model}|{key}|{field}"] = np.asarray(fields[field], dtype=np.float64)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sim_golden.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} with {len(out)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path to the reference checkout (amnsbr/cubnm)>")
    main(sys.argv[1])
