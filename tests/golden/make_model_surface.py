"""Records the parameter / variable surface of the reference's five models from
their code-generation recipes, for ``tests/test_model_surface.py``.

Run once, in a checkout that has the reference next to it:

    python tests/golden/make_model_surface.py /path/to/cubnm

It reads ``codegen/recipes/{rww,wc,jr,kuramoto,rwwex}.yaml`` as data (the
reference generates its model classes and kernels from them) and writes
``tests/golden/model_surface.json``: per model the state variables, global and
regional parameters (with their default values as written), noise terms,
global output flags and counters, the coupling and BOLD state variables, the
oscillator flag, the Python-side ``sel_state_var`` and the named constants.
"""
import json
import os
import sys

import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "model_surface.json")
RECIPES = ("rww", "wc", "jr", "kuramoto", "rwwex")


def main(ref_root):
    surface = {}
    for r in RECIPES:
        d = yaml.safe_load(open(os.path.join(ref_root, "codegen", "recipes", f"{r}.yaml")))
        by_type = {}
        for v in d["variables"]:
            by_type.setdefault(v["type"], []).append(v)
        names = lambda t: [v["name"] for v in by_type.get(t, [])]  # noqa: E731
        surface[d["model_name"]] = {
            "state_vars": names("state_var"),
            "global_params": names("global_param"),
            "regional_params": names("regional_param"),
            "regional_defaults": {v["name"]: (None if v.get("value") is None else str(v["value"]))
                                  for v in by_type.get("regional_param", [])},
            "noise": names("noise"),
            "global_out_bool": names("global_out_bool"),
            "global_out_int": names("global_out_int"),
            "conn_state_var": d["conn_state_var"],
            "bold_state_var": d["bold_state_var"],
            "is_osc": bool(d["is_osc"]),
            "sel_state_var": d.get("python_config", {}).get("sel_state_var"),
            "constants": {c["name"]: str(c["value"]) for c in d.get("constants", [])},
        }
    with open(OUT, "w") as f:
        json.dump(surface, f, indent=1, sort_keys=True)
    print(f"wrote {OUT}: {len(surface)} models")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUBNM_REFERENCE", "../cubnm"))
