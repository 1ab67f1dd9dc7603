"""Extract the reference's recorded golden values into committed fixtures.

Reads, as text, the reference's own test data and tests (this script is the
only place that touches the reference checkout; it is run by hand in the
build container, never on a GPU host):

* test/test_2d.jl:316-321 -- isentropic-vortex L2 errors and observed order;
* test/data/snapshot_fixture/{baseline,method}.json -- quant-suite case
  reports (1D smooth-order L2 errors, Sod and Shu-Osher step counts and
  extrema, and their scoring fields: shock thickness, overshoot, excess
  dissipation, L1 against the exact or reference density) recorded by
  Julia 1.11.7;
* test/data/shu_osher_ref.csv -- the self-generated Shu-Osher density
  reference (p=1, Ne=200, c_av=0.5, CFL 0.1).

Usage: python tests/golden/make_golden.py /path/to/reference
   or: FRFORGE_REFERENCE=/path/to/reference python tests/golden/make_golden.py
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    out = {"source": "RcktMan77/FRForge reference tests and fixtures"}
    txt = open(os.path.join(ref_root, "test", "test_2d.jl")).read()
    m = re.search(r'c\["l2_errors"\]\[1\],\s*([0-9.eE+-]+);\s*rtol\s*=\s*([0-9.eE+-]+)', txt)
    m2 = re.search(r'c\["l2_errors"\]\[2\],\s*([0-9.eE+-]+);', txt)
    m3 = re.search(r'c\["observed_orders"\]\[1\],\s*([0-9.eE+-]+);\s*rtol\s*=\s*([0-9.eE+-]+)', txt)
    out["vortex"] = {
        "file": "test/test_2d.jl:316-321",
        "p": 2, "n_list": [8, 16], "t_final": 0.5, "cfl": 0.08,
        "l2_errors": [float(m.group(1)), float(m2.group(1))], "rtol_l2": float(m.group(2)),
        "observed_order": float(m3.group(1)), "rtol_order": float(m3.group(2)),
    }
    snap = {}
    for name in ("baseline", "method"):
        d = json.load(open(os.path.join(ref_root, "test", "data", "snapshot_fixture", name + ".json")))
        cases = {}
        for c in d["cases"]:
            keep = {k: c[k] for k in ("name", "p", "capturing_method", "diverged", "nan_detected",
                                      "positivity_ok", "pass") if k in c}
            for k in ("l2_errors", "mesh_sizes", "observed_orders", "n_elements", "t_final", "shock_thickness",
                      "overshoot", "excess_dissipation", "l1_error_vs_reference"):
                if k in c:
                    keep[k] = c[k]
            if "method_params" in c:
                keep["method_params"] = c["method_params"]
            mt = c.get("metrics", {})
            for k in ("n_steps", "u_min", "u_max", "mass_change", "dt_fixed", "cfl", "n_elements_list",
                      "excess_dissipation_vs_exact", "excess_dissipation_vs_null", "l1_density_vs_exact"):
                if k in mt:
                    keep[k] = mt[k]
            cases[c["name"]] = keep
        snap[name] = {"julia_version": d.get("julia_version"), "git_commit": d.get("git_commit"),
                      "cases": cases}
    out["snapshot_fixture"] = snap
    rows = []
    for line in open(os.path.join(ref_root, "test", "data", "shu_osher_ref.csv")):
        if line.startswith("#") or not line.strip():
            continue
        a, b = line.strip().split(",")[:2]
        rows.append([float(a), float(b)])
    out["shu_osher_ref"] = {"file": "test/data/shu_osher_ref.csv", "p": 1, "ne": 200, "c_av": 0.5,
                            "cfl": 0.1, "t_final": 1.8, "x_rho": rows}
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_golden.json"))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FRFORGE_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py /path/to/reference (or set FRFORGE_REFERENCE)")
    main(ref)
