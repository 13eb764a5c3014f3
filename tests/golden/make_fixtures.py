"""Extract the reference's golden vectors for this path into small fixtures.

Reads the reference tree (default /root/reference, read-only) and writes JSON
fixtures next to this script.  Every value is copied from the reference's own
test data, not recomputed:

  boys.json          tests/golden/boys/reference.json (F_m(T), SciPy hyp1f1)
  rys.json           tests/golden/rys/reference.json (roots/weights, orders 1-10)
  rhf_energies.json  tests/benchmarks/criterion/iqcp_iteration_counts.json, RHF
                     rows (the reference's own FP64 energies, 12 decimals) and
                     tests/benchmarks/wasm/results/determinism.json (IEEE hex)
  gradients.json     tests/golden/dft/gradient_validation{,_extended}.json, RHF
                     rows (PySCF analytic gradients, cart=True)
  presets.json       content/presets/systems/*.json (PySCF S, H, ERIs in the
                     eri_compressed layout, reference energies)
  fock_h2.json       the PySCF J/K/G/F/D values hard-coded in
                     crates/qc-core/src/scf/fock.rs:192-229

Usage: python tests/golden/make_fixtures.py [reference_root]
"""
import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = {}
    b = json.load(open(os.path.join(ref, "tests/golden/boys/reference.json")))
    out["boys.json"] = {"source": "tests/golden/boys/reference.json", "tolerance": float(b["tolerance"]),
                        "values": [[v["m"], v["T"], float(v["value"])] for v in b["values"]]}
    r = json.load(open(os.path.join(ref, "tests/golden/rys/reference.json")))
    out["rys.json"] = {"source": "tests/golden/rys/reference.json",
                       "cases": [{"n": c["order"], "T": c["T"], "roots": [float(x) for x in c["roots"]],
                                  "weights": [float(x) for x in c["weights"]], "F0": float(c["F_0_T"])}
                                 for c in r["test_cases"]]}
    it = json.load(open(os.path.join(ref, "tests/benchmarks/criterion/iqcp_iteration_counts.json")))
    det = json.load(open(os.path.join(ref, "tests/benchmarks/wasm/results/determinism.json")))
    out["rhf_energies.json"] = {
        "source": "tests/benchmarks/criterion/iqcp_iteration_counts.json (ScfConfig::tight + DIIS)",
        "rows": [{"molecule": x["molecule"], "basis": x["basis"], "n_basis": x["n_basis"], "energy": x["energy"],
                  "iterations": x["iterations"]} for x in it["results"] if x["method"] == "RHF"],
        "determinism_hex": {s["system"]: s["hex"] for s in det["systems"] if s["system"].startswith("RHF")},
    }
    rows = []
    for fn in ("gradient_validation.json", "gradient_validation_extended.json"):
        g = json.load(open(os.path.join(ref, "tests/golden/dft", fn)))
        for x in g["results"]:
            if x["method"] == "RHF":
                rows.append({"molecule": x["molecule"], "basis": x["basis"], "n_basis": x["n_basis"],
                             "energy": x["energy"], "gradient": x["gradient"], "source": "tests/golden/dft/" + fn})
    out["gradients.json"] = {"rows": rows}
    presets = []
    for fn in sorted(glob.glob(os.path.join(ref, "content/presets/systems/*.json"))):
        p = json.load(open(fn))
        presets.append({k: p[k] for k in ("system_id", "geometry", "basis_id", "nbf", "nelec", "e_nuc", "s_matrix",
                                           "h_core", "eri_compressed", "reference")})
    out["presets.json"] = {"source": "content/presets/systems", "systems": presets}
    # fock.rs PySCF H2 golden matrices: `const NAME: [f64; 4] = [...]`
    src = open(os.path.join(ref, "crates/qc-core/src/scf/fock.rs")).read()
    mats = {}
    for name, body in re.findall(r"const (PYSCF_\w+): \[f64; \d+\] = \[(.*?)\];", src, re.S):
        mats[name] = [float(v) for v in re.findall(r"[-+]?\d+\.\d+(?:[eE][-+]?\d+)?", body)]
    out["fock_h2.json"] = {"source": "crates/qc-core/src/scf/fock.rs:192-229", "matrices": mats}
    for name, data in out.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=0)
        print("wrote", name)


if __name__ == "__main__":
    main()
