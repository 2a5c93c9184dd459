"""Extracts the reference crate's own printed outputs for inputs it builds
deterministically (no RNG stream involved), from its README smoke tables,
into ``reference_outputs.json``:

* ``stress_cpu 64`` (Docker smoke) rows of ``Small`` on the RNG-free profiles
  jordan_defective / sparse_structured / nearly_diagonal: rel_recon, orth_u,
  orth_v (README.md "Docker N=64 Smoke");
* ``stress_cpu 32 --auto-trace`` rows of the same profiles (Auto -> Small):
  rel_recon (README.md "Adaptive N=32 Smoke");
* ``compare/`` harness (run under ``--platform linux/amd64``, a host whose
  matrixmultiply kernel has no FMA): ``LieSvdSmall::solve`` orth_u and
  rel_recon of the named matrices (compare/README.md "Measured results");
* ``stress_cpu --joint`` Phase-JADE smoke (family built by
  ``print_joint_phase_jade_smoke``, src/bin/stress_cpu.rs:472-500) and
  ``--joint-svd`` smoke (``print_joint_svd_smoke``, :597-624).

Run here, where the reference checkout exists:

    python tests/golden/extract_reference_outputs.py /path/to/reference
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
RNG_FREE = ("jordan_defective", "sparse_structured", "nearly_diagonal")


def main(ref_root: str) -> None:
    lines = open(os.path.join(ref_root, "README.md"), encoding="utf-8").read().splitlines()
    out = {"source": "README.md of lie_cliffalg_analog_svd v0.44.0 (stress_cpu smoke tables)",
           "small_n64": [], "auto_n32": [], "jade": [], "joint_svd": []}
    section = None
    for no, line in enumerate(lines, 1):
        if line.startswith("### "):
            section = line[4:].strip()
        cells = [c.strip() for c in line.strip().strip("|").split("|")] if line.startswith("|") else []
        if section == "Docker `N=64` Smoke" and len(cells) == 6:
            prof = cells[0].strip("`")
            if prof in RNG_FREE and cells[1] == "`Small`":
                out["small_n64"].append({"n": 64, "profile": prof, "rel_recon": cells[3], "orth_u": cells[4],
                                         "orth_v": cells[5], "readme_line": no})
        if section == "Adaptive `N=32` Smoke" and len(cells) == 4:
            prof = cells[0].strip("`")
            if prof in RNG_FREE and cells[1] == "`Small`":
                out["auto_n32"].append({"n": 32, "profile": prof, "rel_recon": cells[2], "readme_line": no})
        m = re.fullmatch(r"\| (\d+) \| (\d+) \| ([0-9.e-]+) -> ([0-9.e-]+) \| (\d+) \| (\d+) \| [0-9.]+s \|",
                         line.strip())
        if m:
            row = {"n": int(m[1]), "family": int(m[2]), "initial_offdiag": m[3], "final_offdiag": m[4],
                   "sweeps": int(m[5]), "rotations": int(m[6]), "readme_line": no}
            prev = "\n".join(lines[max(0, no - 12):no])
            out["joint_svd" if "Joint SVD Offdiag" in prev else "jade"].append(row)
    out["compare_named"] = []
    names = {"Kahan": "kahan", "Pei (`alpha=0.01`)": "pei", "Vandermonde": "vandermonde", "Hilbert": "hilbert"}
    clines = open(os.path.join(ref_root, "compare", "README.md"), encoding="utf-8").read().splitlines()
    for no, line in enumerate(clines, 1):
        cells = [c.strip() for c in line.strip().strip("|").split("|")] if line.startswith("|") else []
        if len(cells) == 5 and cells[0] in names:
            out["compare_named"].append({"matrix": names[cells[0]], "n": int(cells[1]),
                                         "orth_u": cells[2].split("/")[0].strip(),
                                         "rel_recon": cells[3].split("/")[0].strip(),
                                         "compare_readme_line": no})
    assert len(out["compare_named"]) == 6, out["compare_named"]
    m = re.search(r"max relative error vs exact closed form = ([0-9.e-]+)`\s+at\s+`n=(\d+)`", "\n".join(clines))
    out["compare_pei_closed_form"] = {"n": int(m[2]), "alpha": 0.01, "max_rel": m[1]}
    assert len(out["small_n64"]) == 3 and len(out["auto_n32"]) == 3, out
    assert len(out["jade"]) == 4 and len(out["joint_svd"]) == 2, out
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LSVD_REFERENCE_ROOT", "."))
