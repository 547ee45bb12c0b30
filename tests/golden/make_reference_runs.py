"""Generate tests/golden/reference_runs.json: the inputs and the printed results
of the reference's own regression runs, for pinning the molecular front end
(AO integrals, Cholesky decomposition, AO -> MO transform), the sigma build
and the Davidson solve against TigerCI itself.

For each run (tests/Tests/<run>/ in the reference tree) the fixture holds:
- the molecule, basis and MO coefficients of its Molden file (read with
  oracle/gto.py's Molden reader; coordinates in bohr);
- the input deck as the run's output echoes it (orbital counts, electrons,
  spin, reference occupations, CD THRESHOLD, tolerances, roots);
- what the run printed: "Number of cholesky vectors", "the reference energy
  is (elec + nuclear)", every "Root k total energy", and the final
  "Best guess wavefunction summary" of each root (coefficient, spin function,
  arc weight, internal occupation, virtuals) with the residual norm |Hc - Ec|
  of the last iteration (the run stops on the energy change, so its printed
  coefficients carry an error of that order).

Run once in an environment that has the reference tree:
    python tests/golden/make_reference_runs.py <reference tree>
(or set TIGERCI_REFERENCE).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import gto  # noqa: E402

RUNS = [
    ("Helium2_SDCI", "Helium2_SDCI"),
    ("Methane_SDCI", "Methane_SDCI"),
    ("Ammonia_SDCI", "Ammonia_SDCI"),
    ("Acetylene_SuperMol", "Acetylene_SuperMol"),
    ("Ethylene_HighSpin", "Ethylene_HighSpin"),
]


def keywords(lines):
    """The Keyword / Value table at the top of an output."""
    out, cur = {}, None
    start = next(i for i, ln in enumerate(lines) if ln.startswith("Keyword") and "Value" in ln) + 2
    for ln in lines[start:]:
        if ln.startswith("!") or ln.startswith("*"):
            break
        if not ln.strip():
            continue
        if ln[:40].strip():
            cur = ln[:40].strip()
            out[cur] = [ln[40:].strip()]
        else:
            out[cur].append(ln[40:].strip())
    return out


def listings(lines):
    """Last final-wavefunction listing of every root: [(coef, spin_func, arc_weight, occ, v1, v2)]."""
    res = {}
    for i, ln in enumerate(lines):
        m = re.search(r"Final wavefunction output for root =\s*(\d+)", ln)
        if not m:
            continue
        root = int(m.group(1))
        rows = []
        k = i + 1
        while k < len(lines) and "Coefficient" not in lines[k]:
            k += 1
        k += 1
        while k < len(lines) and "Weight of all" not in lines[k] and "Final wavefunction" not in lines[k]:
            t = lines[k].split()
            if len(t) == 7 and t[4] == "|":
                rows.append([abs(float(t[0])), int(t[1]), int(t[2]), t[3], int(t[5]), int(t[6])])
            k += 1
        res[root] = rows
    return [res[r] for r in sorted(res)]


def final_residuals(lines):
    """|Hc - Ec| of the last Davidson iteration of every root (the iteration tables' rows)."""
    res = {}
    for ln in lines:
        m = re.match(r"\s+(\d+)\s+(\d+)\s+(-?\d\.\d+D[+-]\d+)\s+(\d\.\d+D[+-]\d+)\s+(\d\.\d+D[+-]\d+)\s+[\d.]+\s*$", ln)
        if m:
            res[int(m.group(2))] = float(m.group(4).replace("D", "E"))
    return [res[r] for r in sorted(res)]


def aposteriori(lines):
    """The 'A Posteriori Corrections' block (one-root runs): [{"c0sq": x, name: value, ...}] for the two
    definitions of c0^2 it prints (sum of reference c^2, then <ref|ci>^2)."""
    out, cur = [], None
    names = {"Davidson": "davidson", "Renormalized Davidson": "renormalized_davidson",
             "Davidson-Silver": "davidson_silver", "Meissner": "meissner", "Pople": "pople"}
    for ln in lines:
        m = re.match(r"\s*Define c_0\^2 = .*=\s*(-?\d\.\d+E[+-]\d+)", ln)
        if m:
            cur = {"c0sq": float(m.group(1))}
            out.append(cur)
            continue
        m = re.match(r"\s*(Davidson|Renormalized Davidson|Davidson-Silver|Meissner|Pople)\s+(-?\d\.\d+E[+-]\d+)\s*$", ln)
        if m and cur is not None:
            cur[names[m.group(1)]] = float(m.group(2))
    return out


def grab(lines, pattern):
    return [float(m.group(1)) for ln in lines for m in [re.search(pattern, ln)] if m]


def main(ref_root):
    tdir = os.path.join(ref_root, "tests", "Tests")
    runs = []
    for run, stem in RUNS:
        out = open(os.path.join(tdir, run, stem + ".output")).read().splitlines()
        molden = os.path.join(tdir, run, stem + ".molden")
        kw = keywords(out)
        atoms, shells, C, ene, occ = gto.read_molden(molden)
        centres = [a[1] for a in atoms]
        shell_rows = []
        for centre, L, ex, cf in shells:
            idx = next(i for i, c in enumerate(centres) if c == centre)
            shell_rows.append([idx, L, ex, cf])
        nchol = grab(out, r"Number of cholesky vectors\s*[=.]*\s*(\d+)")
        runs.append({
            "run": run,
            "source": f"tests/Tests/{run}/{stem}.output and {stem}.molden",
            "molecule": {"charges": [a[0] for a in atoms], "coords_bohr": centres, "shells": shell_rows,
                         "pure_d": gto.molden_is_pure(molden)},
            "mo_coefficients": C.tolist(),
            "deck": {
                "num_orbitals": int(kw["NUMBER OF ORBITALS"][0]),
                "num_frozen": int(kw["NUMBER OF FROZEN ORBITALS"][0]),
                "num_inactive": int(kw["NUMBER OF INACTIVE ORBITALS"][0]),
                "num_active": int(kw["NUMBER OF ACTIVE ORBITALS"][0]),
                "num_elec": int(kw["NUMBER OF ELECTRONS"][0]),
                "spin_mult": int(kw["SPIN MULTIPLICITY"][0]),
                "refs": [r for r in kw["REFERENCE OCCUPATIONS"] if r],
                "num_roots": int(kw["NUM ROOTS"][0]),
            },
            "cd_threshold": float(kw["CD THRESHOLD"][0]),
            "energy_tolerance": float(kw["ENERGY TOLERANCE"][0]),
            "residual_tolerance": float(kw["RESIDUAL TOLERANCE"][0]),
            "printed": {
                "nchol": int(nchol[0]),
                "reference_energy": grab(out, r"the reference energy is \(elec \+ nuclear\) =\s*(-?\d+\.\d+)")[0],
                "roots": grab(out, r"Root\s+\d+ total energy \(electronic \+ nuclear\) is :\s*(-?\d+\.\d+)"),
                "listings": listings(out),
                "final_residual_norms": final_residuals(out),
                "aposteriori": aposteriori(out),
            },
        })
    path = os.path.join(HERE, "reference_runs.json")
    with open(path, "w") as f:
        json.dump({"runs": runs}, f)
    for r in runs:
        print(r["run"], r["deck"], "nchol", r["printed"]["nchol"], "roots", r["printed"]["roots"],
              "listing rows", [len(x) for x in r["printed"]["listings"]])
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("TIGERCI_REFERENCE"):
        sys.exit("usage: make_reference_runs.py <reference tree> (or set TIGERCI_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["TIGERCI_REFERENCE"])
