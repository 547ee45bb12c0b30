"""Generate tests/golden/csf_counts.json from TigerCI's recorded regression
outputs (tests/Tests/*/*.output in the reference tree).

Each TigerCI run echoes its input parameters and reference occupations
(fetch_globals.f90) and then prints the CSF-space statistics written by
index_vector_internal (graph_mod.f90:1007-1589).  These counts are
known-answer data for the graph, tree search and index vectors: they depend
only on orbital counts, electrons, spin and references.  For local runs
(NONLOCAL F) the N-1/N-2 counts also depend on molecular geometry, so only the
valence counts and the maximum open-shell count are kept.

Run once in an environment that has the reference tree:
    python tests/golden/make_golden.py /path/to/reference
"""
import glob
import json
import os
import re
import sys

INT_KEYS = {
    "NUMBER OF ORBITALS": "num_orbitals",
    "NUMBER OF FROZEN ORBITALS": "num_frozen",
    "NUMBER OF INACTIVE ORBITALS": "num_inactive",
    "NUMBER OF ACTIVE ORBITALS": "num_active",
    "SPIN MULTIPLICITY": "spin_mult",
    "NUMBER OF ELECTRONS": "num_elec",
    "NUMBER OF REFERENCES": "num_ref",
}


def parse_output(path):
    lines = open(path, errors="replace").read().splitlines()
    runs = []
    cur = None
    section = None
    i = 0
    while i < len(lines):
        ln = lines[i]
        if "TIGER CI IS USING THE FOLLOWING INPUT PARAMETERS" in ln:
            cur = {"source": None, "counts": {"valence": {}, "nm1": {}, "nm2": {}}}
            runs.append(cur)
            section = "valence"
        elif cur is not None:
            m = re.match(r"^ (NUMBER OF [A-Z ]+?|SPIN MULTIPLICITY)\s{2,}(-?\d+)\s*$", ln)
            if m and m.group(1).strip() in INT_KEYS:
                cur[INT_KEYS[m.group(1).strip()]] = int(m.group(2))
            m = re.match(r"^ NONLOCAL\s+([TF])\s*$", ln)
            if m:
                cur["nonlocal"] = m.group(1) == "T"
            m = re.match(r"^ (REFERENCE|VALENCE) CI FLAG\s+([TF])\s*$", ln)
            if m and m.group(2) == "T":
                cur["restricted_ci"] = True
            m = re.search(r"Number of (.+?) thrown out by WP\.+\s+(\d+)", ln)
            if m and "total_csfs" not in cur:
                # only the first CSF space of a run counts
                cur["wp_thrown"] = cur.get("wp_thrown", 0) + int(m.group(2))
            if re.match(r"^\s+Reference #\s+\d+", ln):
                occ = lines[i + 1].split()
                cur.setdefault("refs", []).append("".join(occ))
                i += 1
            m = re.search(r"Maximum number of open shells allowed:\s+(\d+)", ln)
            if m and "open_shells" not in cur:
                cur["open_shells"] = int(m.group(1))
            m = re.search(r"For\s+(\d+) singles there are\s+(\d+) spinfunctions and\s+(\d+) configurations", ln)
            if m and "total_csfs" not in cur:
                cur["counts"][section][m.group(1)] = [int(m.group(2)), int(m.group(3))]
            m = re.search(r"Number of valence CSFs:\s+(\d+)", ln)
            if m and "num_valence" not in cur:
                cur["num_valence"] = int(m.group(1))
                section = "nm1"
            m = re.search(r"Number of N-1 states:\s+(\d+)", ln)
            if m and "num_nm1" not in cur:
                cur["num_nm1"] = int(m.group(1))
                section = "nm2"
            m = re.search(r"Number of N-2 states:\s+(\d+)", ln)
            if m and "num_nm2" not in cur:
                cur["num_nm2"] = int(m.group(1))
            for key, pat in (
                ("total_configurations", r"Total number of configurations\.+\s+(\d+)"),
                ("kept", r"Number of configurations kept\.+\s+(\d+)"),
                ("removed", r"Number of configurations removed\.+\s+(\d+)"),
                ("total_csfs", r"Total number of full CSFs \.+\s+(\d+)"),
            ):
                m = re.search(pat, ln)
                if m and key not in cur:
                    cur[key] = int(m.group(1))
        i += 1
    out = []
    for r in runs:
        if "num_valence" not in r or "refs" not in r:
            continue
        nint = r.get("num_inactive", 0) + r.get("num_active", 0)
        r["refs"] = [x[:nint] for x in r["refs"]]
        r.setdefault("num_frozen", 0)
        r.setdefault("num_active", 0)
        r["source"] = os.path.relpath(path, os.path.dirname(os.path.dirname(os.path.dirname(path))))
        if r.pop("restricted_ci", False):
            continue
        if not r.get("nonlocal", False) or r.get("wp_thrown", 0) > 0:
            r["nonlocal"] = False
            for k in ("num_nm1", "num_nm2", "total_csfs", "kept", "removed"):
                r.pop(k, None)
            r["counts"].pop("nm1")
            r["counts"].pop("nm2")
        out.append(r)
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TIGERCI_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference tree> (or set TIGERCI_REFERENCE)")
    runs = []
    seen = set()
    for p in sorted(glob.glob(os.path.join(ref, "tests", "Tests", "*", "*.output"))):
        for r in parse_output(p):
            key = json.dumps({k: v for k, v in r.items() if k != "source"}, sort_keys=True)
            if key in seen:
                continue
            seen.add(key)
            r["source"] = "tests/Tests/" + os.path.relpath(p, os.path.join(ref, "tests", "Tests"))
            runs.append(r)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csf_counts.json")
    with open(dst, "w") as f:
        json.dump(runs, f, indent=1, sort_keys=True)
    print(f"wrote {len(runs)} runs to {dst}")


if __name__ == "__main__":
    main()
