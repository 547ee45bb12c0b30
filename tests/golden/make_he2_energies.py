"""Generate tests/golden/he2_631gss_sdci.json: an MO Hamiltonian and the energies
TigerCI printed for it, to pin sigma and the Davidson solve against the
reference's own regression runs.

Source runs (reference tree, tests/Tests/):
- Helium2_SDCI: He2 at 1.5 Angstrom, 6-31G** Cartesian (10 functions), 10
  orbitals, 2 inactive, 4 electrons, singlet, reference "22"
  (driver.sh input deck); printed reference energy and root-1 total energy.
- Helium2_SDCI_excited: the same deck with NUM ROOTS 2 (same Molden orbitals);
  printed root-1 and root-2 total energies.
- Helium2_ACPF: the same deck with ACPF FLAG 1 (same Molden orbitals); printed
  ACPF total energy.

The reference reads the orbitals from the Molden file and computes AO integrals
with libint (absent from its tree).  Here the AO integrals come from
oracle/gto.py (McMurchie-Davidson, restated), the MO coefficients from the
Molden file, and the Cholesky vectors of the MO (pq|rs) matrix from a pivoted
Cholesky decomposition to 1e-13.

Run once in an environment that has the reference tree:
    python tests/golden/make_he2_energies.py /path/to/reference
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import gto  # noqa: E402


def grab(path, pattern):
    out = []
    for ln in open(path):
        m = re.search(pattern, ln)
        if m:
            out.append(float(m.group(1)))
    return out


def main(ref_root):
    tdir = os.path.join(ref_root, "tests", "Tests")
    molden = os.path.join(tdir, "Helium2_SDCI", "Helium2_SDCI.molden")
    out1 = os.path.join(tdir, "Helium2_SDCI", "Helium2_SDCI.output")
    outx = os.path.join(tdir, "Helium2_SDCI_excited", "Helium2_SDCI_excited.output")
    outa = os.path.join(tdir, "Helium2_ACPF", "Helium2_ACPF.output")
    atoms, shells, C, ene, occ = gto.read_molden(molden)
    h, L, e_nuc, S = gto.mo_operator(atoms, shells, C)
    ortho = float(np.abs(C.T @ S @ C - np.eye(C.shape[1])).max())
    e_ref = grab(out1, r"the reference energy is \(elec \+ nuclear\) =\s*(-?\d+\.\d+)")
    e_sd = grab(out1, r"Root\s+1 total energy \(electronic \+ nuclear\) is :\s*(-?\d+\.\d+)")
    e_x = grab(outx, r"Root\s+\d+ total energy \(electronic \+ nuclear\) is :\s*(-?\d+\.\d+)")
    e_a = grab(outa, r"Root\s+1 total energy \(electronic \+ nuclear\) is :\s*(-?\d+\.\d+)")
    fixture = {
        "source": "tests/Tests/Helium2_SDCI (+ Helium2_SDCI_excited), reference tree",
        "deck": {"num_orbitals": 10, "num_inactive": 2, "num_active": 0, "num_elec": 4, "spin_mult": 1,
                 "refs": ["22"], "num_frozen": 0},
        "nuclear_repulsion": e_nuc,
        "mo_orthonormality_max_dev": ortho,
        "h": h.tolist(),
        "chol": L.tolist(),
        "reference_energy": e_ref[0],
        "sdci_root1": e_sd[0],
        "sdci_roots_excited_run": e_x,
        "acpf_root1": e_a[0],
        "reference_energy_tolerance_of_its_test": 1e-6,
    }
    path = os.path.join(HERE, "he2_631gss_sdci.json")
    with open(path, "w") as f:
        json.dump(fixture, f, indent=1)
    print(path, "nchol", L.shape[1], "E_nuc", e_nuc, "ortho", ortho, "energies", e_ref, e_sd, e_x)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("TIGERCI_REFERENCE"):
        sys.exit("usage: make_he2_energies.py <reference tree> (or set TIGERCI_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["TIGERCI_REFERENCE"])
