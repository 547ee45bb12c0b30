"""The molecular front end, the sigma build and the Davidson solve against the
reference's own regression runs (tests/golden/reference_runs.json, written by
tests/golden/make_reference_runs.py from tests/Tests/<run>/ of the reference):

- He2 / 6-31G** SDCI, Methane / 6-31G** SDCI, Ammonia / 6-31G** SDCI
  (closed shell, one reference, Cartesian d);
- Acetylene / cc-pVDZ, three references 22222220, 22222211, 22222202
  (multireference with an open-shell singlet reference, Cartesian d);
- Ethylene / aug-cc-pVDZ triplet, 13 references over 4 active orbitals,
  6 frozen orbitals (open-shell high spin, pure d, CD THRESHOLD 1e-6).

Each run's Molden orbitals go through the library's own AO integrals, pivoted
Cholesky decomposition (at the run's CD THRESHOLD) and AO -> MO transform,
then the device sigma build and Davidson solve.  Checked against what the
reference printed: the number of Cholesky vectors (exactly), the closed-shell
reference energy, every root's total energy (within the 1e-6 Eh tolerance
of the reference's own test scripts, tests/Tests/*/driver.sh), and the final
wavefunction listing of each root (the ten largest |c| with their spin
function, arc weight, internal occupation and virtual orbitals; |c| within
the residual norm the reference's last iteration printed, since it stops on
the energy change with |Hc - Ec| of a few 1e-4 left), and for the one-root runs
the a posteriori block: c0^2 of the converged vector and the five corrections."""
import json
import os

import numpy as np
import pytest

import tigerci_b200 as T
from tigerci_b200 import molecule as M

HERE = os.path.dirname(os.path.abspath(__file__))
RUNS = json.load(open(os.path.join(HERE, "golden", "reference_runs.json")))["runs"]
IDS = [r["run"] for r in RUNS]

ENERGY_TOL = 1e-6      # the reference's regression-test tolerance (driver.sh)
REF_ENERGY_TOL = 1e-7  # closed-shell reference energy from the same orbitals and integrals


def _molecule(r):
    m = r["molecule"]
    return M.Molecule(m["charges"], np.array(m["coords_bohr"]), [tuple(s) for s in m["shells"]], m["pure_d"])


def _deck(r):
    d = r["deck"]
    return T.Deck(d["num_orbitals"], d["num_inactive"], d["num_active"], d["num_elec"], d["spin_mult"], d["refs"],
                  num_frozen=d["num_frozen"])


def _operator(r):
    it = M.Integrals(_molecule(r), r["cd_threshold"])
    h, L = it.mo_operator(np.array(r["mo_coefficients"]))
    return it, T.Operator(h, L, it.nuclear_repulsion)


@pytest.mark.parametrize("r", RUNS, ids=IDS)
def test_cholesky_vector_count_matches_reference(r):
    it = M.Integrals(_molecule(r), r["cd_threshold"])
    assert it.nchol == r["printed"]["nchol"]
    assert it.max_remaining <= r["cd_threshold"]


@pytest.mark.parametrize("r", [x for x in RUNS if len(x["deck"]["refs"]) == 1 and set(x["deck"]["refs"][0]) == {"2"}],
                         ids=lambda r: r["run"])
def test_closed_shell_reference_energy(r):
    it, op = _operator(r)
    nocc = len(r["deck"]["refs"][0])
    n = op.h.shape[0]
    idx = np.array([[max(p, q) * (max(p, q) + 1) // 2 + min(p, q) for q in range(n)] for p in range(n)])
    d = op.chol[idx[np.arange(nocc), np.arange(nocc)]]
    J = d @ d.T
    K = np.array([[op.chol[idx[i, j]] @ op.chol[idx[i, j]] for j in range(nocc)] for i in range(nocc)])
    e = 2.0 * np.trace(op.h[:nocc, :nocc]) + 2.0 * J.sum() - K.sum() + op.core_energy
    assert abs(e - r["printed"]["reference_energy"]) <= REF_ENERGY_TOL


def csf_descriptors(space: T.CsfSpace, nint: int, n_virt: int):
    """(spin function, arc weight, internal occupation, virtual 1, virtual 2) of every CSF, in the
    reference's listing convention: virtual orbitals numbered from 1 over all orbitals, the larger first,
    0 where there is none (valence CSF, or the second of an N-1 CSF / a doubly occupied virtual)."""
    c = space.counts()
    n = c["total_csfs"]
    sf = np.zeros(n, dtype=np.int64)
    arc = np.zeros(n, dtype=np.int64)
    v1 = np.zeros(n, dtype=np.int64)
    v2 = np.zeros(n, dtype=np.int64)
    occ = np.empty(n, dtype=object)
    nab = n_virt * (n_virt - 1) // 2
    ii, jj = np.tril_indices(n_virt, -1)  # i > j
    order = np.argsort(ii * (ii - 1) // 2 + jj)
    ii, jj = ii[order], jj[order]
    for kind, n_paths in ((0, c["paths_v"]), (1, c["paths_nm1"]), (2, c["paths_nm2"])):
        offs = space.index_vector(kind)
        offs_aa = space.index_vector(3) if kind == 2 else None
        for lex in range(1, n_paths + 1):
            o, info = space.path(kind, lex)
            s = "".join(str(int(x)) for x in o)
            blocks = []
            if offs[lex - 1] > 0:
                blocks.append(("ab" if kind == 2 else kind, offs[lex - 1] - 1, info["nsf"]))
            if kind == 2 and offs_aa[lex - 1] > 0:
                blocks.append(("aa", offs_aa[lex - 1] - 1, info["nsf_aa"]))
            for b, off, nsf in blocks:
                width = {0: 1, 1: n_virt, "aa": n_virt, "ab": nab}[b]
                for k in range(nsf):
                    sl = slice(off + k * width, off + (k + 1) * width)
                    sf[sl] = k + 1
                    arc[sl] = lex
                    occ[sl] = s
                    if b in (1, "aa"):
                        v1[sl] = nint + 1 + np.arange(n_virt)
                    elif b == "ab":
                        v1[sl] = nint + 1 + ii
                        v2[sl] = nint + 1 + jj
    return sf, arc, occ, v1, v2


@pytest.mark.gpu
@pytest.mark.parametrize("r", RUNS, ids=IDS)
def test_sdci_roots_and_wavefunction_listing_match_reference(r, need_gpu):
    it, op = _operator(r)
    deck = _deck(r)
    nroots = r["deck"]["num_roots"]
    sb = T.SigmaBuilder(deck, op, device=0, precision="fp64")
    e, vecs, _ = sb.davidson(nroots, 1e-8, 1e-12, want_vectors=True)
    sb.close()
    total = e + op.core_energy
    printed = r["printed"]["roots"][-nroots:]
    assert np.abs(total - np.array(printed)).max() <= ENERGY_TOL, (total, printed)
    sp = T.CsfSpace(deck)
    nint = deck.num_internal
    sf, arc, occ, v1, v2 = csf_descriptors(sp, nint, deck.num_external)
    for root, listing in enumerate(r["printed"]["listings"][-nroots:]):
        c = np.abs(vecs[root])
        top = np.argsort(-c)[:len(listing)]
        got = {(int(sf[i]), int(arc[i]), occ[i], int(v1[i]), int(v2[i])): c[i] for i in top}
        want = {(s, a, o, x, y): cf for cf, s, a, o, x, y in listing}
        # the ten largest coefficients of the two lists agree to print precision; ties at the cut-off
        # may swap entries of equal magnitude, so compare the entries both lists hold
        common = set(got) & set(want)
        assert len(common) >= len(want) - 1, (sorted(got.items()), sorted(want.items()))
        # the reference stops on the energy change, with |Hc - Ec| of a few 1e-4 left: its printed
        # coefficients are that far from the converged ones (plus the print's 6 digits)
        tol = r["printed"]["final_residual_norms"][root] + 5e-6
        for key in common:
            assert abs(got[key] - want[key]) <= tol, (key, got[key], want[key], tol)
    # a posteriori corrections of the one-root runs: c0^2 of the converged vector against the printed one
    # (the reference's vector is a residual norm away from converged, so c0^2 is about twice that away)
    blocks = r["printed"].get("aposteriori")
    if nroots == 1 and blocks:
        c0sq = sp.reference_weight(vecs[0])
        tol = 2.0 * r["printed"]["final_residual_norms"][0] + 1e-7
        assert abs(c0sq - blocks[0]["c0sq"]) <= tol, (c0sq, blocks[0]["c0sq"], tol)
        n_corr = deck.num_elec - 2 * deck.num_frozen
        got = T.aposteriori(c0sq, float(total[0]) - r["printed"]["reference_energy"], n_corr)
        e_corr = abs(r["printed"]["roots"][-1] - r["printed"]["reference_energy"])
        for name, v in got.items():
            assert abs(v - blocks[0][name]) <= e_corr * tol + ENERGY_TOL, (name, v, blocks[0][name])


@pytest.mark.gpu
@pytest.mark.parametrize("r", [x for x in RUNS if x["run"] in ("Methane_SDCI", "Acetylene_SuperMol")],
                         ids=lambda r: r["run"])
def test_mixed_form_roots_within_one_microhartree(r, need_gpu):
    it, op = _operator(r)
    deck = _deck(r)
    sb = T.SigmaBuilder(deck, op, device=0, precision="tf32x3")
    e, _, _ = sb.davidson(r["deck"]["num_roots"], 1e-8, 1e-12)
    sb.close()
    printed = r["printed"]["roots"][-r["deck"]["num_roots"]:]
    assert np.abs(e + op.core_energy - np.array(printed)).max() <= ENERGY_TOL
