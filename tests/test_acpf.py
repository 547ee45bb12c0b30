"""ACPF-type functionals (acpf_driver, davidson_liu_gen_eig, gtimesc.f90).

- The metric's CSF classes and values (tci_acpf_gdiag) against a restatement of
  build_g_diagonal / get_gvalues over the path occupations, for every small test
  space and every functional.
- The He2 / 6-31G** ACPF energy that TigerCI printed (Helium2_ACPF run, fixture
  tests/golden/he2_631gss_sdci.json): the dense generalized eigenproblem
  (H - E_ref) c = lambda G c of the oracle reproduces it (observed 1.1e-9 Eh), and
  the device solve (tci_davidson_gen) must too: 1e-8 Eh in FP64, 1 uEh mixed.
"""
import json
import os

import numpy as np
import pytest

import tigerci_b200 as T
from cases import SMALL_CASES, case_id, product_deck

FIX = os.path.join(os.path.dirname(__file__), "golden", "he2_631gss_sdci.json")


def _gvalues(flag, n_corr, custom=0.0):  # get_gvalues (gtimesc.f90:316-378)
    a = (4.0 / n_corr) * (1.0 - 1.0 / (2.0 * (n_corr - 1.0)))
    return {1: [1, 1, 2 / n_corr, 2 / n_corr, 2 / n_corr], 2: [1, 1, a, a, 2 / n_corr], 3: [1, 1, a, a, a],
            4: [1, 1, custom, custom, 2 / n_corr], 9: [1, 1, 1, 1, 1]}[flag]


@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_metric_classes_follow_the_path_occupations(c):
    deck = product_deck(c)
    sp = T.CsfSpace(deck)
    cnt = sp.counts()
    n = cnt["total_csfs"]
    expect = np.zeros(n, dtype=np.int64)
    expect[cnt["num_valence"]:cnt["num_valence"] + cnt["num_nm1"]] = 4
    expect[cnt["num_valence"] + cnt["num_nm1"]:] = 5
    nin, ni = c["ni"], c["ni"] + c["na"]
    refs = [[int(ch) for ch in r] for r in c["refs"]]
    iv = sp.index_vector(0)
    for lex in range(1, cnt["paths_v"] + 1):
        if iv[lex - 1] <= 0:
            continue
        occ, info = sp.path(0, lex)
        nsf = info["nsf"]
        if nsf <= 0:
            continue
        if sum(occ[:nin]) != 2 * nin:
            k = 3
        else:
            k = 1 if any(list(occ[nin:ni]) == r[nin:ni] for r in refs) else 2
        expect[iv[lex - 1] - 1:iv[lex - 1] - 1 + nsf] = k
    ncorr = c["ne"] - 2 * c.get("nf", 0)
    for flag in (1, 2, 3, 4, 9):
        g, cls = sp.acpf_gdiag(flag, 0.3)
        assert np.array_equal(cls, expect)
        assert np.allclose(g, np.array(_gvalues(flag, ncorr, 0.3))[cls - 1], rtol=0, atol=1e-15)


def _he2():
    with open(FIX) as f:
        fx = json.load(f)
    d = fx["deck"]
    deck = T.Deck(d["num_orbitals"], d["num_inactive"], d["num_active"], d["num_elec"], d["spin_mult"], d["refs"])
    return fx, deck, np.array(fx["h"]), np.array(fx["chol"]), fx["nuclear_repulsion"]


def test_oracle_acpf_energy_matches_the_printed_one():
    import scipy.linalg as sla
    from oracle import dense, sgga

    fx, deck, h, L, en = _he2()
    d = fx["deck"]
    od = dense.DenseSigma(sgga.Deck(d["num_orbitals"], d["num_inactive"], d["num_active"], d["num_elec"],
                                    d["spin_mult"], d["refs"], d["num_frozen"]))
    H = od.hamiltonian(h, L)
    g, cls = T.CsfSpace(deck).acpf_gdiag(1)
    ref = np.nonzero(cls == 1)[0]
    e_ref = np.linalg.eigvalsh(H[np.ix_(ref, ref)])[0]
    lam = sla.eigh(H - e_ref * np.eye(od.ncsf), np.diag(g), eigvals_only=True)[0]
    assert abs(e_ref + en - fx["reference_energy"]) < 1e-8
    assert abs(lam + e_ref + en - fx["acpf_root1"]) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("tf32x3", 1e-6)])
def test_device_acpf_matches_the_printed_energy(need_gpu, precision, tol):
    fx, deck, h, L, en = _he2()
    sb = T.SigmaBuilder(deck, T.Operator(h, L), device=0, precision=precision, tc_gemms="all")
    e, v, it, e_ref = sb.acpf(1, flag=1, tol_residual=1e-6, tol_energy=1e-8, want_vectors=True)
    sb.close()
    assert abs(e_ref + en - fx["reference_energy"]) < 1e-8
    assert abs(e[0] + en - fx["acpf_root1"]) < tol
    assert abs(np.linalg.norm(v[0]) - 1.0) < 1e-12


@pytest.mark.gpu
def test_water_mr_acpf_converges_in_both_forms(need_gpu):
    """MR-ACPF on H2O / cc-pVDZ with CAS(4,4) references through the molecular front end: the generalized
    solve converges on the reference's residual in both forms, the mixed root is within 1 uEh of the FP64
    one, and the ACPF energy lies below the MRCI energy of the same space (its size-extensivity shift)."""
    from tigerci_b200 import molecule as M

    deck, op, _ = M.water_c1()
    out = {}
    for f in ("fp64", "tf32x3"):
        sb = T.SigmaBuilder(deck, op, device=0, precision=f)
        e, _, it, e_ref = sb.acpf(1, flag=1, tol_residual=1e-6, tol_energy=1e-10)
        assert sb.stats()["converged"] == 1.0, (f, it)
        out[f] = float(e[0])
        if f == "fp64":
            ci, _, _ = sb.davidson(1, 1e-6, 1e-10)
            assert out[f] < float(ci[0]) < float(e_ref)
        sb.close()
    assert abs(out["tf32x3"] - out["fp64"]) <= 1e-6
