"""Molecular front end (host): AO integrals against the oracle's
McMurchie-Davidson restatement, pure-d combinations, the pivoted Cholesky
decomposition, RHF against an independent SCF on the exact ERI tensor, and
the AO -> MO transform against numpy."""
import itertools

import numpy as np
import pytest

import tigerci_b200 as T
from oracle import gto
from tigerci_b200 import molecule as M

# a small molecule with s, p and d shells on three centres (contracted and uncontracted)
ATOMS = [(6, [0.0, 0.1, -0.2]), (1, [0.3, -0.2, 2.0]), (8, [1.9, 0.4, 0.7])]
SHELLS = [(0, 0, [5.0, 1.2], [0.6, 0.5]), (0, 1, [1.1, 0.3], [0.5, 0.6]), (0, 2, [0.8], [1.0]),
          (1, 0, [0.9], [1.0]), (2, 2, [1.3, 0.5], [0.3, 0.8])]


def _mol(pure):
    return M.Molecule([a[0] for a in ATOMS], np.array([a[1] for a in ATOMS]), SHELLS, pure)


def test_one_and_two_electron_integrals_match_oracle():
    it = M.Integrals(_mol(False), 1e-12)
    bas = gto.Basis(ATOMS, [(ATOMS[s[0]][1], s[1], s[2], s[3]) for s in SHELLS])
    S, h = it.one_electron()
    assert np.abs(S - gto.overlap(bas)).max() < 1e-13
    assert np.abs(h - (gto.kinetic(bas) + gto.nuclear(bas))).max() < 1e-12
    g = it.ao_eri()
    go = gto.eri(bas)
    assert np.abs(g - go).max() < 1e-12 * max(1.0, np.abs(go).max())
    assert abs(it.nuclear_repulsion - gto.nuclear_repulsion(ATOMS)) < 1e-12


def test_pure_d_is_the_normalised_combination_of_cartesian_components():
    cart = M.Integrals(_mol(False), 1e-12)
    pure = M.Integrals(_mol(True), 1e-12)
    # the transformation, written out here: d0 = zz - (xx + yy)/2, d+1 = xz, d-1 = yz, d+2 = sqrt(3)/2 (xx - yy),
    # d-2 = xy over the normalised Cartesian components xx yy zz xy xz yz
    Td = np.array([[-0.5, -0.5, 1, 0, 0, 0], [0, 0, 0, 0, 1, 0], [0, 0, 0, 0, 0, 1],
                   [np.sqrt(3) / 2, -np.sqrt(3) / 2, 0, 0, 0, 0], [0, 0, 0, 1, 0, 0]])
    blocks = []
    for _, l, _, _ in SHELLS:
        blocks.append(Td if l == 2 else np.eye((l + 1) * (l + 2) // 2))
    Tm = np.zeros((sum(b.shape[0] for b in blocks), sum(b.shape[1] for b in blocks)))
    r = c = 0
    for b in blocks:
        Tm[r:r + b.shape[0], c:c + b.shape[1]] = b
        r, c = r + b.shape[0], c + b.shape[1]
    S_c, h_c = cart.one_electron()
    S_p, h_p = pure.one_electron()
    assert np.abs(S_p - Tm @ S_c @ Tm.T).max() < 1e-13
    assert np.abs(np.diag(S_p) - 1.0).max() < 1e-13  # the pure functions are normalised
    assert np.abs(h_p - Tm @ h_c @ Tm.T).max() < 1e-12
    g_p = np.einsum("ai,bj,ck,dl,ijkl->abcd", Tm, Tm, Tm, Tm, cart.ao_eri(), optimize=True)
    assert np.abs(pure.ao_eri() - g_p).max() < 1e-12


@pytest.mark.parametrize("thr", [1e-4, 1e-8, 1e-12])
def test_pivoted_cholesky_reconstructs_to_threshold(thr):
    it = M.Integrals(_mol(True), thr)
    n = it.nbf
    g = it.ao_eri()
    pairs = [(p, q) for p in range(n) for q in range(p + 1)]
    V = np.array([[g[p, q, r, s] for (r, s) in pairs] for (p, q) in pairs])
    L = it.ao_cholesky()
    R = V - L @ L.T
    # remaining diagonal at most the threshold; the error of a positive semidefinite remainder is bounded by it
    assert np.diag(R).max() <= thr * (1 + 1e-9)
    assert np.abs(R).max() <= thr * (1 + 1e-9) + 1e-13
    # the oracle's dense pivoted Cholesky gives the same number of vectors
    assert gto.pivoted_cholesky(V, thr).shape[1] == it.nchol


def _scf_numpy(S, h, g, nocc, e_nuc):
    """Plain Roothaan-Hall iterations with damping, exact ERI tensor (independent of the library's SCF)."""
    w, V = np.linalg.eigh(S)
    X = V @ np.diag(w ** -0.5) @ V.T
    e, Cp = np.linalg.eigh(X.T @ h @ X)
    Cm = X @ Cp
    E_old = 0.0
    D = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
    for _ in range(500):
        F = h + np.einsum("pqrs,rs->pq", g, D) - 0.5 * np.einsum("prqs,rs->pq", g, D)
        E = 0.5 * np.sum(D * (h + F)) + e_nuc
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        Cm = X @ Cp
        Dn = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
        if abs(E - E_old) < 1e-13 and np.abs(Dn - D).max() < 1e-9:
            break
        D, E_old = 0.5 * D + 0.5 * Dn, E
    return E, e


def test_rhf_matches_independent_scf_on_water():
    sym, xyz = M.water()
    mol = M.Molecule.from_atoms(sym, xyz, "cc-pVDZ", pure_d=True)
    it = M.Integrals(mol, 1e-12)
    Cm, eps, E, nit = it.rhf(5, conv=1e-12)
    S, h = it.one_electron()
    E_ref, e_ref = _scf_numpy(S, h, it.ao_eri(), 5, it.nuclear_repulsion)
    assert abs(E - E_ref) < 1e-9
    assert np.abs(eps - e_ref).max() < 1e-6
    assert np.abs(Cm.T @ S @ Cm - np.eye(it.nbf)).max() < 1e-10


def test_mo_operator_is_the_transform_of_the_ao_vectors():
    it = M.Integrals(_mol(True), 1e-10)
    n = it.nbf
    rng = np.random.default_rng(3)
    Cm = rng.standard_normal((n, n - 2))
    h, L = it.mo_operator(Cm)
    _, h_ao = it.one_electron()
    assert np.abs(h - Cm.T @ h_ao @ Cm).max() < 1e-11
    Lao = it.ao_cholesky()
    m = Cm.shape[1]
    for J in (0, it.nchol // 2, it.nchol - 1):
        A = np.zeros((n, n))
        for p in range(n):
            for q in range(p + 1):
                A[p, q] = A[q, p] = Lao[p * (p + 1) // 2 + q, J]
        B = Cm.T @ A @ Cm
        got = np.array([L[p * (p + 1) // 2 + q, J] for p in range(m) for q in range(p + 1)])
        want = np.array([B[p, q] for p in range(m) for q in range(p + 1)])
        assert np.abs(got - want).max() < 1e-11


def test_cc_pvdz_counts_and_errors():
    sym, xyz = M.water()
    assert M.Molecule.from_atoms(sym, xyz, "cc-pVDZ", pure_d=True).nbf == 24
    assert M.Molecule.from_atoms(sym, xyz, "cc-pVDZ", pure_d=False).nbf == 25
    bad = M.Molecule([1.0, 1.0], np.zeros((2, 3)), [(0, 0, [1.0], [1.0]), (1, 0, [1.0], [1.0])])
    with pytest.raises(T._lib.TciError):
        M.Integrals(bad, 1e-6)  # two atoms at the same position
    with pytest.raises(T._lib.TciError):
        M.Integrals(M.Molecule([1.0], np.zeros((1, 3)), [(0, 3, [1.0], [1.0])]), 1e-6)  # f shell
