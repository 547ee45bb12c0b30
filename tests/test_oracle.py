"""The dense oracle itself: its CSF Hamiltonian is symmetric, its spectrum is
a subset of the determinant-space spectrum (the CSF space is the S = target
subspace of a spin-complete determinant space), and for two electrons
(where MRSDCI is full CI) its lowest root equals full CI."""
import itertools

import numpy as np
import pytest

from cases import SMALL_CASES, case_id, oracle_deck
from oracle import dense
from tigerci_b200.synthetic import synthetic_operator


@pytest.mark.parametrize("c", SMALL_CASES[:6], ids=case_id)
def test_csf_spectrum_inside_determinant_spectrum(c):
    od = dense.DenseSigma(oracle_deck(c))
    if od.ncsf > 250:
        pytest.skip("dense diagonalisation too large")
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    H = od.hamiltonian(h, L)
    assert np.abs(H - H.T).max() < 1e-12
    # determinant Hamiltonian over the same determinants
    nd = len(od.dets)
    Hd = np.zeros((nd, nd))
    eri = np.ascontiguousarray(dense.eri_from_chol(L, c["no"]))
    for j in range(nd):
        x = np.zeros(nd)
        x[j] = 1.0
        y = np.zeros(nd)
        dense.lib().oracle_hdet_matvec(nd, od.dets.ctypes.data, c["no"], np.ascontiguousarray(h).ctypes.data,
                                       eri.ctypes.data, x.ctypes.data, y.ctypes.data)
        Hd[:, j] = y
    ec = np.linalg.eigvalsh(H)
    ed = np.linalg.eigvalsh(Hd)
    for e in ec:
        assert np.min(np.abs(ed - e)) < 1e-9


def _s2_matrix(dets, norb):
    """S^2 = S_z^2 + S_z + S_- S_+ over determinants (bit 2p alpha, 2p+1 beta)."""
    idx = {int(d): i for i, d in enumerate(dets)}
    nd = len(dets)
    S2 = np.zeros((nd, nd))

    def par(d, x):
        return bin(d & ((1 << x) - 1)).count("1") & 1

    for j, d in enumerate(dets):
        d = int(d)
        na = sum((d >> (2 * p)) & 1 for p in range(norb))
        nb = sum((d >> (2 * p + 1)) & 1 for p in range(norb))
        sz = 0.5 * (na - nb)
        S2[j, j] += sz * sz + sz
        # S_- S_+ = sum_{p,q} a+_{q b} a_{q a} a+_{p a} a_{p b}
        for p in range(norb):
            if not (d >> (2 * p + 1)) & 1 or (d >> (2 * p)) & 1:
                continue
            ph = par(d, 2 * p + 1)
            d1 = d & ~(1 << (2 * p + 1))
            ph ^= par(d1, 2 * p)
            d1 |= 1 << (2 * p)
            for q in range(norb):
                if not (d1 >> (2 * q)) & 1 or (d1 >> (2 * q + 1)) & 1:
                    continue
                ph2 = ph ^ par(d1, 2 * q)
                d2 = d1 & ~(1 << (2 * q))
                ph2 ^= par(d2, 2 * q + 1)
                d2 |= 1 << (2 * q + 1)
                if d2 in idx:
                    S2[idx[d2], j] += -1.0 if ph2 else 1.0
    return S2


def test_two_electron_full_ci():
    """2 electrons, 1 internal orbital, 5 externals: MRSDCI = full CI of the
    singlets, so every CSF eigenvalue equals a singlet eigenvalue of the full
    determinant Hamiltonian and the counts agree."""
    from oracle import sgga

    norb = 6
    od = dense.DenseSigma(sgga.Deck(norb, 1, 0, 2, 1, ["2"]))
    h, L = synthetic_operator(norb, 8, seed=5, scale=0.4, diag_range=(-2, 1), offdiag_sigma=0.2)
    H = od.hamiltonian(h, L)
    e_csf = np.linalg.eigvalsh(H)
    eri = np.ascontiguousarray(dense.eri_from_chol(L, norb))
    dets = np.array([(1 << (2 * a)) | (1 << (2 * b + 1)) for a, b in itertools.product(range(norb), range(norb))],
                    dtype=np.uint64)
    nd = len(dets)
    Hd = np.zeros((nd, nd))
    for j in range(nd):
        x = np.zeros(nd)
        x[j] = 1
        y = np.zeros(nd)
        dense.lib().oracle_hdet_matvec(nd, dets.ctypes.data, norb, np.ascontiguousarray(h).ctypes.data,
                                       eri.ctypes.data, x.ctypes.data, y.ctypes.data)
        Hd[:, j] = y
    w, U = np.linalg.eigh(_s2_matrix(dets, norb))
    Us = U[:, np.abs(w) < 1e-8]
    e_fci = np.linalg.eigvalsh(Us.T @ Hd @ Us)
    assert len(e_fci) == len(e_csf)
    assert np.abs(np.sort(e_fci) - np.sort(e_csf)).max() < 1e-10


@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_integral_direct_cpu_sigma_equals_dense_oracle(c, tmp_path):
    """The CPU arm's sigma (plancpu.c: integrals formed from the Cholesky vectors, all-external term in the
    reference's loop form, the other couplings replayed from the plan's loop records) equals the
    determinant-space sigma."""
    import tigerci_b200 as T
    from cases import product_deck
    from tigerci_b200.synthetic import random_civec

    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    od = dense.DenseSigma(oracle_deck(c))
    p = str(tmp_path / "plan.bin")
    T.Plan(product_deck(c), T.Operator(h, L)).export(p)
    dense.use_blas()
    pc = dense.PlanSigmaCPU(p, L)
    for seed in (1, 2):
        x = random_civec(od.ncsf, seed)
        ref = od.sigma(h, L, x)
        got = pc.sigma(x)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    pc.close()
