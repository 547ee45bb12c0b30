"""Parity at the kernel-scale configuration's full size (16 internal: 8 inactive
+ 8 active, 240 virtuals, Cholesky rank 1600, 16 electrons, singlet, one
closed-shell reference; 1,971,105 CSFs), against the oracle.

The all-external term is isolated exactly: with every Cholesky row that
touches an internal orbital set to zero and h = 0, the only non-zero
integrals are (ab|cd) over external orbitals, so H c restricted to N-2 CSFs
is the all-external term (three_and_four_seg_mod_1.f90:3240-3518) and
nothing else.  The device FP64 sigma of that operator is compared with the
oracle's restatement of the reference's integral-driven loop (slab (ab|cd)
formed by dgemm, mod_1:556) on every CSF whose external pair (a, c) has its
larger index a in a sampled range; those entries are complete sums in the
oracle.  Tolerance: the plain-FP64 bound of 1e-10 relative."""
import numpy as np
import pytest

import tigerci_b200 as T
from oracle import dense, sgga
from tigerci_b200.synthetic import random_civec, synthetic_operator

pytestmark = pytest.mark.gpu

RTOL = 1e-10
NINT, NVIRT, NCHOL = 16, 240, 1600


def _pair_rows(osp, n, a0, a1):
    """CSF indices of the N-2 entries whose larger external index lies in [a0, a1)."""
    nab = n * (n - 1) // 2
    idx = []
    for h in osp.paths[2]:
        if h["off"] is not None:
            for k in range(h["nsf"]):
                base = h["off"] + k * nab
                idx.append(np.arange(base + a0 * (a0 - 1) // 2, base + a1 * (a1 - 1) // 2))
        if h["off_aa"] is not None:
            for k in range(h["nsf_aa"]):
                base = h["off_aa"] + k * n
                idx.append(np.arange(base + a0, base + a1))
    return np.concatenate(idx)


def allext_only_operator():
    norb = NINT + NVIRT
    _, L = synthetic_operator(norb, NCHOL, seed=1234)
    p = np.repeat(np.arange(norb), np.arange(1, norb + 1))
    q = np.concatenate([np.arange(i + 1) for i in range(norb)])
    L[(p < NINT) | (q < NINT)] = 0.0
    return np.zeros((norb, norb)), L


def test_allext_sigma_at_full_kernel_scale_against_oracle(need_gpu):
    refs = ["2" * 8 + "0" * 8]
    deck = T.Deck(NINT + NVIRT, 8, 8, 16, 1, refs)
    h, L = allext_only_operator()
    sb = T.SigmaBuilder(deck, T.Operator(h, L), device=0, precision="fp64")
    n = sb.n
    assert n == 1971105
    osp = sgga.build_space(sgga.Deck(NINT + NVIRT, 8, 8, 16, 1, refs))
    nv, n1 = osp.num_valence, osp.num_nm1
    x = random_civec(n, 29)
    x[:nv + n1] = 0.0
    got = sb.sigma(x)
    sb.close()
    dense.use_blas()
    for a0, a1 in [(0, 12), (228, 240)]:
        ref = dense.allext_sigma(osp, NINT, NVIRT, L, x, a_range=(a0, a1))
        rows = _pair_rows(osp, NVIRT, a0, a1)
        scale = np.abs(ref[rows]).max()
        assert scale > 0
        err = np.abs(got[rows] - ref[rows]).max() / scale
        assert err <= RTOL, (a0, a1, err)
    # nothing outside the N-2 blocks
    assert np.abs(got[:nv + n1]).max() == 0.0


def test_full_sigma_at_full_kernel_scale_against_cpu_arm(need_gpu, tmp_path):
    """Every term at once: the device FP64 sigma of the kernel-scale operator (exactly as specified,
    L ~ N(0,1)...) against the integral-direct CPU sigma of the oracle (plancpu.c: integrals formed from
    the Cholesky vectors, the all-external term in the reference's loop form, the other couplings from
    the plan's loop records), on the same CI vector.  1e-10 relative."""
    refs = ["2" * 8 + "0" * 8]
    deck = T.Deck(NINT + NVIRT, 8, 8, 16, 1, refs)
    h, L = synthetic_operator(NINT + NVIRT, NCHOL, seed=1234)
    op = T.Operator(h, L)
    sb = T.SigmaBuilder(deck, op, device=0, precision="fp64")
    x = random_civec(sb.n, 31)
    got = sb.sigma(x)
    sb.close()
    p = str(tmp_path / "c2.plan")
    T.Plan(deck, op).export(p)
    dense.use_blas()
    pc = dense.PlanSigmaCPU(p, L)
    ref = pc.sigma(x)
    pc.close()
    assert np.abs(got - ref).max() <= RTOL * np.abs(ref).max()
