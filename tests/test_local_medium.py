"""Local decks at sizes where every tiling path of the domain kernels runs.

The projected-oracle tests (test_local_sigma.py) use spaces with at most seven
externals, so each domain kernel stays inside its first tile.  Here the
domains reach 90-140 externals: the two-external step on the common virtuals
walks several 64-row blocks, 32-column chunks and 16-deep k chunks; the
three-external forward step several 32-row chunks of the single-hole domain
and 8-row passes of the pair domain; the doublet deck has heads with more
than four pair matrices (two units per head); removed paths and heads
without local CSFs occur.  The reference is the non-local FP64 sigma build of
the same deck (itself pinned to the determinant oracle) on the padded vector:
sigma_loc = P^T H (P c), P the injection of the local CSFs (local_helpers).
FP64 within 1e-10 relative; the mixed form within 1e-5 relative (3xTF32
products)."""
import numpy as np
import pytest

import tigerci_b200 as T
from local_helpers import injection
from oracle import sgga
from tigerci_b200 import local
from tigerci_b200.synthetic import random_civec, synthetic_operator

pytestmark = pytest.mark.gpu


def _random_domains(n_paths, n_ext, lo, hi, rng, removed=0.1):
    out = []
    for _ in range(n_paths):
        if rng.random() < removed:
            out.append([-1])
        else:
            m = int(rng.integers(lo, hi + 1))
            out.append(sorted(rng.choice(n_ext, size=m, replace=False).tolist()))
    return out


def _closed_shell():
    """Six doubly occupied internal orbitals, 150 externals, pair and single-hole domains of 20..140."""
    loc = local.pair_domain_deck(n_int=6, n_virt=150, dmin=20, dmax=140, seed=7)
    base = T.Deck(loc.num_orbitals, 6, 0, 12, 1, ["2" * 6])
    return base, loc, loc.nm1_domains, loc.nm2_domains


def _doublet():
    """Doublet, two references with open shells, 90 externals, domains of 30..90, some paths removed."""
    args = (4 + 90, 2, 2, 5, 2, ["2210", "2201"])
    base = T.Deck(*args)
    cnt = T.CsfSpace(base).counts()
    rng = np.random.default_rng(11)
    nm1 = _random_domains(cnt["paths_nm1"], 90, 30, 90, rng)
    nm2 = _random_domains(cnt["paths_nm2"], 90, 30, 90, rng)
    return base, T.Deck(*args, nm1_domains=nm1, nm2_domains=nm2), nm1, nm2


@pytest.mark.parametrize("make", [_closed_shell, _doublet], ids=["closed-150ext", "doublet-90ext"])
def test_local_sigma_against_padded_nonlocal_sigma(make, need_gpu):
    base, loc, nm1, nm2 = make()
    h, L = synthetic_operator(base.num_orbitals, 96, seed=3, scale=0.05, diag_range=(-2.0, 1.0),
                              offdiag_sigma=0.02)
    op = T.Operator(h, L)
    osp = sgga.build_space(sgga.Deck(base.num_orbitals, base.num_inactive, base.num_active, base.num_elec,
                                     base.spin_mult, base.refs, base.num_frozen))
    P = injection(loc, nm1, nm2, osp, base.num_external)
    nl = T.SigmaBuilder(base, op, device=0, precision="fp64")
    lc = T.SigmaBuilder(loc, op, device=0, precision="fp64")
    lm = T.SigmaBuilder(loc, op, device=0, precision="tf32x3")
    assert lc.n == len(P) and nl.n == osp.total_csfs
    for seed in (1, 2):
        x = random_civec(lc.n, seed)
        full = np.zeros(nl.n)
        full[P] = x
        ref = nl.sigma(full)[P]
        scale = np.abs(ref).max()
        got = lc.sigma(x)
        assert np.abs(got - ref).max() <= 1e-10 * scale, np.abs(got - ref).max() / scale
        gm = lm.sigma(x)
        assert np.abs(gm - ref).max() <= 1e-5 * scale, np.abs(gm - ref).max() / scale
    assert np.abs(lc.diag() - nl.diag()[P]).max() <= 1e-10 * np.abs(nl.diag()).max()
    for s in (nl, lc, lm):
        s.close()
