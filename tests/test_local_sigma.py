"""Local pair domains through the whole sigma build and the Davidson solve.

A deck with allowed-virtual lists per N-1 / N-2 path (the data of
allowed_virtuals_mod.f90 / virtual_truncation, locist_mod.f90:358-451) defines
a local CSF space: each head's blocks span only its domain, some heads
removed.  Its Hamiltonian is the non-local Hamiltonian restricted to those
CSFs, H_loc = P^T H P with P the injection of local CSFs into the non-local
space, so the oracle's local sigma is P^T (H (P c)) from the dense
determinant oracle of the non-local deck, with P built here from the two
spaces' index vectors.  The device computes it as the plan of the non-local
space on padded blocks plus the pair-domain all-external term; FP64 within
1e-10 relative, the lowest root of the local space within 1e-8 Eh."""
import numpy as np
import pytest

import tigerci_b200 as T
from local_helpers import injection
from oracle import dense, sgga
from tigerci_b200.synthetic import random_civec, synthetic_operator

pytestmark = pytest.mark.gpu

CASES = [
    dict(no=9, ni=2, na=1, ne=4, sm=1, refs=["220"]),
    dict(no=9, ni=2, na=2, ne=6, sm=3, refs=["2211"]),
    dict(no=10, ni=2, na=2, ne=6, sm=1, refs=["2220", "2202"], nf=1),
    dict(no=10, ni=1, na=3, ne=5, sm=2, refs=["2210", "2201"]),
]


def _decks(c, seed):
    base = T.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], num_frozen=c.get("nf", 0))
    cnt = T.CsfSpace(base).counts()
    n_ext = base.num_external
    rng = np.random.default_rng(seed)

    def doms(npaths):
        out = []
        for _ in range(npaths):
            if rng.random() < 0.15:
                out.append([-1])  # removed path
            else:
                m = int(rng.integers(1, n_ext + 1))
                out.append(sorted(rng.choice(n_ext, size=m, replace=False).tolist()))
        return out

    nm1, nm2 = doms(cnt["paths_nm1"]), doms(cnt["paths_nm2"])
    loc = T.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], num_frozen=c.get("nf", 0),
                 nm1_domains=nm1, nm2_domains=nm2)
    return base, loc, nm1, nm2


@pytest.mark.parametrize("c", CASES, ids=lambda c: f"no{c['no']}-m{c['sm']}-r{len(c['refs'])}")
def test_local_sigma_and_root_against_projected_oracle(c, need_gpu):
    base, loc, nm1, nm2 = _decks(c, seed=c["no"] * 7 + c["sm"])
    h, L = synthetic_operator(c["no"], 12, seed=5, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    od = dense.DenseSigma(sgga.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], c.get("nf", 0)))
    P = injection(loc, nm1, nm2, od.space, base.num_external)
    H = od.hamiltonian(h, L)
    Hl = H[np.ix_(P, P)]
    sb = T.SigmaBuilder(loc, T.Operator(h, L), device=0, precision="fp64")
    assert sb.n == len(P)
    for seed in (1, 2):
        x = random_civec(sb.n, seed)
        ref = Hl @ x
        got = sb.sigma(x)
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.abs(sb.diag() - np.diag(Hl)).max() <= 1e-10 * np.abs(np.diag(Hl)).max()
    e, _, _ = sb.davidson(1, 1e-8, 1e-12)
    sb.close()
    assert abs(e[0] - np.linalg.eigvalsh(Hl)[0]) <= 1e-8
    sbm = T.SigmaBuilder(loc, T.Operator(h, L), device=0, precision="tf32x3")
    em, _, _ = sbm.davidson(1, 1e-8, 1e-12)
    sbm.close()
    assert abs(em[0] - e[0]) <= 1e-6
