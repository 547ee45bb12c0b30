"""Loop enumeration of the local all-external term against the reference's dry run.

The reference enumerates its local all-external loops once, in a dry run before
the first iteration (three_and_four_seg_mod_1.f90:414-436 calling
build_ext_34seg_dryrun, :3142-3238): one record per external pair a >= c and
N-2 internal path whose allowed virtuals hold both.  The heads and domains this
library's pair-domain term applies (the ones tci_sigma_init builds for a deck
with domains) must give the same records as a multiset: pair, head weight,
positions in the domain, spin counts and the heads' CI addresses, bit for bit
(oracle/dryrun.py restates the dry run over the oracle's index vectors)."""
import numpy as np
import pytest

import tigerci_b200 as T
from oracle import dryrun, sgga
from tigerci_b200 import local
from tigerci_b200._lib import TciError

CASES = [
    dict(no=9, ni=2, na=1, ne=4, sm=1, refs=["220"]),
    dict(no=9, ni=2, na=2, ne=6, sm=3, refs=["2211"]),
    dict(no=10, ni=2, na=2, ne=6, sm=1, refs=["2220", "2202"], nf=1),
    dict(no=10, ni=1, na=3, ne=5, sm=2, refs=["2210", "2201"]),
    dict(no=14, ni=3, na=1, ne=6, sm=1, refs=["2220"]),
]


def _domains(n_paths, n_ext, rng, removed=0.15):
    out = []
    for _ in range(n_paths):
        if rng.random() < removed:
            out.append([-1])
        else:
            m = int(rng.integers(1, n_ext + 1))
            out.append(sorted(rng.choice(n_ext, size=m, replace=False).tolist()))
    return out


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("c", CASES, ids=lambda c: f"no{c['no']}-m{c['sm']}-r{len(c['refs'])}")
def test_allext_records_equal_reference_dry_run(c, seed):
    base = T.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], num_frozen=c.get("nf", 0))
    cnt = T.CsfSpace(base).counts()
    rng = np.random.default_rng(seed)
    nm1 = _domains(cnt["paths_nm1"], base.num_external, rng)
    nm2 = _domains(cnt["paths_nm2"], base.num_external, rng)
    deck = T.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], num_frozen=c.get("nf", 0),
                  nm1_domains=nm1, nm2_domains=nm2)
    got = sorted(tuple(int(x) for x in r) for r in local.allext_records(deck))
    od = sgga.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], c.get("nf", 0))
    want = sorted(dryrun.allext_records(od, nm1, nm2))
    assert len(got) == len(want) and got == want


def test_allext_records_pair_domain_deck():
    """The pair-domain workload's deck at a small size (8 doubly occupied internal orbitals, 30 externals)."""
    deck = local.pair_domain_deck(n_int=8, n_virt=30, dmin=3, dmax=20)
    got = sorted(tuple(int(x) for x in r) for r in local.allext_records(deck))
    od = sgga.Deck(deck.num_orbitals, deck.num_inactive, deck.num_active, deck.num_elec, deck.spin_mult, deck.refs,
                   deck.num_frozen)
    want = sorted(dryrun.allext_records(od, deck.nm1_domains, deck.nm2_domains))
    assert len(got) == len(want) > 0 and got == want


def test_allext_records_need_domains():
    deck = T.Deck(9, 2, 1, 4, 1, ["220"])
    with pytest.raises(TciError):
        local.allext_records(deck)
