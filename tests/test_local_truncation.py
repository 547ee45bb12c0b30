"""WP / TOV local truncation (tigerci_b200/local_truncation.py): the reference's hole-pair rules
(find_hole_pairs), its sphere construction from Mulliken populations (sphere_cylinder.f90) on orbitals
whose populations are known by construction, and the domain lists it produces as a local deck."""
import numpy as np
import pytest

import tigerci_b200 as T
from tigerci_b200 import local_truncation as LT
from tigerci_b200 import molecule as M


def test_hole_pairs_follow_the_reference_rules():
    ref = [[2, 2, 2, 0]]
    assert LT.hole_pairs([2, 2, 2, 0], ref) == (False, [])  # a reference
    assert LT.hole_pairs([2, 2, 1, 0], ref) == (False, [])  # single excitation: one hole
    assert LT.hole_pairs([2, 1, 1, 0], ref) == (True, [(1, 2)])
    assert LT.hole_pairs([0, 2, 2, 0], ref) == (True, [(0, 0)])
    assert LT.hole_pairs([1, 1, 2, 1], ref) == (True, [(0, 1)])  # one electron moved into the active orbital
    # two references: a configuration that is a single excitation from either keeps every virtual
    refs = [[2, 2, 2, 0], [2, 2, 0, 2]]
    assert LT.hole_pairs([2, 2, 1, 1], refs) == (False, [])
    dbl, pairs = LT.hole_pairs([2, 1, 1, 1], refs)
    assert dbl and pairs == [(1, 2), (1, 3)]
    with pytest.raises(ValueError):
        LT.hole_pairs([0, 0, 2, 2], [[2, 2, 2, 2]])  # a quadruple excitation


def test_spheres_from_populations():
    # H2 at 1.4 bohr, STO-like s functions: an orbital on one atom keeps the default radius, one shared
    # equally by both atoms gets multiplier x bond length around the bond midpoint
    s = (0, 0, [1.24], [1.0])
    mol = M.Molecule([1.0, 1.0], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]]), [s, (1, 0, [1.24], [1.0])], False)
    S, _ = M.Integrals(mol, 1e-8).one_electron()
    bond = np.array([1.0, 1.0]) / np.sqrt(2.0 + 2.0 * S[0, 1])
    atom0 = np.array([1.0 / np.sqrt(S[0, 0]), 0.0])  # the first atom's s function alone
    C = np.stack([bond, atom0], axis=1)
    p = LT.TruncationParameters()
    wp, tov = LT.orbital_spheres(mol, C, S, 1, p)
    assert np.allclose(wp[0].center, [0.0, 0.0, 0.7]) and abs(wp[0].radius - 1.38 * 1.4) < 1e-12
    assert abs(tov[0].radius - 1.725 * 1.4) < 1e-12
    assert np.allclose(tov[1].center, [0.0, 0.0, 0.0]) and tov[1].radius == p.tov_virtual_default_radius


def test_domains_make_a_local_deck():
    """Hand-placed spheres: two separated internal orbitals (no WP overlap), virtuals near one or the other."""
    deck = T.Deck(6, 2, 0, 4, 1, ["22"])
    far = 20.0
    wp = [LT.Sphere(np.array([0.0, 0, 0]), 1.0), LT.Sphere(np.array([far, 0, 0]), 1.0)]
    tov = [LT.Sphere(np.array([0.0, 0, 0]), 1.5), LT.Sphere(np.array([far, 0, 0]), 1.5),
           LT.Sphere(np.array([0.5, 0, 0]), 0.8), LT.Sphere(np.array([far + 0.5, 0, 0]), 0.8),
           LT.Sphere(np.array([1.0, 0, 0]), 0.8), LT.Sphere(np.array([far / 2, 0, 0]), 0.8)]
    nm1, nm2, rep = LT.wp_tov_domains(deck, wp, tov)
    sp = T.CsfSpace(deck)
    occ2 = [tuple(sp.path(2, lex)[0]) for lex in range(1, sp.counts()["paths_nm2"] + 1)]
    dom2 = dict(zip(occ2, nm2))
    assert dom2[(0, 2)] == [0, 2]        # pair (0,0): the virtuals near orbital 0
    assert dom2[(2, 0)] == [1]           # pair (1,1): the virtual near orbital 1
    assert dom2[(1, 1)] == [-1]          # pair (0,1): weak pair, removed
    assert rep["nm2_paths_removed"] == 1
    assert all(d == list(range(4)) for d in nm1)  # N-1 paths are single excitations here: all virtuals
    loc = T.Deck(6, 2, 0, 4, 1, ["22"], nm1_domains=nm1, nm2_domains=nm2)
    c = T.CsfSpace(loc).counts()
    # valence 1 + N-1: 2 paths x 4 virtuals + N-2: (0,0) over 2 virtuals: aa 2 + ab 1; (1,1) over 1: aa 1
    assert c["total_csfs"] == 1 + 8 + 3 + 1
