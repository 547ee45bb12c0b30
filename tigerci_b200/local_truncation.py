"""Local truncation of an MRSDCI space: the weak-pairs (WP) and truncation-of-virtuals (TOV) approximations.

TigerCI builds a sphere around every orbital from its Mulliken populations (sphere_setup,
tiger_fortran/sphere_cylinder.f90:90-216: mulliken_pop :253-301, mulliken_sort :308-351,
find_important_centers :356-392, find_center :398-420, find_max_dist :426-449) and then

- removes every internal configuration that is a double excitation from the references whose hole pairs
  (i, j) all fail the WP test (their WP spheres do not overlap; WP_throw_out, locist_mod.f90:204-240,
  find_hole_pairs :532-610, are_interacting_WP, wp_tov_mod.f90:254-284);
- lets the N-1 and N-2 configurations that are double excitations excite only into the virtuals whose TOV
  sphere overlaps the TOV sphere of a hole of an interacting pair (virtual_truncation and
  find_allowed_virtuals, locist_mod.f90:358-530; are_interacting_TOV, wp_tov_mod.f90:286-325); single
  excitations keep every virtual.

`orbital_spheres` computes the spheres, `wp_tov_domains` the allowed-virtual lists of every N-1 and N-2 path
in lexical order (the deck's nm1_domains / nm2_domains, [-1] for a removed path), from which `Deck` builds the
local space.  Orbital cylinders (the CYLINDERS keyword) are not supported.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np


@dataclass
class Sphere:
    center: np.ndarray  # bohr
    radius: float       # bohr

    def overlaps(self, other: "Sphere") -> bool:  # spheres_overlap, sphere_cylinder.f90:548-563
        return float(np.linalg.norm(self.center - other.center)) <= self.radius + other.radius

    def contains(self, point) -> bool:  # point_in_sphere, sphere_cylinder.f90:571-589
        return float(np.linalg.norm(self.center - np.asarray(point, dtype=np.float64))) <= self.radius


@dataclass
class TruncationParameters:
    """The input keywords of the two approximations (radii in bohr)."""
    occupation_threshold: float = 0.8          # OCCUPATION THRESHOLD (internal orbitals)
    virtual_occupation_threshold: float = 0.8  # VIRTUAL OCCUPATION THRESHOLD
    wp_default_radius: float = 0.8             # WP DEFAULT RADIUS
    wp_multiplier: float = 1.38                # WP RADIUS MULTIPLIER
    tov_occupied_default_radius: float = 0.8   # TOV OCCUPIED DEFAULT RADIUS
    tov_occupied_multiplier: float = 1.725     # TOV OCCUPIED RADIUS MULTIPLIER
    tov_virtual_default_radius: float = 0.8    # TOV VIRTUAL DEFAULT RADIUS
    tov_virtual_multiplier: float = 1.725      # TOV VIRTUAL RADIUS MULTIPLIER


def ao_atoms(mol) -> np.ndarray:
    """Atom of every AO of a molecule (tigerci_b200.molecule.Molecule), in the front end's AO order."""
    out = []
    for atom, l, _, _ in mol.shells:
        out += [atom] * ((2 * l + 1) if (l == 2 and mol.pure_d) else (l + 1) * (l + 2) // 2)
    return np.asarray(out, dtype=np.int64)


def _center_and_extent(pop: np.ndarray, geometry: np.ndarray, threshold: float):
    """Center and largest distance between the important atoms of one orbital.  The populations are sorted
    by magnitude (ascending, ties in atom order), their signs kept; the important atoms are the largest ones
    whose signed populations first sum above the threshold; the center is their population-weighted mean."""
    n = len(pop)
    order = sorted(range(n), key=lambda a: abs(pop[a]))
    spop = np.array([pop[a] for a in order])
    total, last = 0.0, -1
    for k in range(n - 1, -1, -1):
        total += spop[k]
        if total > threshold:
            last = k
            break
    if last < 0:
        raise ValueError(f"no set of atoms carries {threshold} of the orbital (populations {pop})")
    part = spop[last:].sum()
    center = np.zeros(3)
    for k in range(n - 1, last - 1, -1):
        center += spop[k] / part * geometry[order[k]]
    dmax = -1.0
    for k in range(last, n):
        for l in range(k, n):
            dmax = max(dmax, float(np.linalg.norm(geometry[order[k]] - geometry[order[l]])))
    return center, dmax


def orbital_spheres(mol, C: np.ndarray, S: np.ndarray, num_internal: int,
                    params: Optional[TruncationParameters] = None):
    """WP spheres of the internal orbitals and TOV spheres of all orbitals (sphere_setup).

    C: AO x MO coefficients, S: the AO overlap matrix (both in the front end's AO basis; Mulliken populations
    do not depend on how the AOs are normalised).  Returns (wp, tov): lists of Sphere."""
    p = params or TruncationParameters()
    geometry = np.asarray(mol.coords, dtype=np.float64)
    atom = ao_atoms(mol)
    n_atoms = len(geometry)
    wp: List[Sphere] = []
    tov: List[Sphere] = []
    for orb in range(C.shape[1]):
        c = C[:, orb]
        trace = c * (S @ c)  # sum_nu C_mu C_nu S_mu,nu for every AO mu
        pop = np.bincount(atom, weights=trace, minlength=n_atoms)
        internal = orb < num_internal
        center, dmax = _center_and_extent(pop, geometry,
                                          p.occupation_threshold if internal else p.virtual_occupation_threshold)
        if internal:
            wp.append(Sphere(center, max(dmax * p.wp_multiplier, p.wp_default_radius)))
            tov.append(Sphere(center, max(dmax * p.tov_occupied_multiplier, p.tov_occupied_default_radius)))
        else:
            tov.append(Sphere(center, max(dmax * p.tov_virtual_multiplier, p.tov_virtual_default_radius)))
    return wp, tov


def hole_pairs(occ: Sequence[int], refs: Sequence[Sequence[int]]):
    """find_hole_pairs (locist_mod.f90:532-610): (only_double, [(i, j), ...]) of an internal occupation:
    only_double is False when the configuration is a reference or a single excitation from one; otherwise
    the hole pair of every reference it is a double excitation from (0-based internal orbitals)."""
    pairs = []
    for r in refs:
        d = [int(a) - int(b) for a, b in zip(r, occ)]
        if all(x == 0 for x in d):
            return False, []
        holes = sum(x for x in d if x > 0)
        particles = -sum(x for x in d if x < 0)
        if holes > 2 or particles > 2:
            continue
        if holes == 1:
            return False, []
        i = j = -1
        for k, x in enumerate(d):
            if x == 2:
                i = j = k
            elif x == 1:
                if i < 0:
                    i = k
                else:
                    j = k
        pairs.append((i, j))
    if not pairs:
        raise ValueError(f"configuration {list(occ)} is no reference, single or double excitation")
    return True, pairs


def wp_tov_domains(deck, wp: Sequence[Sphere], tov: Sequence[Sphere]):
    """The allowed-virtual lists of every N-1 and N-2 path of the deck's (non-local) space under WP and TOV:
    (nm1_domains, nm2_domains, report), each list a sorted list of external indices (0-based) or [-1] for a
    path WP removes.  report counts the removed paths and excitations the way the reference prints them."""
    from .api import CsfSpace, Deck

    base = Deck(deck.num_orbitals, deck.num_inactive, deck.num_active, deck.num_elec, deck.spin_mult,
                list(deck.refs), num_frozen=deck.num_frozen)
    sp = CsfSpace(base)
    cnt = sp.counts()
    nint = base.num_internal
    n_ext = base.num_external
    refs = [[int(ch) for ch in r] for r in base.refs]

    def wp_pair(i, j):
        return wp[i].overlaps(wp[j])

    def tov_pair(i, j, a):  # a: orbital index (internal + external position)
        return tov[a].overlaps(tov[i]) or tov[a].overlaps(tov[j])

    # WP removal of valence paths cannot be expressed by the deck's domain lists: refuse it
    for lex in range(1, cnt["paths_v"] + 1):
        occ, _ = sp.path(0, lex)
        dbl, pairs = hole_pairs(occ, refs)
        if dbl and not any(wp_pair(i, j) for i, j in pairs):
            raise NotImplementedError("the weak-pairs approximation removes a valence configuration")
    report = {"nm1_paths_removed": 0, "nm2_paths_removed": 0}
    out = {}
    for kind in (1, 2):
        doms = []
        for lex in range(1, cnt["paths_nm1" if kind == 1 else "paths_nm2"] + 1):
            occ, _ = sp.path(kind, lex)
            dbl, pairs = hole_pairs(occ, refs)
            if not dbl:
                doms.append(list(range(n_ext)))
                continue
            live = [(i, j) for i, j in pairs if wp_pair(i, j)]
            if not live:
                doms.append([-1])
                report["nm1_paths_removed" if kind == 1 else "nm2_paths_removed"] += 1
                continue
            allowed = set()
            for i, j in live:
                for a in range(n_ext):
                    if tov_pair(i, j, nint + a):
                        allowed.add(a)
            # no virtual left: the path carries no CSF, like a removed one
            doms.append(sorted(allowed) if allowed else [-1])
        out[kind] = doms
    return out[1], out[2], report
