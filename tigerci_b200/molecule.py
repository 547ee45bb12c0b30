"""Molecules, Gaussian basis sets and Molden orbitals for the front end that
turns a molecule into the MO operator (h, Cholesky vectors) of the sigma
build.

The reference reads orbitals, geometry and basis from a Molden file
(`tiger_cpp/OrbitalParsers.cpp` MoldenOrbitalParser; coordinates in Angstrom
converted with ANGSTROMINBOHR = 1.8897261, `erkale/global.h:76`), computes
AO integrals with libint, decomposes them (CD THRESHOLD) and transforms the
Cholesky vectors to the MO basis (`tiger_cpp/main.cpp:270-361`).  Here the
integrals, the decomposition, the transform and an RHF solver for molecules
without orbitals are the library's own (`tci_integrals_*`, `tci_rhf`,
`tci_mo_operator` in include/tigerci_sigma.h); this module holds the
geometry and basis data and the Molden reader.

Basis data: Dunning's cc-pVDZ (T. H. Dunning Jr., J. Chem. Phys. 90, 1007
(1989)) for H, C, N and O in its segmented general-contraction form;
contraction coefficients refer to normalised primitives.
"""
from __future__ import annotations

import ctypes as C
import itertools
import math
import re
import time
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

from ._lib import TciMolecule, check, lib, ptr

ANGSTROM_IN_BOHR = 1.8897261  # the reference's conversion (erkale/global.h:76)
Z_OF = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8}

# cc-pVDZ: element -> list of (l, [(exponent, coefficient), ...])
_S1 = {
    "C": [6665.0, 1000.0, 228.0, 64.71, 21.06, 7.495, 2.797, 0.5215],
    "N": [9046.0, 1357.0, 309.3, 87.73, 28.56, 10.21, 3.838, 0.7466],
    "O": [11720.0, 1759.0, 400.8, 113.7, 37.03, 13.27, 5.025, 1.013],
}
_C1S = {
    "C": [0.000692, 0.005329, 0.027077, 0.101718, 0.274740, 0.448564, 0.285074, 0.015204],
    "N": [0.000700, 0.005389, 0.027406, 0.103207, 0.278723, 0.448540, 0.278238, 0.015440],
    "O": [0.000710, 0.005470, 0.027837, 0.104800, 0.283062, 0.448719, 0.270952, 0.015458],
}
_C2S = {
    "C": [-0.000146, -0.001154, -0.005725, -0.023312, -0.063955, -0.149981, -0.127262, 0.544529],
    "N": [-0.000153, -0.001208, -0.005992, -0.024544, -0.067459, -0.158078, -0.121831, 0.549003],
    "O": [-0.000160, -0.001263, -0.006267, -0.025716, -0.070924, -0.165411, -0.116955, 0.557368],
}
_SP = {  # (s outer, p exps, p coefs, p outer, d)
    "C": (0.1596, [9.439, 2.002, 0.5456], [0.038109, 0.209480, 0.508557], 0.1517, 0.550),
    "N": (0.2248, [13.55, 2.917, 0.7973], [0.039919, 0.217169, 0.510319], 0.2185, 0.817),
    "O": (0.3023, [17.70, 3.854, 1.046], [0.043018, 0.228913, 0.508728], 0.2753, 1.185),
}


def cc_pvdz(element: str):
    """Shells of cc-pVDZ for H, C, N or O: list of (l, exponents, coefficients)."""
    if element == "H":
        return [(0, [13.01, 1.962, 0.4446], [0.019685, 0.137977, 0.478148]), (0, [0.1220], [1.0]),
                (1, [0.7270], [1.0])]
    if element not in _S1:
        raise ValueError(f"cc-pVDZ data for {element} is not included")
    so, pe, pc, po, d = _SP[element]
    return [(0, _S1[element], _C1S[element]), (0, _S1[element], _C2S[element]), (0, [so], [1.0]),
            (1, pe, pc), (1, [po], [1.0]), (2, [d], [1.0])]


BASIS_SETS = {"cc-pvdz": cc_pvdz}


@dataclass
class Molecule:
    """Atoms (nuclear charge, position in bohr) and contracted shells
    (atom index, l, exponents, coefficients of normalised primitives)."""
    charges: Sequence[float]
    coords: np.ndarray                                  # n_atoms x 3, bohr
    shells: List[Tuple[int, int, List[float], List[float]]]
    pure_d: bool = False
    _keep: list = field(default_factory=list, repr=False)

    @classmethod
    def from_atoms(cls, symbols: Sequence[str], coords_bohr, basis: str = "cc-pVDZ", pure_d: bool = True):
        fn = BASIS_SETS[basis.lower()]
        shells = []
        for i, s in enumerate(symbols):
            for l, e, c in fn(s):
                shells.append((i, l, list(e), list(c)))
        return cls([float(Z_OF[s]) for s in symbols], np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3),
                   shells, pure_d)

    @property
    def n_electrons(self) -> int:
        return int(round(sum(self.charges)))

    @property
    def nbf(self) -> int:
        return sum((2 * l + 1) if (l == 2 and self.pure_d) else (l + 1) * (l + 2) // 2 for _, l, _, _ in self.shells)

    def c_struct(self) -> TciMolecule:
        z = np.ascontiguousarray(self.charges, dtype=np.float64)
        xyz = np.ascontiguousarray(self.coords, dtype=np.float64)
        sa = np.array([s[0] for s in self.shells], dtype=np.int64)
        sl = np.array([s[1] for s in self.shells], dtype=np.int64)
        sn = np.array([len(s[2]) for s in self.shells], dtype=np.int64)
        ex = np.array([e for s in self.shells for e in s[2]], dtype=np.float64)
        cf = np.array([c for s in self.shells for c in s[3]], dtype=np.float64)
        self._keep = [z, xyz, sa, sl, sn, ex, cf]
        return TciMolecule(len(z), ptr(z), ptr(xyz), len(sa), ptr(sa), ptr(sl), ptr(sn), ptr(ex), ptr(cf),
                           1 if self.pure_d else 0)


class Integrals:
    """AO integrals and the pivoted Cholesky decomposition of the AO ERI
    matrix to `cd_threshold` (the reference's CD THRESHOLD)."""

    def __init__(self, mol: Molecule, cd_threshold: float = 1e-6):
        self.mol = mol
        m = mol.c_struct()
        h = C.c_void_p()
        check(lib().tci_integrals_create(C.byref(m), float(cd_threshold), C.byref(h)))
        self._h = h
        info = np.zeros(8)
        check(lib().tci_integrals_info(self._h, ptr(info), 8))
        self.nbf, self.nchol = int(info[0]), int(info[1])
        self.nuclear_repulsion = float(info[2])
        self.seconds = float(info[3])
        self.max_remaining = float(info[4])
        self.quartets = int(info[5])

    def one_electron(self):
        S = np.zeros((self.nbf, self.nbf))
        h = np.zeros((self.nbf, self.nbf))
        check(lib().tci_integrals_one_electron(self._h, ptr(S), ptr(h), self.nbf))
        return S, h

    def ao_cholesky(self):
        npair = self.nbf * (self.nbf + 1) // 2
        L = np.zeros((npair, self.nchol))
        check(lib().tci_integrals_ao_cholesky(self._h, ptr(L), npair, self.nchol))
        return L

    def ao_eri(self):
        g = np.zeros((self.nbf,) * 4)
        check(lib().tci_integrals_ao_eri(self._h, ptr(g), self.nbf))
        return g

    def rhf(self, n_occ: int, maxit: int = 100, conv: float = 1e-10):
        """Canonical RHF orbitals: (C nbf x nbf, orbital energies, total energy, iterations)."""
        Cm = np.zeros((self.nbf, self.nbf))
        eps = np.zeros(self.nbf)
        info = np.zeros(4)
        check(lib().tci_rhf(self._h, int(n_occ), int(maxit), float(conv), ptr(Cm), ptr(eps), ptr(info)))
        return Cm, eps, float(info[0]), int(info[1])

    def mo_operator(self, Cmo: np.ndarray):
        """(h, chol) of the orbitals Cmo (nbf x nmo) in the tci_operator layout."""
        Cmo = np.ascontiguousarray(Cmo, dtype=np.float64)
        nmo = Cmo.shape[1]
        h = np.zeros((nmo, nmo))
        L = np.zeros((nmo * (nmo + 1) // 2, self.nchol))
        check(lib().tci_mo_operator(self._h, ptr(Cmo), nmo, ptr(h), ptr(L), self.nchol))
        return h, L

    def close(self):
        if getattr(self, "_h", None):
            lib().tci_integrals_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_molden(path: str):
    """Molecule, MO coefficients (nao x nmo), orbital energies and occupations
    from a Molden file ([Atoms] in Angs or AU, [GTO], [MO]; [5D] selects pure d)."""
    lines = open(path).read().splitlines()
    sec, cur = {}, None
    pure = False
    for ln in lines:
        m = re.match(r"\s*\[([^\]]+)\]\s*\(?(\w*)", ln)
        if m:
            cur = m.group(1).strip().lower()
            if cur in ("5d", "5d7f", "5d10f"):
                pure = True
            sec[cur] = {"unit": m.group(2).lower(), "lines": []}
            continue
        if cur:
            sec[cur]["lines"].append(ln)
    conv = ANGSTROM_IN_BOHR if sec["atoms"]["unit"].startswith("ang") else 1.0
    Z, xyz = [], []
    for ln in sec["atoms"]["lines"]:
        t = ln.split()
        if len(t) >= 6:
            Z.append(float(t[2]))
            xyz.append([float(x) * conv for x in t[3:6]])
    shells, atom = [], None
    g = sec["gto"]["lines"]
    k = 0
    Lmap = {"s": 0, "p": 1, "d": 2}
    while k < len(g):
        t = g[k].split()
        k += 1
        if not t:
            continue
        if all(x.isdigit() for x in t) and len(t) <= 2:
            atom = int(t[0]) - 1
            continue
        lt = t[0].lower()
        if lt not in Lmap:
            raise ValueError(f"unsupported shell type {t[0]!r} (s, p, d only)")
        nprim = int(t[1])
        ex, cf = [], []
        for _ in range(nprim):
            e, c = g[k].replace("D", "E").replace("d", "e").split()[:2]
            ex.append(float(e))
            cf.append(float(c))
            k += 1
        shells.append((atom, Lmap[lt], ex, cf))
    mos, ene, occ = [], [], []
    for ln in sec["mo"]["lines"]:
        s = ln.strip()
        if not s:
            continue
        if "=" in s:
            key, val = [x.strip() for x in s.split("=", 1)]
            if key.lower() == "ene":
                mos.append({})
                ene.append(float(val.replace("D", "E")))
            elif key.lower() == "occup":
                occ.append(float(val.replace("D", "E")))
            continue
        i, v = s.split()[:2]
        mos[-1][int(i)] = float(v.replace("D", "E"))
    mol = Molecule(Z, np.array(xyz), shells, pure)
    nao = mol.nbf
    Cm = np.zeros((nao, len(mos)))
    for j, m in enumerate(mos):
        for i, v in m.items():
            Cm[i - 1, j] = v
    return mol, Cm, np.array(ene), np.array(occ)


# ---- geometries of the benchmark molecules -------------------------------------------------------------

def water(r_angstrom: float = 0.9572, angle_deg: float = 104.52) -> Tuple[List[str], np.ndarray]:
    """H2O with O at the origin and the molecule in the xz plane (bohr)."""
    r = r_angstrom * ANGSTROM_IN_BOHR
    a = math.radians(angle_deg) / 2
    xyz = np.array([[0.0, 0.0, 0.0], [r * math.sin(a), 0.0, r * math.cos(a)], [-r * math.sin(a), 0.0, r * math.cos(a)]])
    return ["O", "H", "H"], xyz


def n_alkane(n_carbon: int = 8, cc: float = 1.53, ch: float = 1.09) -> Tuple[List[str], np.ndarray]:
    """All-trans (staggered) n-alkane C_nH_{2n+2} with tetrahedral angles (bohr): the carbon zigzag in the xy
    plane, two hydrogens per carbon above and below it, one more on each terminal carbon."""
    th = math.acos(-1.0 / 3.0)  # tetrahedral angle
    half = th / 2
    dx, dy = cc * math.sin(half), cc * math.cos(half)
    carbons = [np.array([i * dx, (0.0 if i % 2 == 0 else dy), 0.0]) for i in range(n_carbon)]
    sym, pos = [], []
    for c in carbons:
        sym.append("C")
        pos.append(c)
    for i, c in enumerate(carbons):
        nb = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < n_carbon]
        u = [(b - c) / np.linalg.norm(b - c) for b in nb]
        if len(u) == 2:
            bis = -(u[0] + u[1])
            bis /= np.linalg.norm(bis)
            perp = np.array([0.0, 0.0, 1.0])
            # two H in the plane spanned by the bisector and z, at the tetrahedral angle
            for s in (1.0, -1.0):
                d = math.cos(th / 2) * bis + s * math.sin(th / 2) * perp
                sym.append("H")
                pos.append(c + ch * d / np.linalg.norm(d))
        else:
            a = -u[0]
            # staggered methyl: one H in the carbon plane opposite the zigzag, two out of plane
            y = np.array([0.0, 1.0 if i % 2 == 0 else -1.0, 0.0])
            y -= (y @ a) * a
            y /= np.linalg.norm(y)
            z = np.cross(a, y)
            ct, st = math.cos(math.pi - th), math.sin(math.pi - th)
            for phi in (0.0, 2 * math.pi / 3, 4 * math.pi / 3):
                d = ct * (-a) * -1.0 + st * (math.cos(phi) * (-y) + math.sin(phi) * z)
                sym.append("H")
                pos.append(c + ch * d / np.linalg.norm(d))
    order = [i for i, s in enumerate(sym) if s == "C"] + [i for i, s in enumerate(sym) if s == "H"]
    return [sym[i] for i in order], np.array([pos[i] for i in order]) * ANGSTROM_IN_BOHR


def h_chain(n: int, spacing_bohr: float) -> Tuple[List[str], np.ndarray]:
    """Linear H_n chain along z (bohr)."""
    return ["H"] * n, np.array([[0.0, 0.0, i * spacing_bohr] for i in range(n)])


# ---- MRSDCI problems of a molecule ---------------------------------------------------------------------

def cas_references(n_inactive: int, n_act_el: int, n_act_orb: int, spin_mult: int = 1) -> List[str]:
    """REFERENCE OCCUPATIONS of a complete active space: every occupation (0, 1, 2 per active orbital) with
    n_act_el electrons that can couple to the spin multiplicity, the inactive orbitals doubly occupied."""
    refs = []
    for occ in itertools.product((2, 1, 0), repeat=n_act_orb):
        if sum(occ) != n_act_el:
            continue
        singles = occ.count(1)
        if singles < spin_mult - 1 or (singles - (spin_mult - 1)) % 2:
            continue
        refs.append("2" * n_inactive + "".join(str(x) for x in occ))
    return refs


def mrsdci_problem(symbols, coords_bohr, basis: str = "cc-pVDZ", pure_d: bool = True, n_frozen: int = 0,
                   cas=(4, 4), spin_mult: int = 1, cd_threshold: float = 1e-6, refs=None):
    """Deck and MO operator of a CAS-reference MRSDCI on canonical RHF orbitals: AO integrals, pivoted
    Cholesky at cd_threshold, RHF, AO -> MO transform.  cas = (active electrons, active orbitals) taken
    from the top of the doubly occupied and the bottom of the virtual orbitals; the remaining doubly
    occupied orbitals are inactive, the lowest n_frozen of them frozen.  refs overrides the complete
    active space list.  Returns (Deck, Operator with the nuclear repulsion as core energy, info)."""
    from .api import Deck, Operator

    t0 = time.perf_counter()
    mol = Molecule.from_atoms(symbols, coords_bohr, basis, pure_d=pure_d)
    it = Integrals(mol, cd_threshold)
    t1 = time.perf_counter()
    nel = mol.n_electrons
    if nel % 2:
        raise ValueError("closed-shell RHF orbitals need an even number of electrons")
    nocc = nel // 2
    Cm, eps, e_scf, n_scf = it.rhf(nocc)
    t2 = time.perf_counter()
    h, L = it.mo_operator(Cm)
    t3 = time.perf_counter()
    n_act_el, n_act = cas
    n_inactive = nocc - n_act_el // 2
    if n_act_el % 2 or n_inactive < n_frozen or n_inactive + n_act > it.nbf:
        raise ValueError("inconsistent active space")
    refs = list(refs) if refs is not None else cas_references(n_inactive, n_act_el, n_act, spin_mult)
    deck = Deck(it.nbf, n_inactive, n_act, nel, spin_mult, refs, num_frozen=n_frozen)
    op = Operator(h, L, it.nuclear_repulsion)
    info = {"nbf": it.nbf, "nchol": it.nchol, "e_scf": e_scf, "scf_iterations": n_scf, "n_refs": len(refs),
            "seconds": {"integrals_cholesky": t1 - t0, "scf": t2 - t1, "mo_transform": t3 - t2}}
    it.close()
    return deck, op, info


def water_c1(cd_threshold: float = 1e-6):
    """H2O (R(O-H) 0.9572 A, HOH 104.52 deg), cc-pVDZ (24 functions), O 1s frozen, CAS(4,4) on canonical RHF
    orbitals (19 references), singlet."""
    sym, xyz = water()
    return mrsdci_problem(sym, xyz, "cc-pVDZ", pure_d=True, n_frozen=1, cas=(4, 4), cd_threshold=cd_threshold)


# Reference selection of the octane problem: the CAS(8,8) over the four highest doubly occupied and four lowest
# virtual RHF orbitals has 1107 singlet occupations, whose MRSDCI space no device holds; the references are the
# RHF occupation and the HOMO^2 -> LUMO^2 pair excitation within that active space (17,840,355 CSFs).
OCTANE_REFS = ("22220000", "22202000")


def octane_c3(cd_threshold: float = 1e-6):
    """All-trans n-octane (C-C 1.53 A, C-H 1.09 A, tetrahedral, staggered), cc-pVDZ (202 functions), the 8 C 1s
    frozen, CAS(8,8) active orbitals on canonical RHF orbitals with the references OCTANE_REFS, singlet."""
    sym, xyz = n_alkane(8)
    n_inactive = 33 - 4
    return mrsdci_problem(sym, xyz, "cc-pVDZ", pure_d=True, n_frozen=8, cas=(8, 8), cd_threshold=cd_threshold,
                          refs=["2" * n_inactive + r for r in OCTANE_REFS])
