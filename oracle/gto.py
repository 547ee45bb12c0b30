"""Test infrastructure only: Gaussian-orbital integrals and a Molden reader for
golden fixtures.  Nothing in the product imports this module.

The reference computes its AO integrals with libint (absent from its tree) after
reading the MO coefficients from a Molden file (`tiger_cpp/OrbitalParsers.cpp`
`MoldenOrbitalParser`, coordinates in Angstrom converted with ANGSTROMINBOHR =
1.8897261 from `erkale/global.h:76`).  To pin the sigma/energy path against the
energies that the reference's regression runs print, this module restates the
published McMurchie-Davidson scheme (L. E. McMurchie and E. R. Davidson,
J. Comput. Phys. 26, 218 (1978)) for Cartesian Gaussians:

- Hermite expansion coefficients E^{ij}_t of a product of two 1D Gaussians,
- overlap and kinetic energy from the E coefficients (kinetic via the second
  derivative of the ket Gaussian),
- Hermite Coulomb integrals R^n_{tuv} with the Boys function
  F_n(T) = Gamma(n+1/2) P(n+1/2, T) / (2 T^(n+1/2)) (P the regularised lower
  incomplete gamma function), for nuclear attraction and electron repulsion.

Contracted functions use normalised primitives (Molden / Gaussian basis-set
convention) and are renormalised to unit self-overlap per Cartesian component.
Cartesian components of a shell are ordered x, y, z for p (Molden order).
Plain Python loops: meant for bases of a few dozen functions.
"""
from __future__ import annotations

import math
import re
from functools import lru_cache

import numpy as np
from scipy.special import gammainc, gamma

ANGSTROM_IN_BOHR = 1.8897261  # erkale/global.h:76, used by MoldenOrbitalParser::readCoordinates

_CART = {0: [(0, 0, 0)], 1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
         2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)]}  # Molden d order: xx yy zz xy xz yz
_L = {"s": 0, "p": 1, "d": 2}


def boys(n: int, T: float) -> float:
    if T < 1e-12:
        return 1.0 / (2 * n + 1) - T / (2 * n + 3)
    a = n + 0.5
    return gamma(a) * gammainc(a, T) / (2.0 * T ** a)


def _dfact(k: int) -> float:
    r = 1.0
    while k > 1:
        r *= k
        k -= 2
    return r


def prim_norm(alpha: float, lmn) -> float:
    l, m, n = lmn
    L = l + m + n
    return (2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (L / 2) / math.sqrt(
        _dfact(2 * l - 1) * _dfact(2 * m - 1) * _dfact(2 * n - 1))


def hermite_e(i: int, j: int, t: int, Xab: float, a: float, b: float) -> float:
    """E^{ij}_t for exponents a (centre A) and b (centre B), Xab = A - B."""
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return math.exp(-q * Xab * Xab)
    if j == 0:  # lower i
        return (hermite_e(i - 1, j, t - 1, Xab, a, b) / (2 * p) - (q * Xab / a) * hermite_e(i - 1, j, t, Xab, a, b)
                + (t + 1) * hermite_e(i - 1, j, t + 1, Xab, a, b))
    return (hermite_e(i, j - 1, t - 1, Xab, a, b) / (2 * p) + (q * Xab / b) * hermite_e(i, j - 1, t, Xab, a, b)
            + (t + 1) * hermite_e(i, j - 1, t + 1, Xab, a, b))


def hermite_r(t: int, u: int, v: int, n: int, p: float, X: float, Y: float, Z: float, cache) -> float:
    """R^n_{tuv}(p, P - C)."""
    key = (t, u, v, n)
    if key in cache:
        return cache[key]
    if t < 0 or u < 0 or v < 0:
        return 0.0
    if t == u == v == 0:
        val = (-2 * p) ** n * boys(n, p * (X * X + Y * Y + Z * Z))
    elif t > 0:
        val = (t - 1) * hermite_r(t - 2, u, v, n + 1, p, X, Y, Z, cache) + X * hermite_r(t - 1, u, v, n + 1, p, X, Y, Z, cache)
    elif u > 0:
        val = (u - 1) * hermite_r(t, u - 2, v, n + 1, p, X, Y, Z, cache) + Y * hermite_r(t, u - 1, v, n + 1, p, X, Y, Z, cache)
    else:
        val = (v - 1) * hermite_r(t, u, v - 2, n + 1, p, X, Y, Z, cache) + Z * hermite_r(t, u, v - 1, n + 1, p, X, Y, Z, cache)
    cache[key] = val
    return val


class Basis:
    """Contracted Cartesian functions: list of (centre, lmn, exponents, coefficients incl. norms)."""

    def __init__(self, atoms, shells):
        self.atoms = atoms  # list of (Z, xyz in bohr)
        self.funcs = []
        for centre, L, exps, coefs in shells:
            for lmn in _CART[L]:
                c = np.array([cf * prim_norm(a, lmn) for a, cf in zip(exps, coefs)])
                f = (np.asarray(centre, float), lmn, np.asarray(exps, float), c)
                s = _overlap_prim_sum(f, f)
                self.funcs.append((f[0], lmn, f[2], c / math.sqrt(s)))

    def __len__(self):
        return len(self.funcs)


def _overlap_1d(i, j, Xab, a, b):
    return hermite_e(i, j, 0, Xab, a, b) * math.sqrt(math.pi / (a + b))


def _overlap_prim_sum(fa, fb):
    A, la, ea, ca = fa
    B, lb, eb, cb = fb
    s = 0.0
    for a, cA in zip(ea, ca):
        for b, cB in zip(eb, cb):
            v = 1.0
            for k in range(3):
                v *= _overlap_1d(la[k], lb[k], A[k] - B[k], a, b)
            s += cA * cB * v
    return s


def overlap(basis: Basis) -> np.ndarray:
    n = len(basis)
    S = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1):
            S[i, j] = S[j, i] = _overlap_prim_sum(basis.funcs[i], basis.funcs[j])
    return S


def kinetic(basis: Basis) -> np.ndarray:
    n = len(basis)
    T = np.zeros((n, n))
    for i in range(n):
        A, la, ea, ca = basis.funcs[i]
        for j in range(i + 1):
            B, lb, eb, cb = basis.funcs[j]
            tot = 0.0
            for a, cA in zip(ea, ca):
                for b, cB in zip(eb, cb):
                    s = [_overlap_1d(la[k], lb[k], A[k] - B[k], a, b) for k in range(3)]
                    t = []
                    for k in range(3):
                        l2 = lb[k]
                        d2 = (4 * b * b * _overlap_1d(la[k], l2 + 2, A[k] - B[k], a, b)
                              - 2 * b * (2 * l2 + 1) * _overlap_1d(la[k], l2, A[k] - B[k], a, b))
                        if l2 >= 2:
                            d2 += l2 * (l2 - 1) * _overlap_1d(la[k], l2 - 2, A[k] - B[k], a, b)
                        t.append(-0.5 * d2)
                    tot += cA * cB * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2])
            T[i, j] = T[j, i] = tot
    return T


def nuclear(basis: Basis) -> np.ndarray:
    n = len(basis)
    V = np.zeros((n, n))
    for i in range(n):
        A, la, ea, ca = basis.funcs[i]
        for j in range(i + 1):
            B, lb, eb, cb = basis.funcs[j]
            tot = 0.0
            for a, cA in zip(ea, ca):
                for b, cB in zip(eb, cb):
                    p = a + b
                    P = (a * A + b * B) / p
                    for Zc, C in basis.atoms:
                        cache = {}
                        acc = 0.0
                        for t in range(la[0] + lb[0] + 1):
                            Et = hermite_e(la[0], lb[0], t, A[0] - B[0], a, b)
                            for u in range(la[1] + lb[1] + 1):
                                Eu = hermite_e(la[1], lb[1], u, A[1] - B[1], a, b)
                                for v in range(la[2] + lb[2] + 1):
                                    Ev = hermite_e(la[2], lb[2], v, A[2] - B[2], a, b)
                                    acc += Et * Eu * Ev * hermite_r(t, u, v, 0, p, *(P - C), cache)
                        tot += cA * cB * (-Zc) * 2 * math.pi / p * acc
            V[i, j] = V[j, i] = tot
    return V


def _eri_prim(fa, fb, fc, fd):
    A, la, ea, ca = fa
    B, lb, eb, cb = fb
    C, lc, ec, cc = fc
    D, ld, ed, cd = fd
    tot = 0.0
    for a, cA in zip(ea, ca):
        for b, cB in zip(eb, cb):
            p = a + b
            P = (a * A + b * B) / p
            Eab = [[hermite_e(la[k], lb[k], t, A[k] - B[k], a, b) for t in range(la[k] + lb[k] + 1)] for k in range(3)]
            for c, cC in zip(ec, cc):
                for d, cD in zip(ed, cd):
                    q = c + d
                    Q = (c * C + d * D) / q
                    alpha = p * q / (p + q)
                    Ecd = [[hermite_e(lc[k], ld[k], t, C[k] - D[k], c, d) for t in range(lc[k] + ld[k] + 1)]
                           for k in range(3)]
                    cache = {}
                    PQ = P - Q
                    acc = 0.0
                    for t, et in enumerate(Eab[0]):
                        for u, eu in enumerate(Eab[1]):
                            for v, ev in enumerate(Eab[2]):
                                e1 = et * eu * ev
                                for tau, ft in enumerate(Ecd[0]):
                                    for nu, fu in enumerate(Ecd[1]):
                                        for phi, fv in enumerate(Ecd[2]):
                                            sign = -1.0 if (tau + nu + phi) % 2 else 1.0
                                            acc += e1 * sign * ft * fu * fv * hermite_r(t + tau, u + nu, v + phi, 0, alpha,
                                                                                       *PQ, cache)
                    tot += cA * cB * cC * cD * 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * acc
    return tot


def eri(basis: Basis) -> np.ndarray:
    """(ij|kl), chemists' notation, full 4-index array (8-fold symmetry used)."""
    n = len(basis)
    G = np.zeros((n, n, n, n))
    f = basis.funcs
    for i in range(n):
        for j in range(i + 1):
            ij = i * (i + 1) // 2 + j
            for k in range(n):
                for l in range(k + 1):
                    if k * (k + 1) // 2 + l > ij:
                        continue
                    v = _eri_prim(f[i], f[j], f[k], f[l])
                    for (a, b) in ((i, j), (j, i)):
                        for (c, d) in ((k, l), (l, k)):
                            G[a, b, c, d] = v
                            G[c, d, a, b] = v
    return G


def nuclear_repulsion(atoms) -> float:
    e = 0.0
    for x in range(len(atoms)):
        for y in range(x):
            e += atoms[x][0] * atoms[y][0] / np.linalg.norm(np.asarray(atoms[x][1]) - np.asarray(atoms[y][1]))
    return e


def molden_is_pure(path: str) -> bool:
    """True when the Molden file declares pure (spherical) d functions ([5D], [5D7F] or [5D10F])."""
    return any(re.match(r"\s*\[5D(7F|10F)?\]", ln, re.I) for ln in open(path))


def read_molden(path: str):
    """Atoms (Z, bohr), shells (centre, L, exponents, coefficients) and MO coefficients (nao x nmo) with
    energies and occupations, from a Molden file with [Atoms], [GTO] and [MO] sections."""
    text = open(path).read().splitlines()
    sec = {}
    cur = None
    for ln in text:
        m = re.match(r"\s*\[(\w[\w ]*)\]\s*\(?(\w*)", ln)
        if m:
            cur = m.group(1).strip().lower()
            sec[cur] = {"unit": m.group(2).lower(), "lines": []}
            continue
        if cur:
            sec[cur]["lines"].append(ln)
    conv = ANGSTROM_IN_BOHR if sec["atoms"]["unit"].startswith("ang") else 1.0
    atoms = []
    for ln in sec["atoms"]["lines"]:
        t = ln.split()
        if len(t) >= 6:
            atoms.append((int(t[2]), [float(x) * conv for x in t[3:6]]))
    shells = []
    lines = [ln for ln in sec["gto"]["lines"]]
    k = 0
    centre = None
    while k < len(lines):
        t = lines[k].split()
        k += 1
        if not t:
            continue
        if len(t) <= 2 and t[0].isdigit() and all(x.isdigit() for x in t):
            centre = atoms[int(t[0]) - 1][1]
            continue
        if t[0].lower() in _L:
            L = _L[t[0].lower()]
            nprim = int(t[1])
            exps, coefs = [], []
            for _ in range(nprim):
                e, c = lines[k].replace("D", "E").replace("d", "e").split()[:2]
                exps.append(float(e))
                coefs.append(float(c))
                k += 1
            shells.append((centre, L, exps, coefs))
    mos, ene, occ = [], [], []
    cur_mo = None
    for ln in sec["mo"]["lines"]:
        s = ln.strip()
        if not s:
            continue
        if "=" in s:
            key, val = [x.strip() for x in s.split("=", 1)]
            if key.lower() == "ene":
                cur_mo = {}
                mos.append(cur_mo)
                ene.append(float(val))
            elif key.lower() == "occup":
                occ.append(float(val))
            continue
        i, v = s.split()[:2]
        cur_mo[int(i)] = float(v.replace("D", "E"))
    nao = max(max(m) for m in mos)
    C = np.zeros((nao, len(mos)))
    for j, m in enumerate(mos):
        for i, v in m.items():
            C[i - 1, j] = v
    return atoms, shells, C, np.array(ene), np.array(occ)


def mo_operator(atoms, shells, C, tol=1e-13):
    """h (MO), Cholesky vectors chol[pair, J] (pair = p(p+1)/2 + q, p >= q) of the MO (pq|rs) matrix by
    pivoted Cholesky to `tol`, and the nuclear repulsion."""
    bas = Basis(atoms, shells)
    h_ao = kinetic(bas) + nuclear(bas)
    g_ao = eri(bas)
    h = C.T @ h_ao @ C
    g = np.einsum("pi,qj,rk,sl,pqrs->ijkl", C, C, C, C, g_ao, optimize=True)
    n = C.shape[1]
    pairs = [(p, q) for p in range(n) for q in range(p + 1)]
    M = np.array([[g[p, q, r, s] for (r, s) in pairs] for (p, q) in pairs])
    L = pivoted_cholesky(M, tol)
    return h, L, nuclear_repulsion(atoms), overlap(bas)


def pivoted_cholesky(M: np.ndarray, tol: float) -> np.ndarray:
    M = np.array(M, dtype=np.float64)
    n = M.shape[0]
    d = np.diag(M).copy()
    cols = []
    while True:
        piv = int(np.argmax(d))
        if d[piv] <= tol:
            break
        col = M[:, piv].copy()
        for c in cols:
            col -= c * c[piv]
        col /= math.sqrt(d[piv])
        cols.append(col)
        d -= col * col
        d[piv] = 0.0
        if len(cols) == n:
            break
    return np.ascontiguousarray(np.array(cols).T)
