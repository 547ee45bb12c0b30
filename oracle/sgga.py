"""Oracle (test infrastructure only): CPU restatement of TigerCI's CSF space
and spin package, used to check the product's CSF indexing and spin basis.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module; the product never imports it.

Restated routines (paths relative to ``tiger_ci/tiger_fortran``):
  get_fsn ................ graph_mod.f90:381-491
  graph_border ........... graph_mod.f90:101-259
  drt_maker .............. graph_mod.f90:263-378 (+ ci_utilities_mod.f90:49-124)
  tree_search_internal ... graph_mod.f90:572-1003 (written recursively here)
  index_vector_internal .. graph_mod.f90:1007-1589
  branching_diagram ...... spin_mod.f90:99-228
  sft_graph .............. spin_mod.f90:232-522
  make_cycles ............ spin_mod.f90:526-684
  make_transpositions .... spin_mod.f90:688-830
Pinned by the CSF counts printed in the reference regression outputs
(tests/golden/csf_counts.json, generated by tests/golden/make_golden.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

KILL = -1000000
FSN_SIZE = 150
EXILEVEL = 2


@dataclass
class Deck:
    num_orbitals: int
    num_inactive: int
    num_active: int
    num_elec: int
    spin_mult: int
    refs: list  # list of strings/lists of internal occupations
    num_frozen: int = 0

    @property
    def num_internal(self):
        return self.num_inactive + self.num_active

    def ref_matrix(self):
        return [[int(c) for c in r] for r in self.refs]


def get_fsn(deck):
    refs = deck.ref_matrix()
    os_ = 0
    for r in refs:
        ref_singles = sum(1 for j in range(deck.num_inactive, deck.num_inactive + deck.num_active) if r[j] == 1)
        os_ = max(ref_singles + 4, os_)
    if deck.num_elec < os_:
        os_ = deck.num_elec
    if deck.spin_mult % 2 == 0 and os_ % 2 == 0:
        os_ += 1
    fsn = [0] * (FSN_SIZE + 1)
    fsn3 = [0] * (os_ + 3)
    fsn[0] = 1
    fsn3[0] = 1
    fsn3[1] = 1
    for i in range(1, os_ + 1):
        for j in range(i % 2 + 1, i + 2, 2):
            if j == 1:
                nf = fsn3[2]
            elif j == i + 1:
                nf = 1
            else:
                nf = fsn3[j - 1] + fsn3[j + 1]
            fsn3[j] = nf
        fsn[i] = fsn3[deck.spin_mult] if deck.spin_mult < len(fsn3) else 0
    return os_, fsn


@dataclass
class Space:
    deck: Deck
    open_shells: int
    fsn: list
    total_configurations: int
    paths: dict = field(default_factory=dict)  # k -> list of dict(occ, singles, kept...)
    counts: dict = field(default_factory=dict)  # k -> {singles: configurations}
    num_valence: int = 0
    num_nm1: int = 0
    num_nm2: int = 0
    total_csfs: int = 0
    removed: int = 0


def build_space(deck: Deck, nm1_nvirt=None, nm2_nvirt=None) -> Space:
    """Restates graph_border, drt_maker, tree_search_internal and
    index_vector_internal.  ``nm1_nvirt``/``nm2_nvirt`` give per-path virtual
    counts for local runs (default: every external orbital)."""
    norb, nint, nel = deck.num_orbitals, deck.num_internal, deck.num_elec
    next_ = norb - nint
    refs = deck.ref_matrix()
    os_, fsn = get_fsn(deck)
    spinM = deck.spin_mult
    # graph_border
    min_s = spinM - 1
    r_s, r_d = min_s, (nel - min_s) // 2
    l_s = max(0, min_s)
    l_d = (nel - l_s) // 2
    l_u = norb - l_s - l_d
    lb = [0] * (norb + 1)
    rb = [0] * (norb + 1)
    for i in range(1, norb + 1):
        add = 0 if i <= l_u else (1 if i <= l_u + l_s else 2)
        lb[i] = add if i == 1 else lb[i - 1] + add
        add = 2 if i <= r_d else (1 if i <= r_d + r_s else 0)
        rb[i] = add if i == 1 else rb[i - 1] + add

    def refocc(o1, r):
        return refs[r][o1 - 1] if o1 <= nint else 0

    temp = [refocc(1, r) for r in range(len(refs))]
    for i in range(2, norb + 1):
        mn, mx = 2 * i, 0
        for r in range(len(refs)):
            c = temp[r] + refocc(i, r)
            mx, mn = max(mx, c), min(mn, c)
            temp[r] = c
        lb[i] = max(mn - EXILEVEL, lb[i])
        rb[i] = min(mx + EXILEVEL, rb[i])
    aux = [0] * (norb + 1)
    nv = 1
    aux[0] = 1
    for i in range(1, norb + 1):
        aux[i] = nv + 1 - lb[i]
        nv = rb[i] + aux[i]

    def belong(i, j):
        if i < 0 or j < 0 or i > norb:
            return False
        return lb[i] <= j <= rb[i]

    def vtx(i, j):
        return aux[i] + j

    y0 = [0] * (nv + 2)
    y1 = [0] * (nv + 2)
    y2 = [0] * (nv + 2)

    def add0(i, j):
        return i >= 0 and j >= 0 and belong(i, j) and y0[vtx(i, j)] > 0

    def add1(i, j):
        return i >= 0 and j >= 0 and belong(i, j) and y1[vtx(i, j)] >= 0

    def add2(i, j):
        return i >= 0 and j >= 0 and belong(i, j) and y2[vtx(i, j)] >= 0

    y0[1] = 1 if belong(1, 0) else -1
    y1[1] = 0 if belong(1, 1) else -1
    y2[1] = 0 if belong(1, 2) else -1
    for i in range(1, norb + 1):
        for j in range(rb[i], lb[i] - 1, -1):
            va, v = vtx(i - 1, j), vtx(i, j)
            w = 0
            if add0(i - 1, j):
                w += abs(y0[va])
            if add1(i - 1, j - 1):
                w += abs(y0[va - 1])
            if add2(i - 1, j - 2):
                w += abs(y0[va - 2])
            y0[v] = w if belong(i + 1, j) else -w
            if not belong(i + 1, j + 1):
                w = -1
            else:
                w = abs(y0[vtx(i, j + 1)]) if add0(i, j + 1) else 0
            y1[v] = w
            if not belong(i + 1, j + 2):
                w = -1
            else:
                w = 0
                if add1(i, j + 1):
                    w += abs(y0[vtx(i, j + 1)])
                if add0(i, j + 2):
                    w += abs(y0[vtx(i, j + 2)])
            y2[v] = w
    sp = Space(deck, os_, fsn, abs(y0[nv]))

    # tree search: enumerate internal paths with their lexical index
    heads = {0: {}, 1: {}, 2: {}}

    def walk(level, elec, vert, lex, occ):
        if level == nint:
            k = nel - elec
            heads[k][lex] = list(occ)
            return
        for step, arcs in ((2, y2), (1, y1), (0, y0)):
            arc = arcs[vert]
            if arc < 0:
                continue
            ne = elec + step
            walk(level + 1, ne, aux[level + 1] + ne, lex + (arc if step else 0), occ + [step])

    walk(0, 0, 1, 1, [])

    def keep(occ, k):
        for r in refs:
            diff = sum(abs(a - b) for a, b in zip(occ, r)) + k
            if diff <= 2 * EXILEVEL:
                break
        else:
            return False
        return all(occ[j] == 2 for j in range(deck.num_frozen))

    shell1 = os_ % 2
    shellU = shell1 + 1
    for k in range(3):
        n = abs(y0[vtx(nint, nel - k)]) if belong(nint, nel - k) else 0
        sp.paths[k] = []
        for lex in range(1, n + 1):
            occ = heads[k].get(lex)
            singles = sum(1 for o in occ if o == 1) if occ is not None else 0
            ok = occ is not None and keep(occ, k)
            sp.paths[k].append(dict(lex=lex, occ=occ, singles=singles, raw=singles if ok else KILL))

    def nvirt(k, p):
        lst = nm1_nvirt if k == 1 else nm2_nvirt
        return next_ if lst is None else lst[p]

    tmp = {}

    def T(i):
        return tmp.get(i, 0)

    # valence
    tmp.clear()
    for h in sp.paths[0]:
        s = h["raw"]
        if s < spinM - 1 or s > os_:
            s = shellU
        h["iv"] = s
        tmp[s] = T(s) + 1
    sp.removed = T(shellU)
    sp.counts[0] = {i: T(i) for i in range(spinM - 1, os_ + 1, 2) if T(i) > 0}
    n = sum(T(i) * fsn[i] for i in range(spinM - 1, os_ + 1, 2))
    sp.num_valence = sp.total_csfs = n
    tmp[shellU] = -1
    fsn[shellU] = 0
    c = 1
    for i in range(shell1, os_ + 1, 2):
        cf = T(i)
        tmp[i] = c
        c += cf * fsn[i]
    for h in sp.paths[0]:
        s = h["iv"]
        if s == shellU:
            h["off"], h["nsf"] = None, 0
        else:
            h["off"], h["nsf"] = tmp[s] - 1, fsn[s]
            tmp[s] += fsn[s]
    # N-1
    tmp.clear()
    for p, h in enumerate(sp.paths[1]):
        s = h["raw"]
        if s + 1 < spinM - 1 or s + 1 > os_:
            s = shellU - 1
        h["iv"] = s
        tmp[s + 1] = T(s + 1) + nvirt(1, p)
    sp.removed += T(shellU)
    sp.counts[1] = {i: T(i) for i in range(spinM - 1, os_ + 1, 2) if T(i) > 0}
    sp.total_csfs += sum(T(i) * fsn[i] for i in range(spinM - 1, os_ + 1, 2))
    fsn[shellU] = 0
    start = sp.num_valence + 1
    for p, h in enumerate(sp.paths[1]):
        s = h["iv"] + 1
        if s == shellU:
            h["off"], h["nsf"] = None, 0
        else:
            h["off"], h["nsf"] = start - 1, fsn[s]
            start += fsn[s] * nvirt(1, p)
    sp.num_nm1 = start - sp.num_valence - 1
    # N-2
    tmp.clear()
    for p, h in enumerate(sp.paths[2]):
        s2 = s3 = h["raw"]
        if s2 + 2 < spinM - 1 or s2 + 2 > os_:
            s2 = shellU - 2
        nvv = nvirt(2, p)
        tmp[s2 + 2] = T(s2 + 2) + nvv * (nvv - 1) // 2
        if s3 < spinM - 1 or s3 > os_:
            s3 = shellU
        tmp[s3] = T(s3) + nvv
        h["iv2"], h["iv3"] = s2, s3
    sp.removed += T(shellU)
    sp.counts[2] = {i: T(i) for i in range(spinM - 1, os_ + 1, 2) if T(i) > 0}
    sp.total_csfs += sum(T(i) * fsn[i] for i in range(spinM - 1, os_ + 1, 2))
    fsn[shellU] = 0
    start = sp.num_valence + sp.num_nm1 + 1
    for p, h in enumerate(sp.paths[2]):
        nvv = nvirt(2, p)
        s = h["iv3"]
        if s == shellU:
            h["off_aa"], h["nsf_aa"] = None, 0
        else:
            h["off_aa"], h["nsf_aa"] = start - 1, fsn[s]
            start += fsn[s] * nvv
        s = h["iv2"] + 2
        if s == shellU:
            h["off"], h["nsf"] = None, 0
        else:
            h["off"], h["nsf"] = start - 1, fsn[s]
            start += fsn[s] * (nvv * (nvv - 1) // 2)
    sp.num_nm2 = start - sp.num_valence - sp.num_nm1 - 1
    for i in range(0, spinM - 1):
        fsn[i] = 0
    for i in range(spinM, os_, 2):
        fsn[i] = 0
    for i in range(os_ + 1, FSN_SIZE + 1):
        fsn[i] = 0
    return sp


# ---------------------------------------------------------------------------
# spin package


def branching_diagram(open_shells, spinM):
    up = (open_shells + spinM - 1) // 2
    down = open_shells - up
    B = np.zeros((up + 2, down + 3), dtype=np.int64)
    a, b, amax, bmax = up, down + 1, up, down + 1
    while True:
        if a == up and b == down + 1:
            B[a, b] = 1
        elif b == down + 1 or a + 1 == b:
            B[a, b] = B[a + 1, b]
        elif b == 1 and a < up:
            B[a, b] = B[a + 1, b] + B[a, b + 1]
        elif a == up:
            B[a, b] = 1
        else:
            B[a, b] = B[a + 1, b] + B[a, b + 1]
        if a == 1 and b == 1:
            break
        if b == down + 1 or a + 1 == b or a == b:
            if bmax > 1 and amax == up:
                bmax -= 1
            elif bmax == 1 and amax <= up:
                amax -= 1
            a, b = amax, bmax
        else:
            a, b = a - 1, b + 1
    return B, up, down


def sft_graph(open_shells, spinM, nsf):
    """Returns (sft[arc-1][w-1], spin_matrix[v][w-1])."""
    B, up, down = branching_diagram(open_shells, spinM)
    sft = np.zeros((max(open_shells - 1, 0), nsf), dtype=np.int64)
    sm = np.zeros((open_shells + 1, nsf), dtype=np.int64)
    path = [False] * (open_shells + 1)
    pa = [0] * (open_shells + 1)
    pb = [0] * (open_shells + 1)
    path[open_shells] = True
    shells = open_shells - 1
    pa[open_shells], pb[open_shells] = 0, 1
    pa[shells], pb[shells] = 1, 1
    weight = 1
    sm[0, :] = spinM
    sm[open_shells, :] = 1
    while True:
        while True:
            if pa[shells] == up and pb[shells] == down + 1 and shells == 0:
                break
            if pb[shells] == down + 1 or pb[shells] == pa[shells] + 1:
                path[shells] = True
                shells -= 1
                pa[shells], pb[shells] = pa[shells + 1] + 1, pb[shells + 1]
            else:
                path[shells] = False
                shells -= 1
                pa[shells], pb[shells] = pa[shells + 1], pb[shells + 1] + 1
        W = weight - 1
        for i in range(open_shells - 1, 0, -1):
            prev, cur = path[i + 1], path[i]
            a, b = pa[i], pb[i]
            sm[i, W] = sm[i + 1, W] + (1 if prev else -1)
            if prev and not cur and a == b:
                sft[i - 1, W] = weight
            elif prev and not cur:
                nw = weight - B[a - 1, b + 1]
                if b + 2 <= down + 1:
                    nw += B[a - 1, b + 2]
                sft[i - 1, W] = nw
            elif (not prev) and cur:
                nw = weight + B[a, b]
                if b <= a and b < down + 1:
                    nw -= B[a, b + 1]
                sft[i - 1, W] = -nw
            else:
                sft[i - 1, W] = 0
        shells = 1
        done = False
        while True:
            if shells == open_shells:
                done = True
                break
            if not path[shells] and pa[shells] < up:
                path[shells] = True
                weight += B[pa[shells], pb[shells] + 1]
                shells -= 1
                pa[shells], pb[shells] = pa[shells + 1] + 1, pb[shells + 1]
                break
            shells += 1
            if pb[shells] < down + 1 and pb[shells] <= pa[shells] and path[shells]:
                weight -= B[pa[shells], pb[shells] + 1]
        if done:
            break
    return sft, sm


def make_cycles(open_shells, nsf, sft, sm):
    """cycles[label] (nsf x nsf) for the cycles (l..k), label=(k-1)(k-2)/2+l."""
    ncyc = open_shells * (open_shells - 1) // 2
    cyc = np.zeros((ncyc + 1, nsf, nsf))
    for i in range(nsf):
        for k in range(2, open_shells + 1):
            reorder = [i]
            col = [1.0]
            for l in range(k - 1, 0, -1):
                label = (k - 1) * (k - 2) // 2 + l
                nstates = len(reorder)
                for j in range(nstates):
                    mult = sm[l + 1, reorder[j]]
                    akl = 1.0 / mult
                    net = col[j]
                    v = sft[l - 1, reorder[j]]
                    if v == 0:
                        col[j] = -col[j]
                    elif v > 0:
                        col[j] = akl * net
                        if v != reorder[j] + 1:
                            reorder.append(abs(v) - 1)
                            col.append(-math.sqrt(1.0 - akl * akl) * net)
                    else:
                        col[j] = -akl * net
                        reorder.append(abs(v) - 1)
                        col.append(-math.sqrt(1.0 - akl * akl) * net)
                for j in range(len(reorder)):
                    val = col[j] if abs(col[j]) >= 1e-9 else 0.0
                    cyc[label, reorder[j], i] = val
    return cyc


def make_transpositions(open_shells, nsf, cyc):
    """Full (symmetric) matrices of the transpositions (i,j), i>j, keyed (i,j)."""
    out = {}
    for i in range(1, open_shells):
        lab = i * (i - 1) // 2 + i
        m = np.tril(cyc[lab])
        out[(i + 1, i)] = m + np.tril(m, -1).T
    for i in range(3, open_shells + 1):
        for j in range(i - 2, 0, -1):
            lab = (i - 1) * (i - 2) // 2 + j + 1
            c1t = cyc[lab].T
            c2 = cyc[lab - 1]
            t = c1t @ c2
            m = np.tril(t)
            out[(i, j)] = m + np.tril(m, -1).T
    return out


def spin_tables(open_shells, spinM):
    fsn3 = [0] * (open_shells + 3)
    fsn3[0] = fsn3[1] = 1
    fsn_all = [0] * (open_shells + 1)
    fsn_all[0] = 1 if spinM == 1 else 0
    for i in range(1, open_shells + 1):
        for j in range(i % 2 + 1, i + 2, 2):
            fsn3[j] = fsn3[2] if j == 1 else (1 if j == i + 1 else fsn3[j - 1] + fsn3[j + 1])
        ok = i >= spinM - 1 and (i - spinM + 1) % 2 == 0
        fsn_all[i] = (fsn3[spinM] if spinM < len(fsn3) else 0) if ok else 0
    nsf = fsn_all[open_shells]
    sft, sm = sft_graph(open_shells, spinM, nsf)
    return fsn_all, sft, sm


def yk_expansion(sm, s, nsf_s, spinM):
    """Genealogical coefficients of the first nsf_s SFT functions over spin
    strings of s open shells (bit i set = beta on arc i+1), M_S = S."""
    nbeta = (s - (spinM - 1)) // 2
    strings = [x for x in range(1 << s) if bin(x).count("1") == nbeta]
    theta = np.zeros((len(strings), nsf_s))
    for f in range(nsf_s):
        assert sm[s, f] == 1, "padding pairs expected on arcs above s"
        for r, x in enumerate(strings):
            c, M, S = 1.0, 0.0, 0.0
            for arc in range(s, 0, -1):
                m = -0.5 if (x >> (arc - 1)) & 1 else 0.5
                Sp = 0.5 * (sm[arc - 1, f] - 1)
                Mp = M + m
                if abs(Mp) > Sp + 1e-9:
                    c = 0.0
                    break
                den = 2 * S + 1
                if Sp > S:
                    cg = math.sqrt((S + Mp + 0.5) / den) if m > 0 else math.sqrt((S - Mp + 0.5) / den)
                else:
                    cg = -math.sqrt((S - Mp + 0.5) / den) if m > 0 else math.sqrt((S + Mp + 0.5) / den)
                c *= cg
                S, M = Sp, Mp
            theta[r, f] = c
    return strings, theta
