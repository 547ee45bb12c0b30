"""Helpers of the local-deck tests: the injection of a local CSF space into the non-local space of the same
deck, from the product's local index vectors and the oracle's non-local layout."""
import numpy as np

import tigerci_b200 as T


def injection(loc_deck, nm1, nm2, osp, n):
    """Local CSF index -> non-local CSF index, from the product's local index vectors and the oracle's
    non-local layout."""
    sp = T.CsfSpace(loc_deck)
    c = sp.counts()
    P = np.full(c["total_csfs"], -1, dtype=np.int64)
    nab = n * (n - 1) // 2
    for kind, npaths in ((0, c["paths_v"]), (1, c["paths_nm1"]), (2, c["paths_nm2"])):
        off = sp.index_vector(kind)
        off_aa = sp.index_vector(3) if kind == 2 else None
        for lex in range(1, npaths + 1):
            _, info = sp.path(kind, lex)
            g = osp.paths[kind][lex - 1]
            if kind == 0:
                if off[lex - 1] > 0:
                    for k in range(info["nsf"]):
                        P[off[lex - 1] - 1 + k] = g["off"] + k
                continue
            d = (nm1 if kind == 1 else nm2)[lex - 1]
            if d == [-1]:
                continue
            m = len(d)
            if kind == 1:
                if off[lex - 1] > 0:
                    for k in range(info["nsf"]):
                        for a in range(m):
                            P[off[lex - 1] - 1 + k * m + a] = g["off"] + k * n + d[a]
                continue
            mab = m * (m - 1) // 2
            if off[lex - 1] > 0 and mab > 0:
                for k in range(info["nsf"]):
                    for i in range(1, m):
                        for j in range(i):
                            P[off[lex - 1] - 1 + k * mab + i * (i - 1) // 2 + j] = \
                                g["off"] + k * nab + d[i] * (d[i] - 1) // 2 + d[j]
            if off_aa[lex - 1] > 0:
                for k in range(info["nsf_aa"]):
                    for a in range(m):
                        P[off_aa[lex - 1] - 1 + k * m + a] = g["off_aa"] + k * n + d[a]
    assert (P >= 0).all()
    return P
