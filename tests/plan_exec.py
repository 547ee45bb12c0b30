"""Test-only numpy interpreter of an exported sigma plan.

Replays the same step tables the device executes (GEMM / AXPY / DOT /
UNPACK / PACK / ZERO / WBUILD) so the host-built plan can be checked against
the dense-Hamiltonian oracle on machines without a GPU.  Never used by the
product.
"""
from __future__ import annotations

import numpy as np

from tigerci_b200.plan_io import BUF_NAMES, PlanFile

SQ2 = np.sqrt(2.0)


def _bid(name):
    return BUF_NAMES.index(name)


class PlanInterpreter:
    def __init__(self, path, h, chol):
        self.pf = pf = PlanFile(path)
        self.bufs = [np.zeros(max(0, s), dtype=np.float64) for s in pf.buf_size]
        n, nint = pf.n, pf.nint
        self.bufs[_bid("L")][:] = np.asarray(chol, dtype=np.float64).reshape(-1)
        self.bufs[_bid("JK")][2 * nint * nint * n * n:] = pf.h_vv
        if len(pf.wv):
            self.bufs[_bid("WV")][:len(pf.wv)] = pf.wv
        for st in pf.init_steps:
            self.run(st)

    def view(self, b, off, shape, ld=None):
        buf = self.bufs[b]
        rows, cols = shape
        if ld is None:
            ld = cols
        if rows == 0 or cols == 0:
            return np.zeros(shape)
        return np.lib.stride_tricks.as_strided(buf[off:], shape=(rows, cols), strides=(ld * 8, 8))

    def run(self, st):
        k = st["kind"]
        pf = self.pf
        n = pf.n
        if k == "ZERO":
            self.bufs[st["buf"]][st["off"]:st["off"] + st["len"]] = 0.0
        elif k == "GEMM":
            for g in st["gp"]:
                acc = np.zeros((g["M"], g["N"]))
                for s in st["gs"][g["seg_begin"]:g["seg_end"]]:
                    A = self.view(s["a"], s["offA"], (s["K"], g["M"]) if s["tA"] else (g["M"], s["K"]), s["lda"])
                    B = self.view(s["b"], s["offB"], (g["N"], s["K"]) if s["tB"] else (s["K"], g["N"]), s["ldb"])
                    acc += s["alpha"] * ((A.T if s["tA"] else A) @ (B.T if s["tB"] else B))
                C = self.view(g["c"], g["offC"], (g["M"], g["N"]), g["ldc"])
                C[...] = (g["beta"] * C if g["beta"] != 0.0 else 0.0) + acc
        elif k == "AXPY":
            srcs = st["as_"]
            for t in st["at"]:
                acc = np.zeros(t["len"])
                for s in srcs[t["src_begin"]:t["src_end"]]:
                    c = s["coef"] * (self.bufs[s["sbuf"]][s["sidx"]] if s["sbuf"] >= 0 else 1.0)
                    acc += c * self.bufs[s["src"]][s["off"]:s["off"] + t["len"]]
                self.bufs[t["dst"]][t["off"]:t["off"] + t["len"]] += acc
        elif k == "DOT":
            srcs = st["ds"]
            for t in st["dt"]:
                tot = 0.0
                for s in srcs[t["src_begin"]:t["src_end"]]:
                    tot += s["coef"] * np.dot(self.bufs[s["a"]][s["aoff"]:s["aoff"] + s["len"]],
                                              self.bufs[s["b"]][s["boff"]:s["boff"] + s["len"]])
                self.bufs[t["dst"]][t["off"]] += tot
        elif k == "UNPACK":
            c = self.bufs[_bid("C")]
            D = self.bufs[_bid("D")]
            nab = n * (n - 1) // 2
            iu = np.triu_indices(n, 1)  # (j, i) with j < i
            for h in pf.dheads:
                for kk in range(h["nD"]):
                    M = np.zeros((n, n))
                    p = 1.0 if kk < h["nsing"] else -1.0
                    if kk < h["nsf_ab"]:
                        seg = c[h["off_ab"] + kk * nab:h["off_ab"] + (kk + 1) * nab]
                        # pair index of (j, i), i > j: i(i-1)/2 + j
                        j, i = iu
                        M[j, i] = seg[i * (i - 1) // 2 + j]
                        M[i, j] = p * seg[i * (i - 1) // 2 + j]
                    if kk < h["nsf_aa"]:
                        M[np.arange(n), np.arange(n)] = SQ2 * c[h["off_aa"] + kk * n:h["off_aa"] + (kk + 1) * n]
                    dk = h["dk0"] + kk
                    D[dk * n * n:(dk + 1) * n * n] = M.reshape(-1)
        elif k == "PACK":
            R = self.bufs[_bid("R")]
            S = self.bufs[_bid("S")]
            nab = n * (n - 1) // 2
            iu = np.triu_indices(n, 1)
            for h in pf.dheads:
                for kk in range(h["nD"]):
                    dk = h["dk0"] + kk
                    M = R[dk * n * n:(dk + 1) * n * n].reshape(n, n)
                    p = 1.0 if kk < h["nsing"] else -1.0
                    if kk < h["nsf_ab"]:
                        j, i = iu
                        S[h["off_ab"] + kk * nab + i * (i - 1) // 2 + j] += M[j, i] + p * M[i, j]
                    if kk < h["nsf_aa"]:
                        S[h["off_aa"] + kk * n:h["off_aa"] + (kk + 1) * n] += SQ2 * np.diag(M)
        elif k == "WBUILD":
            X = self.bufs[_bid("X")]
            npk = n * (n + 1) // 2
            Xm = X[:npk * npk].reshape(npk, npk)

            def pk(a, b):
                a, b = np.maximum(a, b), np.minimum(a, b)
                return a * (a + 1) // 2 + b

            def eri(a, b, c, d):
                return Xm[pk(a, b), pk(c, d)]

            diag = [(a, a) for a in range(n)]
            off = [(i, j) for i in range(1, n) for j in range(i)]
            npl = n + len(off)
            rows = diag + off
            Wp = np.zeros((npl, npl))
            for r, (a, cc) in enumerate(rows):
                for q, (b, d) in enumerate(rows):
                    rd, cd = r < n, q < n
                    if rd and cd:
                        v = eri(a, b, a, b)
                    elif rd:
                        v = SQ2 * eri(a, b, a, d)
                    elif cd:
                        v = SQ2 * eri(a, b, cc, b)
                    else:
                        v = eri(a, b, cc, d) + eri(a, d, cc, b)
                    Wp[r, q] = v
            Wm = np.zeros((len(off), len(off)))
            for r, (a, cc) in enumerate(off):
                for q, (b, d) in enumerate(off):
                    Wm[r, q] = eri(a, b, cc, d) - eri(a, d, cc, b)
            W = self.bufs[_bid("W")]
            W[:npl * npl] = Wp.reshape(-1)
            W[npl * npl:npl * npl + Wm.size] = Wm.reshape(-1)
        else:
            raise ValueError(k)

    def sigma(self, c):
        pf = self.pf
        self.bufs[_bid("C")][:] = c
        self.bufs[_bid("S")][:] = 0.0
        for st in pf.sigma_steps:
            self.run(st)
        return self.bufs[_bid("S")].copy()

    def diagonal(self):
        """H_ii assembled from the plan's diagonal entries (same formula as the device)."""
        pf = self.pf
        n = pf.n
        out = np.zeros(pf.total_csfs)
        F = self.bufs[_bid("F")]
        W = self.bufs[_bid("W")]
        npl, nm = pf.np, pf.nm
        for d in pf.diag:
            o, ln, t, b, fo = int(d["off"]), int(d["len"]), int(d["type"]), float(d["beta"]), int(d["foff"])

            def fd(a):
                return F[fo + a * (n + 1)] if fo >= 0 else 0.0

            if t == 0:
                out[o] = b
            elif t == 1:
                out[o:o + ln] = [b + fd(a) for a in range(n)]
            elif t == 2:
                out[o:o + ln] = [b + 2 * fd(a) + W[a * npl + a] for a in range(n)]
            else:
                e = 0
                for i in range(1, n):
                    for j in range(i):
                        w = W[(n + e) * npl + (n + e)] if d["singlet"] else W[npl * npl + e * nm + e]
                        out[o + e] = b + fd(i) + fd(j) + w
                        e += 1
        return out

    def trace(self, c):
        """Per-step sigma increments (for debugging)."""
        pf = self.pf
        self.bufs[_bid("C")][:] = c
        self.bufs[_bid("S")][:] = 0.0
        out = []
        for st in pf.sigma_steps:
            before = self.bufs[_bid("S")].copy()
            self.run(st)
            out.append((st["name"], self.bufs[_bid("S")] - before))
        return out
