"""Reader of the binary plan written by tci_plan_export (host/capi_host.cpp).

Layout (all fields 8 bytes, little endian): magic "TCIPLAN1"; header
(nint, n, nchol, total_csfs, npair_all, nD, n_dheads, NUM_BUFS, n_init,
n_sigma, len h_vv, len wv, np, nm, n_diag); buffer sizes; N-2 head records
(off_ab, off_aa, nsf_ab, nsf_aa, nsing, nD, dk0); dk signs; h_vv; wv; diagonal
entries (off, len, type, beta, foff, singlet); then
each step: kind, 64-byte name, counts (gp, gs, at, as, dt, ds), buf, off,
len and the tables.
"""
from __future__ import annotations

import numpy as np

BUF_NAMES = ["C", "S", "D", "R", "T0", "T1", "T2", "T3", "JK", "V", "W", "F", "WV", "L", "LE", "LV", "LI", "X"]
STEP_KINDS = ["GEMM", "AXPY", "DOT", "UNPACK", "PACK", "ZERO", "WBUILD"]

GP = np.dtype([("c", "<i8"), ("offC", "<i8"), ("ldc", "<i8"), ("M", "<i8"), ("N", "<i8"), ("beta", "<f8"),
               ("seg_begin", "<i8"), ("seg_end", "<i8")])
GS = np.dtype([("a", "<i8"), ("b", "<i8"), ("offA", "<i8"), ("lda", "<i8"), ("offB", "<i8"), ("ldb", "<i8"),
               ("K", "<i8"), ("tA", "<i8"), ("tB", "<i8"), ("alpha", "<f8")])
AT = np.dtype([("dst", "<i8"), ("off", "<i8"), ("len", "<i8"), ("src_begin", "<i8"), ("src_end", "<i8")])
AS = np.dtype([("src", "<i8"), ("off", "<i8"), ("coef", "<f8"), ("sbuf", "<i8"), ("sidx", "<i8")])
DT = np.dtype([("dst", "<i8"), ("off", "<i8"), ("src_begin", "<i8"), ("src_end", "<i8")])
DS = np.dtype([("a", "<i8"), ("b", "<i8"), ("aoff", "<i8"), ("boff", "<i8"), ("len", "<i8"), ("coef", "<f8")])
DG = np.dtype([("off", "<i8"), ("len", "<i8"), ("type", "<i8"), ("beta", "<f8"), ("foff", "<i8"), ("singlet", "<i8")])
DH = np.dtype([("off_ab", "<i8"), ("off_aa", "<i8"), ("nsf_ab", "<i8"), ("nsf_aa", "<i8"), ("nsing", "<i8"),
               ("nD", "<i8"), ("dk0", "<i8")])


class PlanFile:
    def __init__(self, path):
        raw = open(path, "rb").read()
        if raw[:8] != b"TCIPLAN1":
            raise ValueError("not a plan file")
        self._b = raw
        self._p = 8
        (self.nint, self.n, self.nchol, self.total_csfs, self.npair_all, self.nD, ndh, nbuf, ninit, nsig, nh,
         nwv, self.np, self.nm, ndiag) = self._i(15)
        self.buf_size = self._i(nbuf)
        self.dheads = self._arr(DH, ndh)
        self.dk_sign = self._f(self.nD)
        self.h_vv = self._f(nh)
        self.wv = self._f(nwv)
        self.diag = self._arr(DG, ndiag)
        self.init_steps = [self._step() for _ in range(ninit)]
        self.sigma_steps = [self._step() for _ in range(nsig)]

    def _i(self, k):
        v = np.frombuffer(self._b, dtype="<i8", count=k, offset=self._p)
        self._p += 8 * k
        return [int(x) for x in v]

    def _f(self, k):
        v = np.frombuffer(self._b, dtype="<f8", count=k, offset=self._p).copy()
        self._p += 8 * k
        return v

    def _arr(self, dt, k):
        v = np.frombuffer(self._b, dtype=dt, count=k, offset=self._p).copy()
        self._p += dt.itemsize * k
        return v

    def _step(self):
        kind = self._i(1)[0]
        name = self._b[self._p:self._p + 64].split(b"\0")[0].decode()
        self._p += 64
        ngp, ngs, nat, nas, ndt, nds, buf, off, ln = self._i(9)
        return dict(kind=STEP_KINDS[kind], name=name, gp=self._arr(GP, ngp), gs=self._arr(GS, ngs),
                    at=self._arr(AT, nat), as_=self._arr(AS, nas), dt=self._arr(DT, ndt), ds=self._arr(DS, nds),
                    buf=buf, off=off, len=ln)
