"""All-external term of a local MRSDCI space with pair domains (tci_local_*).

`LocalAllExternal` applies, for a set of N-2 heads that each keep their own
sorted domain of external orbitals, the all-external contribution of TigerCI's
local correlation treatment (virtual_truncation, tiger_fortran/locist_mod.f90,
and the local all-external loops of three_and_four_seg_mod_1.f90) batched over
heads of uneven size on one GPU.

`pair_domain_problem` builds the batching workload: internal pairs of a
closed-shell reference in lexical order (i >= j), one singlet-coupled spin
function for i == j and a singlet- plus a triplet-coupled one for i > j, each
with a seeded random domain of external orbitals.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr

PRECISIONS = {"fp64": 0, "tf32x3": 1}
# all-external form: the faster of the two (timed at set-up), the pair-domain Cholesky form, or the dense
# padded integral form (mixed precision only)
FORMS = {"auto": 0, "cholesky": 1, "dense": 2}


def _bind():
    L = lib()
    if not getattr(L, "_local_bound", False):
        P, i64 = C.c_void_p, C.c_int64
        L.tci_local_create.argtypes = [i64, i64, P, i64, i64, P, P, i64, i64, P, i64, C.POINTER(P)]
        L.tci_local_apply.argtypes = [P, P, P, i64, P]
        L.tci_local_apply_host.argtypes = [P, P, P, i64]
        L.tci_local_stats.argtypes = [P, P, i64]
        L.tci_local_destroy.argtypes = [P]
        L.tci_local_destroy.restype = None
        L._local_bound = True
    return L


class LocalAllExternal:
    """heads: int64 rows (off_ab, off_aa, nsf_ab, nsf_aa, nsing, dom_off, dom_len);
    dom_idx: concatenated sorted domains; chol: Cholesky vectors over
    num_internal + num_external orbitals, rows pair = p(p+1)/2 + q (p >= q)."""

    def __init__(self, num_internal, num_external, chol, heads, dom_idx, total_len, device=0, precision="fp64",
                 chunk_bytes=16e9, promote_every=128, autotune=True, form="auto"):
        self._L = _bind()
        self.heads = np.ascontiguousarray(np.asarray(heads, dtype=np.int64).reshape(-1, 7))
        self.dom = np.ascontiguousarray(np.asarray(dom_idx, dtype=np.int64))
        chol = np.ascontiguousarray(chol, dtype=np.float64)
        self.n = int(total_len)
        opts = np.array([PRECISIONS[precision], int(chunk_bytes), promote_every, 1 if autotune else 0, FORMS[form]],
                        dtype=np.int64)
        h = C.c_void_p()
        check(self._L.tci_local_create(num_internal, num_external, ptr(chol), chol.shape[1], len(self.heads),
                                       ptr(self.heads), ptr(self.dom), self.n, device, ptr(opts), 5, C.byref(h)))
        self._h = h

    def apply(self, c: np.ndarray) -> np.ndarray:
        c = np.ascontiguousarray(c, dtype=np.float64)
        s = np.zeros_like(c)
        check(self._L.tci_local_apply_host(self._h, ptr(c), ptr(s), self.n))
        return s

    def apply_device(self, c_ptr: int, s_ptr: int, stream: int = 0):
        """sigma += A c on device arrays (e.g. torch tensors' data_ptr())."""
        check(self._L.tci_local_apply(self._h, C.c_void_p(c_ptr), C.c_void_p(s_ptr), self.n, C.c_void_p(stream or None)))

    def stats(self) -> dict:
        """form: "cholesky" or "dense" (the one applied); tuned_ms / dense_ms: the set-up timings of the two forms
        (0 where a form was not timed); flops: the Cholesky form's 4 nchol sum n^3, dense_flops: the dense form's
        2 np^2 per singlet-coupled and 2 nm^2 per triplet-coupled block; dense_w_bytes: its FP32 W tiles."""
        out = np.zeros(13)
        check(self._L.tci_local_stats(self._h, ptr(out), 13))
        keys = ["flops", "cholesky_bytes", "device_bytes", "chunk", "tile_cfg", "tuned_ms", "candidates", "last_ms",
                "blocks", "form", "dense_ms", "dense_flops", "dense_w_bytes"]
        d = dict(zip(keys, out.tolist()))
        d["form"] = "dense" if d["form"] == 1 else "cholesky"
        return d

    def close(self):
        if getattr(self, "_h", None):
            self._L.tci_local_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


RECORD_FIELDS = ("icount", "head_weight", "ab_address", "aa_address", "nsf_aa", "nsf_ab", "a_pos", "c_pos")


def allext_records(deck) -> np.ndarray:
    """The loop records of the pair-domain all-external term for a deck with domains
    (tci_local_allext_records): one row per (head, external pair a >= c in its domain), columns RECORD_FIELDS,
    as the reference's dry run of the local all-external loops writes them
    (build_ext_34seg_dryrun, three_and_four_seg_mod_1.f90:3142-3238)."""
    d = deck.c_struct()
    n = C.c_int64()
    check(lib().tci_local_allext_records(C.byref(d), None, 0, C.byref(n)))
    out = np.zeros((max(n.value, 1), 8), dtype=np.int64)
    check(lib().tci_local_allext_records(C.byref(d), ptr(out), out.size, C.byref(n)))
    return out[:n.value]


def pair_domain_problem(n_pairs=600, n_int=35, n_virt=400, dmin=20, dmax=180, seed=99):
    """Heads, domains and CI length of the pair-domain batching workload.

    Pairs (i >= j) of n_int doubly occupied internal orbitals in lexical order,
    the first n_pairs of them; domain sizes uniform in [dmin, dmax], each a
    sorted random subset of the n_virt external orbitals.  CI layout per head:
    aa block (n), then the ab blocks (n(n-1)/2 per spin function)."""
    rng = np.random.default_rng(seed)
    heads, dom = [], []
    off = doff = 0
    pairs = [(i, j) for i in range(n_int) for j in range(i + 1)][:n_pairs]
    for i, j in pairs:
        n = int(rng.integers(dmin, dmax + 1))
        d = np.sort(rng.choice(n_virt, size=n, replace=False))
        nsf_ab = 1 if i == j else 2
        nab = n * (n - 1) // 2
        off_aa = off
        off += n
        off_ab = off
        off += nsf_ab * nab
        heads.append([off_ab, off_aa, nsf_ab, 1, 1, doff, n])
        dom.extend(d.tolist())
        doff += n
    return np.array(heads, dtype=np.int64), np.array(dom, dtype=np.int64), off


def pair_domain_deck(n_int=35, n_virt=400, dmin=20, dmax=180, seed=99):
    """Deck of the local MRSDCI with pair domains: n_int doubly occupied internal orbitals (one closed-shell
    reference), n_virt externals, every N-2 path (the n_int (n_int + 1) / 2 internal pairs, lexical order)
    and every N-1 path with a seeded random domain: size uniform in [dmin, dmax], a sorted random subset of
    the externals."""
    from .api import CsfSpace, Deck

    base = Deck(n_int + n_virt, n_int, 0, 2 * n_int, 1, ["2" * n_int])
    cnt = CsfSpace(base).counts()
    rng = np.random.default_rng(seed)

    def doms(k):
        out = []
        for _ in range(k):
            m = int(rng.integers(dmin, dmax + 1))
            out.append(np.sort(rng.choice(n_virt, size=m, replace=False)).tolist())
        return out

    nm2 = doms(cnt["paths_nm2"])
    nm1 = doms(cnt["paths_nm1"])
    return Deck(n_int + n_virt, n_int, 0, 2 * n_int, 1, ["2" * n_int], nm1_domains=nm1, nm2_domains=nm2)
