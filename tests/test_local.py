"""All-external term over pair domains (tci_local_*): the oracle's integral
form over domains against the Cholesky form it is applied in, and the device
(FP64 and mixed) against the oracle."""
import numpy as np
import pytest

from oracle import dense
from tigerci_b200 import local
from tigerci_b200.synthetic import synthetic_operator


def _problem(n_pairs=12, n_int=5, n_virt=30, dmin=3, dmax=14, nchol=40, seed=3):
    heads, dom, total = local.pair_domain_problem(n_pairs, n_int, n_virt, dmin, dmax, seed=seed)
    h, L = synthetic_operator(n_int + n_virt, nchol, seed=seed + 1, scale=0.5)
    c = np.random.default_rng(seed + 2).standard_normal(total)
    return heads, dom, total, L, c


def _pair(p, q):
    return p * (p + 1) // 2 + q if p >= q else q * (q + 1) // 2 + p


def _cholesky_form(n_int, L, heads, dom, c):
    """sigma_hk = pack(1/2 sum_J L^J_h D_hk L^J_h) in numpy (the device's formulation)."""
    s = np.zeros_like(c)
    for off_ab, off_aa, nsf_ab, nsf_aa, nsing, doff, n in heads:
        d = dom[doff:doff + n]
        idx = np.array([[_pair(n_int + a, n_int + b) for b in d] for a in d])
        Lh = np.moveaxis(L[idx], 2, 0)  # (J, n, n)
        nab = n * (n - 1) // 2
        iu, ju = np.tril_indices(n, -1)  # i > j, pair index i(i-1)/2 + j in this order
        for k in range(max(nsf_ab, nsf_aa)):
            p = 1.0 if k < nsing else -1.0
            D = np.zeros((n, n))
            if k < nsf_aa:
                D[np.arange(n), np.arange(n)] = np.sqrt(2) * c[off_aa + k * n:off_aa + (k + 1) * n]
            if k < nsf_ab:
                x = c[off_ab + k * nab:off_ab + (k + 1) * nab]
                D[ju, iu] = x
                D[iu, ju] = p * x
            R = 0.5 * np.einsum("Jac,cd,Jdb->ab", Lh, D, Lh)
            if k < nsf_ab:
                s[off_ab + k * nab:off_ab + (k + 1) * nab] += R[ju, iu] + p * R[iu, ju]
            if k < nsf_aa:
                s[off_aa + k * n:off_aa + (k + 1) * n] += np.sqrt(2) * np.diag(R)
    return s


def test_oracle_integral_form_equals_cholesky_form():
    heads, dom, total, L, c = _problem()
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    sc = _cholesky_form(5, L, heads, dom, c)
    assert np.abs(so - sc).max() <= 1e-12 * np.abs(so).max()


def test_oracle_local_equals_non_local_when_every_domain_is_everything():
    """With every domain the full external space the local oracle is the
    non-local all-external oracle restricted to these heads."""
    heads, dom, total = local.pair_domain_problem(6, 4, 9, 9, 9, seed=5)
    assert all(h[6] == 9 for h in heads)
    h, L = synthetic_operator(13, 20, seed=6, scale=0.5)
    c = np.random.default_rng(1).standard_normal(total)
    so = dense.allext_local_sigma(4, L, heads, dom, c)
    sc = _cholesky_form(4, L, heads, dom, c)
    assert np.abs(so - sc).max() <= 1e-12 * np.abs(so).max()


def _dense_form(n_int, n_virt, L, heads, dom, c):
    """The device's dense padded form in numpy: W+ / W- over all external pairs from X = Lpk Lpk^T (the
    non-local packed integral form), the blocks placed among all externals (U+ rows for singlet-coupled,
    U- rows for triplet-coupled spin functions), Y = U W read back at the domain's pairs."""
    n = n_virt
    ia, ib = np.tril_indices(n, -1)  # a > b
    order = np.argsort(ia * (ia - 1) // 2 + ib)
    ia, ib = ia[order], ib[order]
    rows = np.array([_pair(n_int + a, n_int + b) for a in range(n) for b in range(a + 1)])
    X = L[rows] @ L[rows].T

    def pk(a, b):
        hi, lo = np.maximum(a, b), np.minimum(a, b)
        return hi * (hi + 1) // 2 + lo

    def x(a, b, cc, d):  # (ab|cd)
        return X[pk(a, b), pk(cc, d)]

    ra, rc, qb, qd = ia[:, None], ib[:, None], ia[None, :], ib[None, :]
    # row pair (a, c), column pair (b, d): (ab|cd) +- (cb|ad)
    Wab_p = x(ra, qb, rc, qd) + x(rc, qb, ra, qd)
    Wab_m = x(ra, qb, rc, qd) - x(rc, qb, ra, qd)
    aa = np.arange(n)
    Wdd = x(aa[:, None], aa[None, :], aa[:, None], aa[None, :])  # rows (aa), columns (bb): (ab|ab)
    Wdp = np.sqrt(2) * x(aa[:, None], qb, aa[:, None], qd)  # rows (aa), columns (bd): sqrt2 (ab|ad)
    Wp = np.block([[Wdd, Wdp], [Wdp.T, Wab_p]])
    s = np.zeros_like(c)
    for off_ab, off_aa, nsf_ab, nsf_aa, nsing, doff, m in heads:
        d = dom[doff:doff + m]
        mab = m * (m - 1) // 2
        li, lj = np.tril_indices(m, -1)
        lo = np.argsort(li * (li - 1) // 2 + lj)
        li, lj = li[lo], lj[lo]
        cols = d[li] * (d[li] - 1) // 2 + d[lj]  # pair index among all externals
        for k in range(max(nsf_ab, nsf_aa)):
            if k < nsing:
                u = np.zeros(n + len(ia))
                if k < nsf_aa:
                    u[d] = c[off_aa + k * m:off_aa + (k + 1) * m]
                if k < nsf_ab:
                    u[n + cols] = c[off_ab + k * mab:off_ab + (k + 1) * mab]
                y = Wp @ u
                if k < nsf_aa:
                    s[off_aa + k * m:off_aa + (k + 1) * m] += y[d]
                if k < nsf_ab:
                    s[off_ab + k * mab:off_ab + (k + 1) * mab] += y[n + cols]
            else:
                u = np.zeros(len(ia))
                u[cols] = c[off_ab + k * mab:off_ab + (k + 1) * mab]
                s[off_ab + k * mab:off_ab + (k + 1) * mab] += (Wab_m @ u)[cols]
    return s


def test_dense_padded_form_equals_local_oracle():
    """The dense form's identity: the non-local packed integral form applied to blocks that are zero outside
    their domains, read back at the domains, is the domain-restricted all-external term."""
    heads, dom, total, L, c = _problem(n_pairs=8, n_virt=12, dmin=1, dmax=12, nchol=30, seed=4)
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    sd = _dense_form(5, 12, L, heads, dom, c)
    assert np.abs(sd - so).max() <= 1e-11 * np.abs(so).max()


def test_pair_domain_problem_shapes():
    heads, dom, total = local.pair_domain_problem(600, 35, 400, 20, 180, seed=99)
    assert len(heads) == 600
    n = heads[:, 6]
    assert n.min() >= 20 and n.max() <= 180
    assert ((heads[:, 2] == 1) | (heads[:, 2] == 2)).all()
    # domains sorted and within the external space
    for off_ab, off_aa, nsf_ab, nsf_aa, nsing, doff, m in heads[:20]:
        d = dom[doff:doff + m]
        assert (np.diff(d) > 0).all() and d.min() >= 0 and d.max() < 400
    last = heads[-1]
    assert total == last[0] + last[2] * last[6] * (last[6] - 1) // 2


@pytest.mark.gpu
@pytest.mark.parametrize("chunk_bytes", [16e9, 3e5])
def test_device_fp64_matches_oracle(chunk_bytes, need_gpu):
    heads, dom, total, L, c = _problem()
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    op = local.LocalAllExternal(5, 30, L, heads, dom, total, device=0, precision="fp64", chunk_bytes=chunk_bytes)
    sd = op.apply(c)
    st = op.stats()
    if chunk_bytes < 1e6:
        assert st["chunk"] < 40  # several chunks and a shorter last one
    assert np.abs(sd - so).max() <= 1e-10 * np.abs(so).max()
    assert np.array_equal(sd, op.apply(c))  # deterministic
    op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["auto", "cholesky", "dense"])
def test_device_mixed_matches_oracle(form, need_gpu):
    heads, dom, total, L, c = _problem(n_pairs=15, n_virt=60, dmin=10, dmax=50, nchol=64)
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    op = local.LocalAllExternal(5, 60, L, heads, dom, total, device=0, precision="tf32x3", form=form)
    st = op.stats()
    if form != "auto":
        assert st["form"] == form
    if form == "dense":
        n = 60
        np_, nm = n + n * (n - 1) // 2, n * (n - 1) // 2
        n_trip = int(sum(max(0, h[2] - h[4]) for h in heads))
        assert st["dense_flops"] == 2.0 * np_ * np_ * (st["blocks"] - n_trip) + 2.0 * nm * nm * n_trip
    sd = op.apply(c)
    assert np.linalg.norm(sd - so) <= 2e-5 * np.linalg.norm(so)
    assert np.abs(sd - so).max() <= 1e-5 * np.abs(so).max()
    assert np.array_equal(sd, op.apply(c))
    op.close()


@pytest.mark.gpu
def test_dense_form_with_ragged_domains_and_a_single_external(need_gpu):
    """Domains of one external (no ab block, aa only) and of every external, heads with only a singlet
    block, in the dense form."""
    heads, dom, total, L, c = _problem(n_pairs=10, n_virt=33, dmin=1, dmax=33, nchol=50, seed=1)
    assert heads[:, 6].min() == 1 and heads[:, 6].max() == 33
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    op = local.LocalAllExternal(5, 33, L, heads, dom, total, device=0, precision="tf32x3", form="dense")
    sd = op.apply(c)
    assert np.abs(sd - so).max() <= 1e-5 * np.abs(so).max()
    op.close()


@pytest.mark.gpu
def test_dense_form_refused_in_fp64(need_gpu):
    heads, dom, total, L, c = _problem()
    with pytest.raises(Exception):
        local.LocalAllExternal(5, 30, L, heads, dom, total, device=0, precision="fp64", form="dense")


@pytest.mark.gpu
def test_device_apply_accumulates_on_a_stream(need_gpu):
    import torch

    heads, dom, total, L, c = _problem()
    op = local.LocalAllExternal(5, 30, L, heads, dom, total, device=0)
    ref = op.apply(c)
    ct = torch.from_numpy(c).cuda()
    st = torch.ones(total, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        op.apply_device(ct.data_ptr(), st.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    assert np.abs(st.cpu().numpy() - 1.0 - ref).max() <= 1e-12 * np.abs(ref).max()
    op.close()
