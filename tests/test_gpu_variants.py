"""Every kernel variant of the variable-size batched routines gives the
reference's results (variants change the schedule, never the arithmetic of an
element): dgemm_nt, dpotrf_l, dgetrf_rp (identical pivots) and dgeqrf against
the oracle, on batches that mix instances that fit in shared memory with
instances that do not."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, spd, tol

pytestmark = pytest.mark.gpu
P = lambda x: C.c_void_p(x.data_ptr())


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    blasfeo_b200.set_sync(True)
    return blasfeo_b200


@pytest.fixture(scope="module")
def orc():
    return oracle_api()


def host(m, n, data=None):
    from oracle.pyoracle import HostMat
    h = HostMat(m, n, np.float64)
    if data is not None:
        h.set(data)
    return h


def ivec(v):
    import torch
    return torch.tensor(v, dtype=torch.int32, device="cuda")


def nvar(bf, op):
    return bf.lib.blasfeo_b200_num_variants(op)


def test_variant_counts(bf):
    assert [nvar(bf, i) for i in range(4)] == [6, 6, 6, 6]
    assert nvar(bf, 9) == 0


@pytest.mark.parametrize("variant", range(6))
def test_gemm_variants(bf, variant):
    import torch
    rng = np.random.default_rng(variant)
    ms, ns, ks = [3, 40, 17, 64, 130, 1, 384], [5, 20, 33, 64, 97, 9, 300], [7, 1, 40, 64, 200, 3, 384]
    A = [rng.standard_normal((m, k)) for m, k in zip(ms, ks)]
    B = [rng.standard_normal((n, k)) for n, k in zip(ns, ks)]
    Cm = [rng.standard_normal((m, n)) for m, n in zip(ms, ns)]
    dA = [bf.DMat(m, k).pack(a) for m, k, a in zip(ms, ks, A)]
    dB = [bf.DMat(n, k).pack(b) for n, k, b in zip(ns, ks, B)]
    dC = [bf.DMat(m, n).pack(c) for m, n, c in zip(ms, ns, Cm)]
    dD = [bf.DMat(m, n) for m, n in zip(ms, ns)]
    aA, aB, aC, aD = (bf.descriptor_array(x) for x in (dA, dB, dC, dD))
    mv, nv, kv = ivec(ms), ivec(ns), ivec(ks)
    st = bf.lib.blasfeo_dgemm_nt_vbatch_variant(len(ms), P(mv), P(nv), P(kv), max(ms), max(ns), max(ks), 1.5, P(aA),
                                                P(aB), -0.5, P(aC), P(aD), variant, None)
    assert st == 0
    torch.cuda.synchronize()
    for a, b, c, d in zip(A, B, Cm, dD):
        assert relfro(d.unpack(), 1.5 * a @ b.T - 0.5 * c) <= 1e-14


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3, 4, 5])
def test_potrf_variants(bf, orc, variant):
    import torch
    rng = np.random.default_rng(40 + variant)
    ns = [4, 17, 64, 100, 1, 250, 300, 33, 384]
    S = [spd(rng, n) for n in ns]
    dC = [bf.DMat(n, n).pack(s) for n, s in zip(ns, S)]
    dD = [bf.DMat(n, n) for n in ns]
    aC, aD = bf.descriptor_array(dC), bf.descriptor_array(dD)
    info = ivec([-9] * len(ns))
    nv = ivec(ns)
    st = bf.lib.blasfeo_dpotrf_l_vbatch_variant(len(ns), P(nv), max(ns), P(aC), P(aD), P(info), variant, None)
    assert st == 0
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    for n, s, d in zip(ns, S, dD):
        hC, hD = host(n, n, s), host(n, n)
        orc.potrf_l("d", n, hC, 0, 0, hD, 0, 0)
        assert relfro(np.tril(d.unpack()), np.tril(hD.get())) <= 1e-13, n
        assert relfro(d.diag_array(), hD.diag(n)) <= 1e-13


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3, 4, 5])
def test_getrf_variants(bf, orc, variant):
    import torch
    rng = np.random.default_rng(70 + variant)
    dims = [(4, 4), (17, 9), (9, 17), (64, 64), (170, 170), (200, 130), (1, 5), (384, 384), (300, 300)]
    M = [rng.standard_normal(d) for d in dims]
    dC = [bf.DMat(m, n).pack(x) for (m, n), x in zip(dims, M)]
    dD = [bf.DMat(m, n) for m, n in dims]
    aC, aD = bf.descriptor_array(dC), bf.descriptor_array(dD)
    mv, nv = ivec([d[0] for d in dims]), ivec([d[1] for d in dims])
    mx_m, mx_n = max(d[0] for d in dims), max(d[1] for d in dims)
    mn = max(min(d) for d in dims)
    piv = ivec([-1] * (len(dims) * mn))
    info = ivec([-9] * len(dims))
    st = bf.lib.blasfeo_dgetrf_rp_vbatch_variant(len(dims), P(mv), P(nv), mx_m, mx_n, P(aC), P(aD), P(piv), mn,
                                                 P(info), variant, None)
    assert st == 0
    torch.cuda.synchronize()
    pv = piv.cpu().numpy().reshape(len(dims), mn)
    assert (info.cpu().numpy() == 0).all()
    for i, ((m, n), x, d) in enumerate(zip(dims, M, dD)):
        hC, hD = host(m, n, x), host(m, n)
        pr = orc.getrf_rp("d", m, n, hC, 0, 0, hD, 0, 0)
        assert np.array_equal(pv[i, :min(m, n)], pr), (m, n)
        assert relfro(d.unpack(), hD.get()) <= 1e-13, (m, n)


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3, 4, 5])
def test_geqrf_variants(bf, orc, variant):
    import torch
    rng = np.random.default_rng(90 + variant)
    dims = [(8, 4), (34, 17), (128, 64), (240, 120), (9, 13), (300, 150), (2, 1), (384, 192)]
    M = [rng.standard_normal(d) for d in dims]
    dC = [bf.DMat(m, n).pack(x) for (m, n), x in zip(dims, M)]
    dD = [bf.DMat(m, n) for m, n in dims]
    aC, aD = bf.descriptor_array(dC), bf.descriptor_array(dD)
    mv, nv = ivec([d[0] for d in dims]), ivec([d[1] for d in dims])
    st = bf.lib.blasfeo_dgeqrf_vbatch_variant(len(dims), P(mv), P(nv), max(d[0] for d in dims),
                                              max(d[1] for d in dims), P(aC), P(aD), variant, None)
    assert st == 0
    torch.cuda.synchronize()
    for (m, n), x, d in zip(dims, M, dD):
        hC, hD = host(m, n, x), host(m, n)
        orc.geqrf("d", m, n, hC, 0, 0, hD, 0, 0)
        tol = 1e-13
        assert relfro(d.unpack(), hD.get()) <= tol, (m, n)
        k = min(m, n)
        assert relfro(d.diag_array()[:k], hD.diag(k)) <= tol, (m, n)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_geqrf_blocked_variants_small_batch(bf, orc, variant):
    """The blocked QR kernels on a batch whose largest matrix is small
    (96 x 48): the launch's dynamic shared memory is then just under 48 KB and
    the kernel's static shared memory takes it over, so the launch must opt in
    all the same."""
    import torch
    rng = np.random.default_rng(120 + variant)
    dims = [(96, 48), (70, 40), (96, 7)]
    M = [rng.standard_normal(d) for d in dims]
    dC = [bf.DMat(m, n).pack(x) for (m, n), x in zip(dims, M)]
    dD = [bf.DMat(m, n) for m, n in dims]
    aC, aD = bf.descriptor_array(dC), bf.descriptor_array(dD)
    mv, nv = ivec([d[0] for d in dims]), ivec([d[1] for d in dims])
    st = bf.lib.blasfeo_dgeqrf_vbatch_variant(len(dims), P(mv), P(nv), 96, 48, P(aC), P(aD), variant, None)
    assert st == 0
    torch.cuda.synchronize()
    for (m, n), x, d in zip(dims, M, dD):
        hC, hD = host(m, n, x), host(m, n)
        orc.geqrf("d", m, n, hC, 0, 0, hD, 0, 0)
        assert relfro(d.unpack(), hD.get()) <= 1e-13, (m, n)


def test_variant_out_of_range_rejected(bf):
    nv = ivec([4])
    d = bf.descriptor_array([bf.DMat(4, 4)])
    assert bf.lib.blasfeo_dpotrf_l_vbatch_variant(1, P(nv), 4, P(d), P(d), None, 6, None) == 1
    assert bf.lib.blasfeo_dgemm_nt_vbatch_variant(1, P(nv), P(nv), P(nv), 4, 4, 4, 1.0, P(d), P(d), 0.0, P(d), P(d),
                                                  6, None) == 1


def test_potrf_dmma_warp_kernel_mixed_sizes_and_bad_pivots(bf, orc):
    # the one-warp FP64 tensor-core Cholesky (variant 5, n <= 64): every 8-block
    # padding case, plus indefinite instances whose zero pivots must follow the
    # reference (L_jj = 0, dA_j = 0, computation continues)
    import torch
    rng = np.random.default_rng(123)
    ns = [1, 2, 3, 7, 8, 9, 15, 16, 17, 31, 33, 40, 47, 55, 63, 64, 64, 20]
    S = [spd(rng, n) for n in ns]
    S[-2][10, 10] = -3.0                       # first bad pivot at 10 (or earlier)
    S[-1] = S[-1] - 40.0 * np.eye(20)          # indefinite from the start
    dC = [bf.DMat(n, n).pack(s) for n, s in zip(ns, S)]
    dD = [bf.DMat(n, n) for n in ns]
    aC, aD = bf.descriptor_array(dC), bf.descriptor_array(dD)
    info = ivec([-9] * len(ns))
    st = bf.lib.blasfeo_dpotrf_l_vbatch_variant(len(ns), P(ivec(ns)), max(ns), P(aC), P(aD), P(info), 5, None)
    assert st == 0
    torch.cuda.synchronize()
    inf = info.cpu().numpy()
    assert (inf[:-2] == 0).all(), inf
    assert 1 <= inf[-2] <= 11 and inf[-1] >= 1, inf
    for n, s, d, i in zip(ns, S, dD, inf):
        hC, hD = host(n, n, s), host(n, n)
        orc.potrf_l("d", n, hC, 0, 0, hD, 0, 0)
        ref = np.tril(hD.get())
        if i == 0:
            assert relfro(np.tril(d.unpack()), ref) <= 1e-13, n
            assert relfro(d.diag_array(), hD.diag(n)) <= 1e-13, n
        else:
            # same zero pattern on the diagonal from the first bad pivot on
            got = np.tril(d.unpack())
            assert (np.diag(got) == 0).sum() == (np.diag(ref) == 0).sum()
            assert relfro(got[: i - 1, : i - 1], ref[: i - 1, : i - 1]) <= 1e-13
