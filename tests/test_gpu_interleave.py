"""GPU tests of the batch-interleaved layout: lossless conversion from and to
the back-to-back slab and from and to host column-major batches (whole and
partial groups of 16), and potrf_l on it
against the oracle, with the reference's pivot rule and per-instance info."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, spd

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    return blasfeo_b200


@pytest.mark.parametrize("shape", [(16, 16, 48), (5, 7, 37), (12, 12, 3), (16, 32, 17)])
def test_round_trip(bf, shape):
    import torch
    from blasfeo_b200.api import DMatBatchIL
    m, n, nb = shape
    rng = np.random.default_rng(m * n + nb)
    X = rng.standard_normal((nb, m, n))
    src = bf.DMatBatch(m, n, nb).pack_all(X)
    il = DMatBatchIL(m, n, nb).from_batch(src)
    out = bf.DMatBatch(m, n, nb)
    il.to_batch(out)
    torch.cuda.synchronize()
    assert np.array_equal(out.unpack_all(), X)
    # layout: element (i, j) of instance b at slot (i - i%4)*cn + 4j + i%4 of group b // 16, lane b % 16
    raw = il.buf.cpu().numpy().view(np.float64)
    cn, gs = il.s.cn, il.s.gstride
    for b, i, j in ((0, 0, 0), (nb - 1, m - 1, n - 1), (nb // 2, m // 2, n // 3)):
        e = (i - i % 4) * cn + 4 * j + i % 4
        assert raw[(b // 16) * gs + 16 * e + b % 16] == X[b, i, j]


@pytest.mark.parametrize("shape", [(16, 16, 48), (5, 7, 37), (12, 12, 3), (16, 32, 17), (1, 1, 1)])
def test_host_pack_unpack_il(bf, shape):
    """Host column-major <-> interleaved slab directly: the same slots as the
    route through the back-to-back slab, a strided host batch (lda > m,
    stride > lda n) in both directions, and the slots outside the block left
    as they were."""
    import torch
    from blasfeo_b200.api import DMatBatchIL
    m, n, nb = shape
    rng = np.random.default_rng(7 * m + n + nb)
    X = rng.standard_normal((nb, m, n))
    il = DMatBatchIL(m, n, nb).pack_all(X)
    ref = DMatBatchIL(m, n, nb).from_batch(bf.DMatBatch(m, n, nb).pack_all(X))
    torch.cuda.synchronize()
    raw, rraw = il.buf.cpu().numpy().view(np.float64), ref.buf.cpu().numpy().view(np.float64)
    cn, gs = il.s.cn, il.s.gstride
    for b in range(nb):
        for i in range(m):
            for j in range(n):
                e = (i - i % 4) * cn + 4 * j + i % 4
                assert raw[(b // 16) * gs + 16 * e + b % 16] == rraw[(b // 16) * gs + 16 * e + b % 16] == X[b, i, j]
    assert np.array_equal(il.unpack_all(), X)
    # strided host batch: lda = m + 3, stride = lda n + 5; a sub-block (m', n') of the slab
    mm, nn = max(1, m - 1), max(1, n - 2)
    lda, stride = m + 3, (m + 3) * n + 5
    host = np.full(nb * stride, np.nan)
    for b in range(nb):
        for j in range(nn):
            host[b * stride + j * lda: b * stride + j * lda + mm] = -X[b, :mm, j]
    st = bf.lib.blasfeo_pack_dmat_batch_il(nb, mm, nn, C.c_void_p(host.ctypes.data), lda, stride, il.ref, None)
    assert st == 0
    got = il.unpack_all()
    want = X.copy()
    want[:, :mm, :nn] *= -1
    assert np.array_equal(got, want)
    back = np.full(nb * stride, 7.0)
    st = bf.lib.blasfeo_unpack_dmat_batch_il(nb, mm, nn, il.ref, C.c_void_p(back.ctypes.data), lda, stride, None)
    assert st == 0
    for b in range(nb):
        for j in range(nn):
            col = back[b * stride + j * lda: b * stride + (j + 1) * lda]
            assert np.array_equal(col[:mm], -X[b, :mm, j]) and (col[mm:] == 7.0).all()
    # argument errors: lda < m, a block larger than the slab, a batch larger than the slab
    bad = np.zeros(4 * nb * (m + 1) * (n + 1))
    P = C.c_void_p(bad.ctypes.data)
    if m > 1:
        assert bf.lib.blasfeo_pack_dmat_batch_il(nb, m, n, P, m - 1, m * n, il.ref, None) == 1
    assert bf.lib.blasfeo_pack_dmat_batch_il(nb, m + 1, n, P, m + 1, (m + 1) * n, il.ref, None) == 1
    assert bf.lib.blasfeo_unpack_dmat_batch_il(nb + 1, m, n, il.ref, P, m, m * n, None) == 1


@pytest.mark.parametrize("n", [1, 5, 12, 16])
@pytest.mark.parametrize("nb", [37, 64])
def test_potrf_il_vs_oracle(bf, n, nb):
    import torch
    from blasfeo_b200.api import DMatBatchIL
    rng = np.random.default_rng(100 * n + nb)
    S = np.stack([spd(rng, n) for _ in range(nb)])
    if nb == 37:
        S[9, n // 2, n // 2] = -4.0  # one indefinite instance: zero pivot from there on
    src = bf.DMatBatch(n, n, nb).pack_all(S)
    ilC = DMatBatchIL(n, n, nb).from_batch(src)
    ilD = DMatBatchIL(n, n, nb)
    info = torch.full((nb,), -7, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dpotrf_l_batch_il(nb, n, ilC.ref, ilD.ref, C.c_void_p(info.data_ptr()), None)
    assert st == 0
    out = bf.DMatBatch(n, n, nb)
    ilD.to_batch(out)
    torch.cuda.synchronize()
    got, dg, inf = out.unpack_all(), out.diag_all(n), info.cpu().numpy()
    orc = oracle_api()
    from oracle.pyoracle import HostMat
    for b in range(nb):
        hC, hD = HostMat(n, n).set(S[b]), HostMat(n, n)
        orc.potrf_l("d", n, hC, 0, 0, hD, 0, 0)
        ref = np.tril(hD.get())
        assert relfro(np.tril(got[b]), ref) <= 1e-13, b
        assert relfro(dg[b], hD.diag(n)) <= 1e-13, b
        bad = int(np.argmax(np.diag(ref) == 0)) + 1 if (np.diag(ref) == 0).any() else 0
        assert inf[b] == bad, (b, inf[b], bad)
    # the same instances through the back-to-back batch kernel agree to rounding
    D2 = bf.DMatBatch(n, n, nb)
    bf.lib.blasfeo_dpotrf_l_batch(nb, n, src.ref, 0, 0, D2.ref, 0, 0, None, None)
    torch.cuda.synchronize()
    assert relfro(np.tril(D2.unpack_all()), np.tril(got)) <= 1e-13


def test_potrf_il_rejects(bf):
    from blasfeo_b200.api import DMatBatchIL
    a = DMatBatchIL(20, 20, 4)
    assert bf.lib.blasfeo_dpotrf_l_batch_il(4, 20, a.ref, a.ref, None, None) == 4   # n > 16
    b = DMatBatchIL(16, 16, 4)
    assert bf.lib.blasfeo_dpotrf_l_batch_il(5, 16, b.ref, b.ref, None, None) == 1   # batch beyond the slab


def _il_chain(bf, A, R, Cm, G, shift):
    import torch
    from blasfeo_b200.api import DMatBatchIL
    nb, m, k = A.shape
    ins = []
    for X in (A, R, Cm, G):
        ins.append(DMatBatchIL(X.shape[1], X.shape[2], nb).from_batch(bf.DMatBatch(X.shape[1], X.shape[2],
                                                                                   nb).pack_all(X)))
    outs = [DMatBatchIL(m, m, nb) for _ in range(3)]
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il(nb, m, k, shift, *(x.ref for x in ins),
                                                          *(x.ref for x in outs), C.c_void_p(info.data_ptr()), None)
    assert st == 0
    res = [o.to_batch(bf.DMatBatch(m, m, nb)) for o in outs]
    torch.cuda.synchronize()
    return res, info.cpu().numpy()


def test_chain_il_vs_golden_reference_outputs(bf):
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cfg2.npz"))
    (dL, dX, dD), info = _il_chain(bf, g["A"], g["R"], g["C"], g["G"], 16.0)
    assert (info == 0).all()
    L, X, D = dL.unpack_all(), dX.unpack_all(), dD.unpack_all()
    for b in range(g["A"].shape[0]):
        assert relfro(np.tril(L[b]), g["L"][b]) <= 1e-13
        assert relfro(X[b], g["X"][b]) <= 1e-13
        assert relfro(D[b], g["D"][b]) <= 1e-13


@pytest.mark.parametrize("nb,k", [(1037, 32), (45, 7), (8, 1)])
def test_chain_il_vs_back_to_back_and_oracle(bf, nb, k):
    """Partial last group, partial last warp, k not a multiple of 4, and one
    instance with a zero row of A under shift 0 (zero pivot, info = row + 1)."""
    import torch
    rng = np.random.default_rng(nb + k)
    m = 16
    A = rng.standard_normal((nb, m, k))
    R, Cm, G = (rng.standard_normal((nb, m, m)) for _ in range(3))
    shift = 0.0 if k >= m else 16.0
    bad = min(5, nb - 1)
    if shift == 0.0:
        A[bad, 5, :] = 0.0
    (dL, dX, dD), info = _il_chain(bf, A, R, Cm, G, shift)
    # the back-to-back kernel on the same instances
    bb = [bf.DMatBatch(X.shape[1], X.shape[2], nb).pack_all(X) for X in (A, R, Cm, G)]
    oL, oX, oD = (bf.DMatBatch(m, m, nb) for _ in range(3))
    info2 = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    assert bf.lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(nb, m, k, shift, *(x.ref for x in bb), oL.ref, oX.ref,
                                                         oD.ref, C.c_void_p(info2.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(info, info2.cpu().numpy())
    if shift == 0.0:
        assert info[bad] == 6 and (np.delete(info, bad) == 0).all()
    else:
        assert (info == 0).all()
    L, X, D, dg = dL.unpack_all(), dX.unpack_all(), dD.unpack_all(), dL.diag_all(m)
    ok = info == 0
    assert relfro(np.tril(L[ok]), np.tril(oL.unpack_all()[ok])) <= 1e-13
    assert relfro(X[ok], oX.unpack_all()[ok]) <= 1e-13
    assert relfro(D[ok], oD.unpack_all()[ok]) <= 1e-13
    assert relfro(dg[ok], oL.diag_all(m)[ok]) <= 1e-13
    orc = oracle_api()
    from oracle.pyoracle import HostMat
    for b in sorted({0, nb // 2, nb - 1}):
        if not ok[b]:
            continue
        hS = HostMat(m, m).set(A[b] @ A[b].T + shift * np.eye(m))
        hL = HostMat(m, m)
        orc.potrf_l("d", m, hS, 0, 0, hL, 0, 0)
        Lr = np.tril(hL.get())
        Xr = np.linalg.solve(Lr, R[b].T).T
        assert relfro(np.tril(L[b]), Lr) <= 1e-13
        assert relfro(X[b], Xr) <= 1e-12
        assert relfro(D[b], Cm[b] - Xr @ G[b].T) <= 1e-12


def test_chain_il_rejects(bf):
    from blasfeo_b200.api import DMatBatchIL
    A, Q = DMatBatchIL(16, 32, 4), [DMatBatchIL(16, 16, 4) for _ in range(6)]
    f = bf.lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il
    assert f(4, 12, 32, 1.0, A.ref, *(x.ref for x in Q), None, None) == 4      # m != 16
    assert f(4, 16, 32, 1.0, A.ref, *(x.ref for x in Q), None, None) == 0
    assert f(5, 16, 32, 1.0, A.ref, *(x.ref for x in Q), None, None) == 1      # batch beyond the slabs
    assert f(4, 16, 31, 1.0, A.ref, *(x.ref for x in Q), None, None) == 1      # k disagrees with sA
    B = DMatBatchIL(16, 12, 4)
    assert f(4, 16, 32, 1.0, A.ref, B.ref, *(x.ref for x in Q[1:]), None, None) == 1  # R not 16 x 16
    assert f(0, 16, 32, 1.0, A.ref, *(x.ref for x in Q), None, None) == 0
