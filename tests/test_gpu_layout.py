"""GPU tests of the host<->device layout converters through the C ABI:
blasfeo_pack_tran_*mat / blasfeo_unpack_tran_*mat (the reference's rule,
pinned on the compiled reference by tests/test_oracle.py), and the batched
column-major <-> uniform-slab converters, against independent numpy
restatements of the panel layout.  Layout conversions are exact: every check
is bit equality."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
NP = {"d": np.float64, "s": np.float32}


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    blasfeo_b200.set_sync(True)
    return blasfeo_b200


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("shape", [(5, 7, 1, 2), (12, 3, 0, 0), (1, 9, 3, 1), (9, 1, 2, 0), (64, 33, 4, 5)])
def test_pack_unpack_tran(bf, prec, shape):
    m, n, ai, aj = shape
    rng = np.random.default_rng(m * 13 + n)
    A = np.asfortranarray(rng.standard_normal((m, n)).astype(NP[prec]))
    rows, cols = max(n + ai, m + ai) + 1, max(m + aj, n + aj) + 2
    base = rng.standard_normal((rows, cols)).astype(NP[prec])
    D = (bf.DMat if prec == "d" else bf.SMat)(rows, cols).pack(base)
    getattr(bf.lib, "blasfeo_pack_tran_%smat" % prec)(m, n, _ptr(A), m, D.ref, ai, aj)
    assert bf.lib.blasfeo_b200_last_error() == 0
    want = base.copy()
    want[ai:ai + n, aj:aj + m] = A.T
    assert np.array_equal(D.unpack(), want)
    out = np.asfortranarray(np.zeros((n + 3, m), dtype=NP[prec]))
    getattr(bf.lib, "blasfeo_unpack_tran_%smat" % prec)(m, n, D.ref, ai, aj, _ptr(out), n + 3)
    assert bf.lib.blasfeo_b200_last_error() == 0
    assert np.array_equal(out[:n], want[ai:ai + m, aj:aj + n].T)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("case", [(37, 5, 7, 0, 0, 0), (11, 16, 16, 1, 2, 0), (3, 9, 4, 0, 1, 5)])
def test_batch_pack_unpack(bf, prec, case):
    batch, m, n, bi, bj, gap = case
    rng = np.random.default_rng(batch + m + n)
    lda = m + 2
    stride = lda * n + gap          # gap > 0: instances not back to back (per-instance copies)
    host = rng.standard_normal(stride * batch + 8).astype(NP[prec])
    Bt = (bf.DMatBatch if prec == "d" else bf.SMatBatch)(m + bi + 1, n + bj + 1, batch)
    base = rng.standard_normal((batch, m + bi + 1, n + bj + 1)).astype(NP[prec])
    Bt.pack_all(base)
    fn_p = getattr(bf.lib, "blasfeo_pack_%smat_batch" % prec)
    fn_u = getattr(bf.lib, "blasfeo_unpack_%smat_batch" % prec)
    assert fn_p(batch, m, n, _ptr(host), lda, stride, Bt.ref, bi, bj, None) == 0
    want = base.copy()
    for b in range(batch):
        blk = host[b * stride: b * stride + lda * n].reshape(n, lda).T[:m]
        want[b, bi:bi + m, bj:bj + n] = blk
    assert np.array_equal(Bt.unpack_all(), want)
    out = np.zeros_like(host)
    assert fn_u(batch, m, n, Bt.ref, bi, bj, _ptr(out), lda, stride, None) == 0
    for b in range(batch):
        got = out[b * stride: b * stride + lda * n].reshape(n, lda).T[:m]
        assert np.array_equal(got, want[b, bi:bi + m, bj:bj + n])
    # rejected before any device work: block outside the slab, stride too small
    assert fn_p(batch, m + bi + 2, n, _ptr(host), m + bi + 2, stride * 4, Bt.ref, 0, 0, None) == 1
    assert fn_p(batch, m, n, _ptr(host), lda, lda * (n - 1) + m - 1, Bt.ref, bi, bj, None) == 1
