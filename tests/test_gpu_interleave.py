"""GPU tests of the batch-interleaved layout: lossless conversion from and to
the back-to-back slab (whole and partial groups of 16), and potrf_l on it
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
