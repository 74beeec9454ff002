"""GPU parity of the adjacent variants through the C ABI -- syrk_ln_mn,
trsm_rltu, potrf_l_mn, getrf_np (single instance with row/column offsets and
uniform batches, both precisions) -- against the CPU oracle on the same
seeded inputs and against the golden outputs of the compiled reference."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, tol

pytestmark = pytest.mark.gpu
NP = {"d": np.float64, "s": np.float32}
TOL = {"d": 1e-13, "s": 2e-5}
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    blasfeo_b200.set_sync(True)
    return blasfeo_b200


@pytest.fixture(scope="module")
def orc():
    return oracle_api()


def host(m, n, prec, data=None):
    from oracle.pyoracle import HostMat
    h = HostMat(m, n, NP[prec])
    if data is not None:
        h.set(data)
    return h


def dev(bf, m, n, prec, data=None):
    M = (bf.DMat if prec == "d" else bf.SMat)(m, n)
    if data is not None:
        M.pack(np.asarray(data, dtype=NP[prec]))
    return M


def fn(bf, prec, name):
    return getattr(bf, "blasfeo_%s%s" % (prec, name))


@pytest.mark.parametrize("prec", ["d", "s"])
def test_adjacent_vs_golden(bf, prec):
    g = np.load(os.path.join(GOLD, "adjacent.npz"))
    A, B, Cm = g[prec + "_syrkmn_A"], g[prec + "_syrkmn_B"], g[prec + "_syrkmn_C"]
    m, k = A.shape
    n = B.shape[0]
    dD = dev(bf, m, n, prec)
    fn(bf, prec, "syrk_ln_mn")(m, n, k, 0.5, dev(bf, m, k, prec, A), 0, 0, dev(bf, n, k, prec, B), 0, 0, -1.5,
                               dev(bf, m, n, prec, Cm), 0, 0, dD, 0, 0)
    want = g[prec + "_syrkmn_D"]
    assert relfro(np.tril(dD.unpack()), np.tril(want)) <= tol(prec, 10)
    dY = dev(bf, m, n, prec)
    fn(bf, prec, "trsm_rltu")(m, n, 1.25, dev(bf, n, n, prec, g[prec + "_trsmu_L"]), 0, 0,
                              dev(bf, m, n, prec, g[prec + "_trsmu_X"]), 0, 0, dY, 0, 0)
    assert relfro(dY.unpack(), g[prec + "_trsmu_Y"]) <= tol(prec, 10)
    dP = dev(bf, m, m, prec)
    fn(bf, prec, "potrf_l_mn")(m, n, dev(bf, m, m, prec, g[prec + "_potrfmn_S"]), 0, 0, dP, 0, 0)
    Lw = g[prec + "_potrfmn_L"]
    assert relfro(np.tril(dP.unpack())[:, :n], np.tril(Lw)[:, :n]) <= tol(prec, 10)
    assert relfro(dP.diag_array(n), g[prec + "_potrfmn_dA"]) <= tol(prec, 10)
    assert dP.use_dA == 1
    for tag in ("sq", "rect"):
        M = g[prec + "_lunp_%s_in" % tag]
        r, c = M.shape
        dLU = dev(bf, r, c, prec)
        fn(bf, prec, "getrf_np")(r, c, dev(bf, r, c, prec, M), 0, 0, dLU, 0, 0)
        assert relfro(dLU.unpack(), g[prec + "_lunp_%s" % tag]) <= tol(prec, 10), tag
        assert relfro(dLU.diag_array(min(r, c)), g[prec + "_lunp_%s_dA" % tag]) <= tol(prec, 10), tag


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("off", [(1, 2, 3), (3, 0, 1), (4, 5, 0)])
def test_adjacent_offsets_vs_oracle(bf, orc, prec, off):
    oi, oj, od = off
    rng = np.random.default_rng(23 + oi + 2 * oj + 3 * od)
    m, n, k = 37, 21, 11
    A, B, Cm = rng.standard_normal((m + oi, k + oj)), rng.standard_normal((n + oi, k + oj)), rng.standard_normal((m + oi, n + oj))
    Lu = np.tril(rng.standard_normal((n + oi, n + oj)), -1) * 0.3 + 9 * np.eye(n + oi, n + oj)
    X = rng.standard_normal((m + oi, n + oj))
    g = rng.standard_normal((m + oi, m + oi))
    S = g @ g.T + (m + oi) * np.eye(m + oi)
    M = rng.standard_normal((m + oi, n + oj)) + 6 * np.eye(m + oi, n + oj)
    D0 = rng.standard_normal((m + od, m + od))
    # oracle
    hD, hY, hP, hLU = (host(m + od, n + od, prec, D0[:, : n + od]), host(m + od, n + od, prec, D0[:, : n + od]),
                       host(m + od, m + od, prec, D0), host(m + od, n + od, prec, D0[:, : n + od]))
    orc.syrk_ln_mn(prec, m, n, k, 1.0, host(m + oi, k + oj, prec, A), oi, oj, host(n + oi, k + oj, prec, B), oi, oj,
                   0.5, host(m + oi, n + oj, prec, Cm), oi, oj, hD, od, od)
    orc.trsm_rltu(prec, m, n, -0.5, host(n + oi, n + oj, prec, Lu), oi, oj, host(m + oi, n + oj, prec, X), oi, oj,
                  hY, od, od)
    orc.potrf_l_mn(prec, m, n, host(m + oi, m + oi, prec, S), oi, oi, hP, od, od)
    orc.getrf_np(prec, m, n, host(m + oi, n + oj, prec, M), oi, oj, hLU, od, od)
    # device
    dD, dY, dP, dLU = (dev(bf, m + od, n + od, prec, D0[:, : n + od]), dev(bf, m + od, n + od, prec, D0[:, : n + od]),
                       dev(bf, m + od, m + od, prec, D0), dev(bf, m + od, n + od, prec, D0[:, : n + od]))
    fn(bf, prec, "syrk_ln_mn")(m, n, k, 1.0, dev(bf, m + oi, k + oj, prec, A), oi, oj, dev(bf, n + oi, k + oj, prec, B),
                               oi, oj, 0.5, dev(bf, m + oi, n + oj, prec, Cm), oi, oj, dD, od, od)
    fn(bf, prec, "trsm_rltu")(m, n, -0.5, dev(bf, n + oi, n + oj, prec, Lu), oi, oj, dev(bf, m + oi, n + oj, prec, X),
                              oi, oj, dY, od, od)
    fn(bf, prec, "potrf_l_mn")(m, n, dev(bf, m + oi, m + oi, prec, S), oi, oi, dP, od, od)
    fn(bf, prec, "getrf_np")(m, n, dev(bf, m + oi, n + oj, prec, M), oi, oj, dLU, od, od)
    # untouched parts (upper part of the trapezoids, columns >= n of the potrf target) keep D0
    for name, d, h in (("syrk", dD, hD), ("trsm", dY, hY), ("potrf", dP, hP), ("getrf", dLU, hLU)):
        assert relfro(d.unpack(), h.get()) <= tol(prec, 10), name
    assert relfro(dP.diag_array(n), hP.diag(n)) <= tol(prec, 10)
    assert relfro(dLU.diag_array(n), hLU.diag(n)) <= tol(prec, 10)
    assert dP.use_dA == (1 if od == 0 else 0) and dLU.use_dA == (1 if od == 0 else 0)


@pytest.mark.parametrize("prec", ["d", "s"])
def test_adjacent_batches_vs_oracle(bf, orc, prec):
    import torch
    rng = np.random.default_rng(99)
    nb, m, n, k = 9, 30, 17, 6

    def batch(arr):
        b, r, c = arr.shape
        return (bf.DMatBatch if prec == "d" else bf.SMatBatch)(r, c, b).pack_all(arr)
    A, B, Cm = rng.standard_normal((nb, m, k)), rng.standard_normal((nb, n, k)), rng.standard_normal((nb, m, n))
    dA, dB, dC, dD = batch(A), batch(B), batch(Cm), batch(np.zeros((nb, m, n)))
    assert getattr(bf.lib, "blasfeo_%ssyrk_ln_mn_batch" % prec)(nb, m, n, k, 2.0, dA.ref, 0, 0, dB.ref, 0, 0, -1.0,
                                                                dC.ref, 0, 0, dD.ref, 0, 0, None) == 0
    L = np.tril(rng.standard_normal((nb, n, n)), -1) * 0.3 + 3 * np.eye(n)
    X = rng.standard_normal((nb, m, n))
    dL, dX, dY = batch(L), batch(X), batch(np.zeros((nb, m, n)))
    assert getattr(bf.lib, "blasfeo_%strsm_rltu_batch" % prec)(nb, m, n, 1.0, dL.ref, 0, 0, dX.ref, 0, 0, dY.ref, 0, 0,
                                                               None) == 0
    G = rng.standard_normal((nb, m, m))
    S = G @ G.transpose(0, 2, 1) + m * np.eye(m)
    S[4, 8, 8] = -1e3  # first non-positive pivot at 8 -> info 9
    dS, dP = batch(S), batch(np.zeros((nb, m, m)))
    info = torch.full((nb,), -7, dtype=torch.int32, device="cuda")
    assert getattr(bf.lib, "blasfeo_%spotrf_l_mn_batch" % prec)(nb, m, n, dS.ref, 0, 0, dP.ref, 0, 0,
                                                                C.c_void_p(info.data_ptr()), None) == 0
    M = rng.standard_normal((nb, m, n)) + 6 * np.eye(m, n)
    dM, dLU = batch(M), batch(np.zeros((nb, m, n)))
    info2 = torch.full((nb,), -7, dtype=torch.int32, device="cuda")
    assert getattr(bf.lib, "blasfeo_%sgetrf_np_batch" % prec)(nb, m, n, dM.ref, 0, 0, dLU.ref, 0, 0,
                                                              C.c_void_p(info2.data_ptr()), None) == 0
    torch.cuda.synchronize()
    inf = info.cpu().numpy()
    assert inf[4] == 9 and (np.delete(inf, 4) == 0).all(), inf
    assert (info2.cpu().numpy() == 0).all()
    gD, gY, gP, gLU = dD.unpack_all(), dY.unpack_all(), dP.unpack_all(), dLU.unpack_all()
    for b in (0, 4, nb - 1):
        hD = host(m, n, prec, np.zeros((m, n)))
        orc.syrk_ln_mn(prec, m, n, k, 2.0, host(m, k, prec, A[b]), 0, 0, host(n, k, prec, B[b]), 0, 0, -1.0,
                       host(m, n, prec, Cm[b]), 0, 0, hD, 0, 0)
        assert relfro(gD[b], hD.get()) <= tol(prec, 10)
        hY = host(m, n, prec)
        orc.trsm_rltu(prec, m, n, 1.0, host(n, n, prec, L[b]), 0, 0, host(m, n, prec, X[b]), 0, 0, hY, 0, 0)
        assert relfro(gY[b], hY.get()) <= tol(prec, 10)
        hP = host(m, m, prec)
        orc.potrf_l_mn(prec, m, n, host(m, m, prec, S[b]), 0, 0, hP, 0, 0)
        if b != 4:
            assert relfro(np.tril(gP[b])[:, :n], np.tril(hP.get())[:, :n]) <= tol(prec, 10)
        hLU = host(m, n, prec)
        orc.getrf_np(prec, m, n, host(m, n, prec, M[b]), 0, 0, hLU, 0, 0)
        assert relfro(gLU[b], hLU.get()) <= tol(prec, 10)
