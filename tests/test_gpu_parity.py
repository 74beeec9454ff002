"""GPU parity: every hot-path routine through the C ABI vs the CPU oracle.

Mirrors the reference's differential harness (tests/test_x.c: routine vs
blasfeo_ref_* on identical inputs, sweeping sizes and row offsets), with the
tolerances of this port: relative Frobenius error <= 1e-13 in FP64 and
<= 2e-5 in FP32, identical pivot vectors.
"""
import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, spd, tol

pytestmark = pytest.mark.gpu

TOL = {"d": 1e-13, "s": 2e-5}
NP = {"d": np.float64, "s": np.float32}


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
        M.pack(data)
    return M


GEMM_CASES = [(64, 64, 64, 0, 0, 0, 0), (16, 16, 16, 0, 0, 0, 0), (17, 13, 9, 0, 0, 0, 0), (5, 3, 7, 1, 2, 3, 1),
              (1, 1, 1, 0, 0, 0, 0), (33, 70, 21, 2, 1, 0, 3), (130, 65, 40, 0, 0, 0, 0), (8, 8, 0, 0, 0, 0, 0),
              # the mixed-op stream's largest sizes (m, n, k up to 384)
              (384, 384, 384, 0, 0, 0, 0), (300, 384, 211, 0, 0, 0, 0), (384, 97, 384, 3, 0, 1, 2)]


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("case", GEMM_CASES)
@pytest.mark.parametrize("ab", [(1.0, 0.0), (1.5, -0.5)])
def test_gemm_nt(bf, orc, prec, case, ab):
    m, n, k, ai, bi, ci, di = case
    alpha, beta = ab
    rng = np.random.default_rng(m * 131 + n * 7 + k)
    A = rng.uniform(-1, 1, (m + ai, k + 1))
    B = rng.uniform(-1, 1, (n + bi, k + 1))
    Cm = rng.uniform(-1, 1, (m + ci, n + 2))
    D0 = rng.uniform(-1, 1, (m + di, n + 2))
    hA, hB, hC, hD = host(m + ai, k + 1, prec, A), host(n + bi, k + 1, prec, B), host(m + ci, n + 2, prec, Cm), host(m + di, n + 2, prec, D0)
    orc.gemm_nt(prec, m, n, k, alpha, hA, ai, 1, hB, bi, 1, beta, hC, ci, 1, hD, di, 1)
    dA, dB, dC, dD = dev(bf, m + ai, k + 1, prec, A), dev(bf, n + bi, k + 1, prec, B), dev(bf, m + ci, n + 2, prec, Cm), dev(bf, m + di, n + 2, prec, D0)
    getattr(bf, "blasfeo_%sgemm_nt" % prec)(m, n, k, alpha, dA, ai, 1, dB, bi, 1, beta, dC, ci, 1, dD, di, 1)
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mk", [(16, 32, 0), (13, 7, 1), (64, 64, 0), (5, 9, 3), (100, 20, 2)])
def test_syrk_ln(bf, orc, prec, mk):
    m, k, off = mk
    rng = np.random.default_rng(m + 1000 * k)
    A = rng.standard_normal((m + off, k))
    Cm = rng.standard_normal((m + off, m + off))
    D0 = rng.standard_normal((m + off, m + off))
    hA, hC, hD = host(m + off, k, prec, A), host(m + off, m + off, prec, Cm), host(m + off, m + off, prec, D0)
    orc.syrk_ln(prec, m, k, 0.7, hA, off, 0, hA, off, 0, 1.3, hC, off, off, hD, off, off)
    dA, dC, dD = dev(bf, m + off, k, prec, A), dev(bf, m + off, m + off, prec, Cm), dev(bf, m + off, m + off, prec, D0)
    getattr(bf, "blasfeo_%ssyrk_ln" % prec)(m, k, 0.7, dA, off, 0, dA, off, 0, 1.3, dC, off, off, dD, off, off)
    # the strictly-upper part of D must be untouched as well
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]


POTRF_N = [1, 2, 3, 4, 5, 7, 13, 16, 17, 31, 33, 50, 56, 60, 64, 100, 129, 200, 257, 300, 384]


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", POTRF_N)
def test_potrf_l(bf, orc, prec, n):
    rng = np.random.default_rng(n)
    S = spd(rng, n)
    D0 = rng.standard_normal((n, n))
    hC, hD = host(n, n, prec, S), host(n, n, prec, D0)
    orc.potrf_l(prec, n, hC, 0, 0, hD, 0, 0)
    dC, dD = dev(bf, n, n, prec, S), dev(bf, n, n, prec, D0)
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, dC, 0, 0, dD, 0, 0)
    assert relfro(dD.unpack(), hD.get()) <= tol(prec, 10 if n > 100 else 1)
    assert relfro(dD.diag_array(n), hD.diag(n)) <= tol(prec, 10)
    assert dD.use_dA == n


@pytest.mark.parametrize("prec", ["d", "s"])
def test_potrf_l_offsets(bf, orc, prec):
    rng = np.random.default_rng(5)
    n = 21
    S = spd(rng, n)
    big = rng.standard_normal((n + 3, n + 5))
    big[2:2 + n, 1:1 + n] = S
    hC, hD = host(n + 3, n + 5, prec, big), host(n + 4, n + 4, prec)
    orc.potrf_l(prec, n, hC, 2, 1, hD, 3, 2)
    dC, dD = dev(bf, n + 3, n + 5, prec, big), dev(bf, n + 4, n + 4, prec, np.zeros((n + 4, n + 4)))
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, dC, 2, 1, dD, 3, 2)
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]
    assert dD.use_dA == 0


@pytest.mark.parametrize("prec", ["d", "s"])
def test_potrf_l_not_spd(bf, orc, prec):
    # non-positive pivots: L_jj = 0 and inverse 0, no error (reference rule)
    rng = np.random.default_rng(9)
    n = 24
    S = spd(rng, n)
    S[5, 5] = -1.0
    S[17, 17] = 0.0
    hC, hD = host(n, n, prec, S), host(n, n, prec)
    orc.potrf_l(prec, n, hC, 0, 0, hD, 0, 0)
    dC, dD = dev(bf, n, n, prec, S), dev(bf, n, n, prec, np.zeros((n, n)))
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, dC, 0, 0, dD, 0, 0)
    got, ref = dD.unpack(), hD.get()
    assert np.all(np.isfinite(got) == np.isfinite(ref))
    assert relfro(np.nan_to_num(got), np.nan_to_num(ref)) <= tol(prec, 100)
    assert dD.diag_array(n)[5] == 0.0


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mn", [(64, 64, 0, 0), (16, 16, 0, 0), (19, 13, 0, 0), (7, 30, 2, 1), (1, 1, 0, 0),
                                (100, 130, 0, 0), (64, 384, 1, 3), (384, 200, 0, 0)])
@pytest.mark.parametrize("alpha", [1.0, -2.0])
def test_trsm_rltn(bf, orc, prec, mn, alpha):
    m, n, bi, di = mn
    rng = np.random.default_rng(m * 17 + n)
    S = spd(rng, n)
    X = rng.standard_normal((m + bi, n))
    hS, hL = host(n, n, prec, S), host(n, n, prec)
    orc.potrf_l(prec, n, hS, 0, 0, hL, 0, 0)
    hB, hD = host(m + bi, n, prec, X), host(m + di, n, prec)
    orc.trsm_rltn(prec, m, n, alpha, hL, 0, 0, hB, bi, 0, hD, di, 0)
    dS, dL = dev(bf, n, n, prec, S), dev(bf, n, n, prec, np.zeros((n, n)))
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, dS, 0, 0, dL, 0, 0)
    dB, dD = dev(bf, m + bi, n, prec, X), dev(bf, m + di, n, prec, np.zeros((m + di, n)))
    getattr(bf, "blasfeo_%strsm_rltn" % prec)(m, n, alpha, dL, 0, 0, dB, bi, 0, dD, di, 0)
    assert relfro(dD.unpack(), hD.get()) <= tol(prec, 10)


@pytest.mark.parametrize("prec", ["d", "s"])
def test_trsm_rltn_uncached_diag(bf, orc, prec):
    # A given directly (use_dA == 0): the inverse diagonal is computed from A
    rng = np.random.default_rng(3)
    n, m = 12, 9
    L = np.tril(rng.uniform(0.5, 1.5, (n, n)))
    X = rng.standard_normal((m, n))
    hL, hB, hD = host(n, n, prec, L), host(m, n, prec, X), host(m, n, prec)
    orc.trsm_rltn(prec, m, n, 1.0, hL, 0, 0, hB, 0, 0, hD, 0, 0)
    dL, dB, dD = dev(bf, n, n, prec, L), dev(bf, m, n, prec, X), dev(bf, m, n, prec, np.zeros((m, n)))
    getattr(bf, "blasfeo_%strsm_rltn" % prec)(m, n, 1.0, dL, 0, 0, dB, 0, 0, dD, 0, 0)
    assert relfro(dD.unpack(), hD.get()) <= tol(prec, 10)
    assert dL.use_dA == n
    assert relfro(dL.diag_array(n), hL.diag(n)) <= TOL[prec]


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mn", [(64, 64), (16, 16), (1, 1), (5, 5), (37, 37), (40, 23), (23, 40), (130, 130),
                                (300, 300), (384, 384), (384, 250)])
def test_getrf_rp(bf, orc, prec, mn):
    m, n = mn
    rng = np.random.default_rng(m * 3 + n)
    M = rng.standard_normal((m, n))
    hC, hD = host(m, n, prec, M), host(m, n, prec)
    piv_ref = orc.getrf_rp(prec, m, n, hC, 0, 0, hD, 0, 0)
    dC, dD = dev(bf, m, n, prec, M), dev(bf, m, n, prec)
    piv = getattr(bf, "blasfeo_%sgetrf_rp" % prec)(m, n, dC, 0, 0, dD, 0, 0)
    assert np.array_equal(piv, piv_ref)
    t = tol(prec, 100)
    assert relfro(dD.unpack(), hD.get()) <= t
    k = min(m, n)
    assert relfro(dD.diag_array(k), hD.diag(k)) <= t


@pytest.mark.parametrize("prec", ["d", "s"])
def test_getrf_rp_ties_and_zero_pivot(bf, orc, prec):
    # equal |a| candidates: the first (lowest) row wins; a zero column gives inverse 0
    M = np.array([[1.0, 2.0, 0.0, 1.0], [-1.0, 1.0, 0.0, 2.0], [1.0, -3.0, 0.0, 0.5], [0.5, 1.0, 0.0, 4.0]])
    hC, hD = host(4, 4, prec, M), host(4, 4, prec)
    piv_ref = orc.getrf_rp(prec, 4, 4, hC, 0, 0, hD, 0, 0)
    dC, dD = dev(bf, 4, 4, prec, M), dev(bf, 4, 4, prec)
    piv = getattr(bf, "blasfeo_%sgetrf_rp" % prec)(4, 4, dC, 0, 0, dD, 0, 0)
    assert np.array_equal(piv, piv_ref)
    assert piv[0] == 0
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]
    assert dD.diag_array(4)[2] == 0.0


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mn", [(128, 64), (32, 16), (9, 9), (5, 3), (3, 5), (1, 1), (200, 100), (300, 150),
                                (384, 192), (100, 400), (70, 300)])
def test_geqrf(bf, orc, prec, mn):
    # wide cases: more than 256 trailing columns, updated in several chunks
    m, n = mn
    rng = np.random.default_rng(m + 7 * n)
    M = rng.standard_normal((m, n))
    hC, hD = host(m, n, prec, M), host(m, n, prec)
    orc.geqrf(prec, m, n, hC, 0, 0, hD, 0, 0)
    dC, dD = dev(bf, m, n, prec, M), dev(bf, m, n, prec)
    getattr(bf, "blasfeo_%sgeqrf" % prec)(m, n, dC, 0, 0, dD, 0, 0)
    t = tol(prec, 50)
    assert relfro(dD.unpack(), hD.get()) <= t
    k = min(m, n)
    assert relfro(dD.diag_array(k), hD.diag(k)) <= t


@pytest.mark.parametrize("prec", ["d", "s"])
def test_syrk_potrf_ln(bf, orc, prec):
    rng = np.random.default_rng(11)
    m, k = 16, 12
    A = rng.standard_normal((m, k))
    Cm = np.eye(m) * 2.0
    hA, hC, hD = host(m, k, prec, A), host(m, m, prec, Cm), host(m, m, prec)
    orc.syrk_potrf_ln(prec, m, k, hA, 0, 0, hA, 0, 0, hC, 0, 0, hD, 0, 0)
    dA, dC, dD = dev(bf, m, k, prec, A), dev(bf, m, m, prec, Cm), dev(bf, m, m, prec, np.zeros((m, m)))
    getattr(bf, "blasfeo_%ssyrk_%spotrf_ln" % (prec, prec))(m, k, dA, 0, 0, dA, 0, 0, dC, 0, 0, dD, 0, 0)
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]


@pytest.mark.parametrize("prec", ["d", "s"])
def test_trmm_rlnn(bf, orc, prec):
    rng = np.random.default_rng(12)
    m, n = 16, 12
    L = np.tril(rng.standard_normal((n, n)))
    B = rng.standard_normal((m, n))
    hL, hB, hD = host(n, n, prec, L), host(m, n, prec, B), host(m, n, prec)
    orc.trmm_rlnn(prec, m, n, 1.0, hL, 0, 0, hB, 0, 0, hD, 0, 0)
    dL, dB, dD = dev(bf, n, n, prec, L), dev(bf, m, n, prec, B), dev(bf, m, n, prec)
    getattr(bf, "blasfeo_%strmm_rlnn" % prec)(m, n, 1.0, dL, 0, 0, dB, 0, 0, dD, 0, 0)
    assert relfro(dD.unpack(), hD.get()) <= TOL[prec]


def test_aux_gecp_diare_rowsw(bf, orc):
    rng = np.random.default_rng(2)
    M = rng.standard_normal((9, 7))
    d = bf.DMat(9, 7).pack(M)
    e = bf.DMat(9, 7).pack(np.zeros((9, 7)))
    bf.blasfeo_dgecp(5, 4, d, 1, 2, e, 3, 1)
    ref = np.zeros((9, 7))
    ref[3:8, 1:5] = M[1:6, 2:6]
    assert np.array_equal(e.unpack(), ref)
    bf.blasfeo_ddiare(5, 2.5, d, 1, 0)
    M2 = M.copy()
    for l in range(5):
        M2[1 + l, l] += 2.5
    assert np.array_equal(d.unpack(), M2)
    bf.blasfeo_drowsw(7, d, 0, 0, d, 6, 0)
    M2[[0, 6], :] = M2[[6, 0], :]
    assert np.array_equal(d.unpack(), M2)


def test_level2_solves(bf, orc):
    rng = np.random.default_rng(4)
    n = 37
    S = spd(rng, n)
    b = rng.standard_normal(n)
    dS, dL = bf.DMat(n, n).pack(S), bf.DMat(n, n)
    bf.blasfeo_dpotrf_l(n, dS, 0, 0, dL, 0, 0)
    xb, y, x = bf.DVec(n).pack(b), bf.DVec(n), bf.DVec(n)
    bf.blasfeo_dtrsv_lnn(n, dL, 0, 0, xb, 0, y, 0)
    bf.blasfeo_dtrsv_ltn(n, dL, 0, 0, y, 0, x, 0)
    xs = x.unpack()
    assert np.linalg.norm(S @ xs - b) / (np.linalg.norm(S) * np.linalg.norm(xs)) < 1e-14
    r = bf.DVec(n)
    bf.blasfeo_dgemv_n(n, n, 1.0, dS, 0, 0, x, 0, -1.0, xb, 0, r, 0)
    assert np.abs(r.unpack()).max() < 1e-11

