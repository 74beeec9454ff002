"""GPU parity of the column-major drop-in (blasfeo_cm_*): device column-major
matrices with row/column offsets and leading dimensions larger than the
blocks.  Each routine must give exactly the result of the panel-major routine
of the same name on the same blocks (the same kernels run), agree with the CPU
oracle within the FP64 / FP32 tolerances of the panel-major parity tests, and
leave everything outside the block (or triangle) it writes untouched."""
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


def cm(bf, prec, data):
    return (bf.CmDMat if prec == "d" else bf.CmSMat)(*data.shape).pack(data)


def pm(bf, prec, data):
    return (bf.DMat if prec == "d" else bf.SMat)(*data.shape).pack(data)


def host(prec, data):
    from oracle.pyoracle import HostMat
    return HostMat(data.shape[0], data.shape[1], NP[prec]).set(data)


def outside_unchanged(got, before, r0, c0, m, n, lower=False):
    mask = np.ones(got.shape, dtype=bool)
    blk = np.ones((m, n), dtype=bool)
    if lower:
        blk = np.tril(blk)
    mask[r0:r0 + m, c0:c0 + n] &= ~blk
    return np.array_equal(got[mask], np.asarray(before, dtype=got.dtype)[mask])


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("case", [(64, 64, 64, 0, 0, 0, 0), (17, 13, 9, 1, 2, 3, 1), (5, 3, 7, 2, 0, 1, 4),
                                  (130, 65, 40, 0, 3, 0, 2), (8, 8, 0, 0, 0, 0, 0)])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (1.5, -0.5)])
def test_cm_gemm_nt(bf, orc, prec, case, ab):
    m, n, k, ai, bi, ci, di = case
    alpha, beta = ab
    rng = np.random.default_rng(m * 31 + n * 7 + k + ai)
    A = rng.uniform(-1, 1, (m + ai + 2, k + 3)).astype(NP[prec])
    B = rng.uniform(-1, 1, (n + bi + 1, k + 3)).astype(NP[prec])
    Cm = rng.uniform(-1, 1, (m + ci + 3, n + 2)).astype(NP[prec])
    D0 = rng.uniform(-1, 1, (m + di + 1, n + 4)).astype(NP[prec])
    cA, cB, cC, cD = cm(bf, prec, A), cm(bf, prec, B), cm(bf, prec, Cm), cm(bf, prec, D0)
    getattr(bf, "blasfeo_cm_%sgemm_nt" % prec)(m, n, k, alpha, cA, ai, 1, cB, bi, 2, beta, cC, ci, 1, cD, di, 3)
    got = cD.unpack()
    pA, pB, pC, pD = pm(bf, prec, A), pm(bf, prec, B), pm(bf, prec, Cm), pm(bf, prec, D0)
    getattr(bf, "blasfeo_%sgemm_nt" % prec)(m, n, k, alpha, pA, ai, 1, pB, bi, 2, beta, pC, ci, 1, pD, di, 3)
    assert np.array_equal(got[di:di + m, 3:3 + n], pD.unpack()[di:di + m, 3:3 + n])
    hA, hB, hC, hD = host(prec, A), host(prec, B), host(prec, Cm), host(prec, D0)
    orc.gemm_nt(prec, m, n, k, alpha, hA, ai, 1, hB, bi, 2, beta, hC, ci, 1, hD, di, 3)
    assert relfro(got, hD.get()) <= TOL[prec]
    assert outside_unchanged(got, D0, di, 3, m, n)


@pytest.mark.parametrize("mk", [(16, 32, 0), (13, 7, 1), (100, 20, 2)])
def test_cm_syrk_ln(bf, orc, mk):
    m, k, off = mk
    rng = np.random.default_rng(m + 100 * k)
    A = rng.standard_normal((m + off + 1, k))
    Cm = rng.standard_normal((m + off, m + off))
    D0 = rng.standard_normal((m + off + 2, m + off + 1))
    cA, cC, cD = cm(bf, "d", A), cm(bf, "d", Cm), cm(bf, "d", D0)
    bf.blasfeo_cm_dsyrk_ln(m, k, 0.7, cA, off, 0, cA, off + 1, 0, 1.3, cC, off, off, cD, off + 1, off)
    got = cD.unpack()
    pA, pC, pD = pm(bf, "d", A), pm(bf, "d", Cm), pm(bf, "d", D0)
    bf.blasfeo_dsyrk_ln(m, k, 0.7, pA, off, 0, pA, off + 1, 0, 1.3, pC, off, off, pD, off + 1, off)
    blk = np.tril(np.ones((m, m), dtype=bool))
    assert np.array_equal(got[off + 1:off + 1 + m, off:off + m][blk], pD.unpack()[off + 1:off + 1 + m, off:off + m][blk])
    hA, hC, hD = host("d", A), host("d", Cm), host("d", D0)
    orc.syrk_ln("d", m, k, 0.7, hA, off, 0, hA, off + 1, 0, 1.3, hC, off, off, hD, off + 1, off)
    assert relfro(got, hD.get()) <= TOL["d"]
    # the strictly upper part of the block and everything around it untouched
    assert outside_unchanged(got, D0, off + 1, off, m, m, lower=True)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mn", [(64, 64), (13, 21), (40, 7), (200, 33)])
def test_cm_trsm_rltn(bf, orc, prec, mn):
    m, n = mn
    rng = np.random.default_rng(m * 3 + n)
    L = np.linalg.cholesky(spd(rng, n))
    Abig = rng.standard_normal((n + 2, n + 1))
    Abig[2:2 + n, 1:1 + n] = L
    Abig = Abig.astype(NP[prec])
    B = rng.standard_normal((m + 1, n + 3)).astype(NP[prec])
    D0 = rng.standard_normal((m + 3, n + 2)).astype(NP[prec])
    cA, cB, cD = cm(bf, prec, Abig), cm(bf, prec, B), cm(bf, prec, D0)
    getattr(bf, "blasfeo_cm_%strsm_rltn" % prec)(m, n, 1.0, cA, 2, 1, cB, 1, 3, cD, 3, 2)
    got = cD.unpack()
    pA, pB, pD = pm(bf, prec, Abig), pm(bf, prec, B), pm(bf, prec, D0)
    getattr(bf, "blasfeo_%strsm_rltn" % prec)(m, n, 1.0, pA, 2, 1, pB, 1, 3, pD, 3, 2)
    assert np.array_equal(got[3:3 + m, 2:2 + n], pD.unpack()[3:3 + m, 2:2 + n])
    hA, hB, hD = host(prec, Abig), host(prec, B), host(prec, D0)
    orc.trsm_rltn(prec, m, n, 1.0, hA, 2, 1, hB, 1, 3, hD, 3, 2)
    assert relfro(got, hD.get()) <= tol(prec, 10)
    assert outside_unchanged(got, D0, 3, 2, m, n)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", [1, 5, 16, 33, 64, 100, 129, 200])
def test_cm_potrf_l(bf, orc, prec, n):
    rng = np.random.default_rng(n + 7)
    big = rng.standard_normal((n + 3, n + 2))
    big[1:1 + n, 2:2 + n] = spd(rng, n)
    big = big.astype(NP[prec])
    D0 = rng.standard_normal((n + 2, n + 4)).astype(NP[prec])
    cC, cD = cm(bf, prec, big), cm(bf, prec, D0)
    getattr(bf, "blasfeo_cm_%spotrf_l" % prec)(n, cC, 1, 2, cD, 2, 1)
    got = cD.unpack()
    pC, pD = pm(bf, prec, big), pm(bf, prec, D0)
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, pC, 1, 2, pD, 2, 1)
    blk = np.tril(np.ones((n, n), dtype=bool))
    assert np.array_equal(got[2:2 + n, 1:1 + n][blk], pD.unpack()[2:2 + n, 1:1 + n][blk])
    hC, hD = host(prec, big), host(prec, D0)
    orc.potrf_l(prec, n, hC, 1, 2, hD, 2, 1)
    assert relfro(np.tril(got[2:2 + n, 1:1 + n]), np.tril(hD.get()[2:2 + n, 1:1 + n])) <= tol(prec, 10 if n > 100 else 1)
    assert outside_unchanged(got, D0, 2, 1, n, n, lower=True)


@pytest.mark.parametrize("prec", ["d", "s"])
def test_cm_potrf_l_in_place_and_not_spd(bf, orc, prec):
    # C and D the same matrix and block; non-positive pivots give zero columns (reference rule)
    rng = np.random.default_rng(3)
    n = 24
    S = spd(rng, n)
    S[5, 5] = -1.0
    S[17, 17] = 0.0
    S = S.astype(NP[prec])
    c = cm(bf, prec, S)
    getattr(bf, "blasfeo_cm_%spotrf_l" % prec)(n, c, 0, 0, c, 0, 0)
    got = c.unpack()
    p = pm(bf, prec, S)
    getattr(bf, "blasfeo_%spotrf_l" % prec)(n, p, 0, 0, p, 0, 0)
    assert np.array_equal(np.tril(got), np.tril(p.unpack()))
    assert np.array_equal(np.triu(got, 1), np.triu(S, 1))


@pytest.mark.parametrize("mn", [(64, 64), (37, 20), (20, 37), (130, 90)])
def test_cm_getrf_rp(bf, orc, mn):
    m, n = mn
    rng = np.random.default_rng(m + 3 * n)
    big = rng.standard_normal((m + 2, n + 1))
    D0 = rng.standard_normal((m + 1, n + 3))
    cC, cD = cm(bf, "d", big), cm(bf, "d", D0)
    piv = bf.blasfeo_cm_dgetrf_rp(m, n, cC, 2, 1, cD, 1, 3)
    got = cD.unpack()
    pC, pD = pm(bf, "d", big), pm(bf, "d", D0)
    ppiv = bf.blasfeo_dgetrf_rp(m, n, pC, 2, 1, pD, 1, 3)
    assert np.array_equal(piv, ppiv)
    assert np.array_equal(got[1:1 + m, 3:3 + n], pD.unpack()[1:1 + m, 3:3 + n])
    hC, hD = host("d", big), host("d", D0)
    hpiv = orc.getrf_rp("d", m, n, hC, 2, 1, hD, 1, 3)
    assert np.array_equal(piv, hpiv)
    assert relfro(got, hD.get()) <= 1e-13
    assert outside_unchanged(got, D0, 1, 3, m, n)
