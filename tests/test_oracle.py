"""CPU tests of the oracle: pinned against the golden fixtures generated from
the compiled reference (tests/golden/make_golden.py) and, where the compiled
reference is present (oracle/_ref), against the reference itself on random
inputs with row/column offsets (the sweep structure of the reference's
tests/test_x.c)."""
import hashlib
import json
import os

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, spd

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
NP = {"d": np.float64, "s": np.float32}
TOL = {"d": 1e-13, "s": 2e-6}


@pytest.fixture(scope="module")
def orc():
    return oracle_api()


def gold(name):
    return np.load(os.path.join(GOLD, name))


def host(m, n, prec="d", data=None):
    from oracle.pyoracle import HostMat
    h = HostMat(m, n, NP[prec])
    if data is not None:
        h.set(data)
    return h


def test_manifest_hashes():
    man = json.load(open(os.path.join(GOLD, "manifest.json")))
    for name, sha in man["files"].items():
        assert hashlib.sha256(open(os.path.join(GOLD, name), "rb").read()).hexdigest() == sha, name


@pytest.mark.parametrize("prec", ["d", "s"])
def test_oracle_vs_golden_testx(orc, prec):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import run_testx
    g = gold("testx_%s.npz" % prec)
    out = run_testx(orc, prec)
    for k in g.files:
        if k.endswith("ipiv"):
            assert np.array_equal(out[k], g[k]), k
        else:
            assert relfro(out[k], g[k]) <= TOL[prec] * (10 if prec == "d" else 100), (k, relfro(out[k], g[k]))


def test_oracle_vs_golden_cfg1(orc):
    g = gold("cfg1.npz")
    n = 64
    hA, hB, hC, hD = host(n, n, data=g["A"]), host(n, n, data=g["B"]), host(n, n), host(n, n)
    orc.gemm_nt("d", n, n, n, 1.0, hA, 0, 0, hB, 0, 0, 0.0, hC, 0, 0, hD, 0, 0)
    assert relfro(hD.get(), g["D"]) <= 1e-13
    hS, hL = host(n, n, data=g["S"]), host(n, n)
    orc.potrf_l("d", n, hS, 0, 0, hL, 0, 0)
    assert relfro(np.tril(hL.get()), g["L"]) <= 1e-13
    assert relfro(hL.diag(n), g["L_dA"]) <= 1e-13
    hR, hX = host(n, n, data=g["R"]), host(n, n)
    orc.trsm_rltn("d", n, n, 1.0, hL, 0, 0, hR, 0, 0, hX, 0, 0)
    assert relfro(hX.get(), g["X"]) <= 1e-13


def test_oracle_vs_golden_cfg3(orc):
    from oracle.pyoracle import HostVec
    g = gold("cfg3.npz")
    for i, n in enumerate(g["ns"]):
        n = int(n)
        hA, hL = host(n, n, data=g["A%d" % i]), host(n, n)
        orc.potrf_l("d", n, hA, 0, 0, hL, 0, 0)
        assert relfro(np.tril(hL.get()), g["L%d" % i]) <= 1e-13
        hb, hy, hx = HostVec(n).set(g["b%d" % i]), HostVec(n), HostVec(n)
        orc.trsv_lnn("d", n, hL, 0, 0, hb, 0, hy, 0)
        orc.trsv_ltn("d", n, hL, 0, 0, hy, 0, hx, 0)
        # cond up to 1e6: solutions of two FP64 solvers agree to ~cond*eps
        assert relfro(hx.get(), g["x%d" % i]) <= 1e-9


def test_oracle_vs_golden_cfg4(orc):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import riccati_ref
    g = gold("cfg4.npz")
    for p in range(2):
        Ls = riccati_ref(orc, g["A%d" % p], g["B%d" % p])
        for k, L in enumerate(Ls):
            ref = g["L%d" % p][k][: L.shape[0], : L.shape[1]]
            assert relfro(L, ref) <= 1e-13, (p, k)


def test_oracle_vs_golden_cfg5(orc):
    g = gold("cfg5.npz")
    for i, n in enumerate([5, 11, 27, 64]):
        hM, hD = host(n, n, data=g["lu_in%d" % i]), host(n, n)
        piv = orc.getrf_rp("d", n, n, hM, 0, 0, hD, 0, 0)
        assert np.array_equal(piv, g["lu_ipiv%d" % i])
        assert relfro(hD.get(), g["lu%d" % i]) <= 1e-13
    for i, n in enumerate([3, 8, 21, 40]):
        hM, hD = host(2 * n, n, data=g["qr_in%d" % i]), host(2 * n, n)
        orc.geqrf("d", 2 * n, n, hM, 0, 0, hD, 0, 0)
        assert relfro(hD.get(), g["qr%d" % i]) <= 1e-13
        assert relfro(hD.diag(n), g["qr_tau%d" % i]) <= 1e-13


def test_oracle_vs_golden_cfg2(orc):
    g = gold("cfg2.npz")
    m, k = 16, 32
    for b in range(g["A"].shape[0]):
        hA, hS = host(m, k, data=g["A"][b]), host(m, m)
        orc.syrk_ln("d", m, k, 1.0, hA, 0, 0, hA, 0, 0, 0.0, hS, 0, 0, hS, 0, 0)
        import ctypes as C
        orc.lib.oracle_d_diare(m, C.c_double(16.0), hS.ref, 0, 0)
        hL = host(m, m)
        orc.potrf_l("d", m, hS, 0, 0, hL, 0, 0)
        hR, hX = host(m, m, data=g["R"][b]), host(m, m)
        orc.trsm_rltn("d", m, m, 1.0, hL, 0, 0, hR, 0, 0, hX, 0, 0)
        hC, hG, hD = host(m, m, data=g["C"][b]), host(m, m, data=g["G"][b]), host(m, m)
        orc.gemm_nt("d", m, m, m, -1.0, hX, 0, 0, hG, 0, 0, 1.0, hC, 0, 0, hD, 0, 0)
        assert relfro(np.tril(hL.get()), g["L"][b]) <= 1e-13
        assert relfro(hD.get(), g["D"][b]) <= 1e-13


# ---- against the compiled reference itself (when built here) ----

def _ref_or_skip(target="generic"):
    from oracle.pyoracle import Api, ref_available
    if not ref_available(target):
        pytest.skip("compiled reference not built (make -C oracle generic)")
    return Api("hp", target), Api("ref", target)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("case", [(7, 5, 3, 1, 2, 3, 0), (16, 16, 16, 0, 0, 0, 0), (33, 19, 40, 2, 1, 0, 3)])
def test_oracle_vs_reference_gemm_offsets(orc, prec, case):
    hp, _ = _ref_or_skip()
    m, n, k, ai, bi, ci, di = case
    rng = np.random.default_rng(m + n + k)
    A, B = rng.standard_normal((m + ai, k + 2)), rng.standard_normal((n + bi, k + 2))
    Cm, D0 = rng.standard_normal((m + ci, n + 1)), rng.standard_normal((m + di, n + 1))
    outs = []
    for api in (orc, hp):
        hA, hB, hC, hD = host(m + ai, k + 2, prec, A), host(n + bi, k + 2, prec, B), host(m + ci, n + 1, prec, Cm), host(m + di, n + 1, prec, D0)
        api.gemm_nt(prec, m, n, k, -0.75, hA, ai, 2, hB, bi, 1, 1.25, hC, ci, 1, hD, di, 0)
        outs.append(hD.get())
    assert relfro(outs[0], outs[1]) <= TOL[prec] * 10


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", [1, 3, 4, 9, 21, 60])
def test_oracle_vs_reference_factorizations(orc, prec, n):
    hp, ref = _ref_or_skip()
    rng = np.random.default_rng(n)
    g = rng.standard_normal((n, n))
    S = g @ g.T + n * np.eye(n)
    M = rng.standard_normal((n, n))
    T = rng.standard_normal((2 * n, n))
    res = {}
    for name, api in (("o", orc), ("hp", hp), ("ref", ref)):
        hS, hL = host(n, n, prec, S), host(n, n, prec)
        api.potrf_l(prec, n, hS, 0, 0, hL, 0, 0)
        hX, hY = host(n + 2, n, prec, rng.standard_normal((n + 2, n)) if name == "o" else res["o"]["X"]), host(n + 2, n, prec)
        api.trsm_rltn(prec, n + 2, n, 1.0, hL, 0, 0, hX, 0, 0, hY, 0, 0)
        hM, hLU = host(n, n, prec, M), host(n, n, prec)
        piv = api.getrf_rp(prec, n, n, hM, 0, 0, hLU, 0, 0)
        hT, hQ = host(2 * n, n, prec, T), host(2 * n, n, prec)
        api.geqrf(prec, 2 * n, n, hT, 0, 0, hQ, 0, 0)
        res[name] = {"L": np.tril(hL.get()), "X": hX.get(), "Y": hY.get(), "LU": hLU.get(), "piv": piv,
                     "QR": hQ.get(), "tau": hQ.diag(n)}
    for other in ("hp", "ref"):
        for k in ("L", "Y", "LU", "QR", "tau"):
            assert relfro(res["o"][k], res[other][k]) <= TOL[prec] * 100, (other, k)
        assert np.array_equal(res["o"]["piv"], res[other]["piv"])


def test_memsize_matches_reference_layout():
    from oracle.pyoracle import oracle_lib
    import ctypes as C
    lib = oracle_lib()
    lib.oracle_d_memsize_mat.restype = C.c_size_t
    for m, n in [(64, 64), (16, 16), (16, 32), (5, 3), (1, 1), (257, 13)]:
        pm, cn = (m + 3) // 4 * 4, (n + 3) // 4 * 4
        dl = (min(m, n) + 15) // 16 * 16
        want = ((pm * cn + dl) * 8 + 63) // 64 * 64
        assert lib.oracle_d_memsize_mat(m, n) == want
    # the figures quoted for the configurations: 64x64 -> 33,280 B, 16x16 -> 2,176 B, 16x32 -> 4,224 B
    assert lib.oracle_d_memsize_mat(64, 64) == 33280
    assert lib.oracle_d_memsize_mat(16, 16) == 2176
    assert lib.oracle_d_memsize_mat(16, 32) == 4224


# ---- the adjacent variants: syrk_ln_mn, trsm_rltu, potrf_l_mn, getrf_np ----

def adjacent_oracle(orc, prec, g):
    """The oracle on the inputs stored in the golden fixture (zero offsets)."""
    out = {}
    m, n, k = g[prec + "_syrkmn_A"].shape[0], g[prec + "_syrkmn_B"].shape[0], g[prec + "_syrkmn_A"].shape[1]
    hA, hB, hC, hD = (host(m, k, prec, g[prec + "_syrkmn_A"]), host(n, k, prec, g[prec + "_syrkmn_B"]),
                      host(m, n, prec, g[prec + "_syrkmn_C"]), host(m, n, prec))
    orc.syrk_ln_mn(prec, m, n, k, 0.5, hA, 0, 0, hB, 0, 0, -1.5, hC, 0, 0, hD, 0, 0)
    out["syrkmn_D"] = hD.get()
    hL, hX, hY = host(n, n, prec, g[prec + "_trsmu_L"]), host(m, n, prec, g[prec + "_trsmu_X"]), host(m, n, prec)
    orc.trsm_rltu(prec, m, n, 1.25, hL, 0, 0, hX, 0, 0, hY, 0, 0)
    out["trsmu_Y"] = hY.get()
    hS, hP = host(m, m, prec, g[prec + "_potrfmn_S"]), host(m, m, prec)
    orc.potrf_l_mn(prec, m, n, hS, 0, 0, hP, 0, 0)
    out["potrfmn_L"], out["potrfmn_dA"] = hP.get(), hP.diag(n)
    for tag in ("sq", "rect"):
        M = g[prec + "_lunp_%s_in" % tag]
        r, c = M.shape
        hM, hLU = host(r, c, prec, M), host(r, c, prec)
        orc.getrf_np(prec, r, c, hM, 0, 0, hLU, 0, 0)
        out["lunp_%s" % tag], out["lunp_%s_dA" % tag] = hLU.get(), hLU.diag(min(r, c))
    return out


@pytest.mark.parametrize("prec", ["d", "s"])
def test_oracle_vs_golden_adjacent(orc, prec):
    g = gold("adjacent.npz")
    out = adjacent_oracle(orc, prec, g)
    for key, v in out.items():
        assert relfro(v, g[prec + "_" + key]) <= TOL[prec] * 10, (key, relfro(v, g[prec + "_" + key]))


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("off", [(0, 0, 0), (1, 2, 3), (3, 0, 1)])
def test_oracle_vs_reference_adjacent_offsets(orc, prec, off):
    # the reference backend (blasfeo_ref_*) takes every offset; the HP routines
    # leave non-zero row offsets to it
    _, ref = _ref_or_skip()
    oi, oj, od = off
    rng = np.random.default_rng(17 + oi + oj + od)
    m, n, k = 19, 10, 7
    A, B, Cm = rng.standard_normal((m + oi, k + oj)), rng.standard_normal((n + oi, k + oj)), rng.standard_normal((m + oi, n + oj))
    Lu = np.tril(rng.standard_normal((n + oi, n + oj)), -1) * 0.4 + 5 * np.eye(n + oi, n + oj)
    X = rng.standard_normal((m + oi, n + oj))
    g = rng.standard_normal((m + oi, m + oi))
    S = g @ g.T + (m + oi) * np.eye(m + oi)
    M = rng.standard_normal((m + oi, n + oj)) + 6 * np.eye(m + oi, n + oj)
    res = []
    for api in (orc, ref):
        r = {}
        hA, hB, hC, hD = (host(m + oi, k + oj, prec, A), host(n + oi, k + oj, prec, B),
                          host(m + oi, n + oj, prec, Cm), host(m + od, n + od, prec))
        api.syrk_ln_mn(prec, m, n, k, 1.0, hA, oi, oj, hB, oi, oj, 0.5, hC, oi, oj, hD, od, od)
        r["syrk"] = hD.get()
        hL, hX, hY = host(n + oi, n + oj, prec, Lu), host(m + oi, n + oj, prec, X), host(m + od, n + od, prec)
        api.trsm_rltu(prec, m, n, -0.5, hL, oi, oj, hX, oi, oj, hY, od, od)
        r["trsm"] = hY.get()
        hS, hP = host(m + oi, m + oi, prec, S), host(m + od, m + od, prec)
        api.potrf_l_mn(prec, m, n, hS, oi, oi, hP, od, od)
        r["potrf"] = hP.get()
        hM, hLU = host(m + oi, n + oj, prec, M), host(m + od, n + od, prec)
        api.getrf_np(prec, m, n, hM, oi, oj, hLU, od, od)
        r["getrf"] = hLU.get()
        res.append(r)
    for key in res[0]:
        assert relfro(res[0][key], res[1][key]) <= TOL[prec] * 100, (key, relfro(res[0][key], res[1][key]))


@pytest.mark.parametrize("shape", [(5, 7, 1, 2), (12, 3, 0, 0), (1, 9, 3, 1), (9, 1, 2, 0)])
def test_reference_pack_tran_semantics(shape):
    # pins the layout rule the device converters implement, on the compiled
    # reference itself: pack_tran puts A^T (A m x n, column-major) into the
    # n x m block at (ai, aj); unpack_tran writes the block's transpose
    import ctypes as C
    from oracle.pyoracle import HostMat, ref_available, ref_lib
    if not ref_available("generic"):
        pytest.skip("compiled reference not built (make -C oracle generic)")
    lib = ref_lib("generic")
    m, n, ai, aj = shape
    rng = np.random.default_rng(m * 10 + n)
    A = np.asfortranarray(rng.standard_normal((m, n)))
    h = HostMat(n + ai + 1, m + aj + 2)
    base = rng.standard_normal((n + ai + 1, m + aj + 2))
    h.set(base)
    lib.blasfeo_pack_tran_dmat(m, n, A.ctypes.data_as(C.c_void_p), m, h.ref, ai, aj)
    want = base.copy()
    want[ai:ai + n, aj:aj + m] = A.T
    assert np.array_equal(h.get(), want)
    # unpack_tran of an m x n block at (ai, aj) where it fits: n x m result
    if ai + m <= h.m and aj + n <= h.n:
        out = np.asfortranarray(np.zeros((n, m)))
        lib.blasfeo_unpack_tran_dmat(m, n, h.ref, ai, aj, out.ctypes.data_as(C.c_void_p), n)
        assert np.array_equal(out, h.get()[ai:ai + m, aj:aj + n].T)


# ---- the reference's column-major routines vs the panel-major oracle ----
# The column-major drop-in stages each block into panel-major storage, runs the
# panel-major routine and writes back the block (or the lower triangle for
# syrk_ln / potrf_l).  These tests pin that equivalence on the reference's own
# column-major code (blasfeo_hp_cm/, GENERIC build): same numbers as the
# panel-major restatement on the same blocks, and nothing written outside.

def _cm_ref():
    from oracle.pyoracle import ref_cm_available, ref_cm_lib
    if not ref_cm_available():
        pytest.skip("column-major reference not built (make -C oracle cm)")
    lib = ref_cm_lib()
    return lib


def _outside_same(got, before, r0, c0, m, n, lower=False):
    mask = np.ones(got.shape, dtype=bool)
    blk = np.tril(np.ones((m, n), dtype=bool)) if lower else np.ones((m, n), dtype=bool)
    mask[r0:r0 + m, c0:c0 + n] &= ~blk
    return np.array_equal(got[mask], before[mask])


CM_NP = {"d": np.float64, "s": np.float32}
CM_TOL = {"d": 1e-13, "s": 2e-5}


def _cm_real(prec, v):
    import ctypes as C
    return C.c_double(v) if prec == "d" else C.c_float(v)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("case", [(17, 13, 9, 1, 2, 3, 1), (64, 64, 64, 0, 0, 0, 0), (5, 3, 7, 2, 0, 1, 4)])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (1.5, -0.5)])
def test_cm_reference_gemm_nt_is_panel_major_gemm_on_blocks(prec, case, ab):
    import ctypes as C
    from oracle.pyoracle import HostCmMat, HostMat
    lib = _cm_ref()
    orc = oracle_api()
    m, n, k, ai, bi, ci, di = case
    alpha, beta = ab
    rng = np.random.default_rng(m + 7 * n + k)
    t = CM_NP[prec]
    A = rng.uniform(-1, 1, (m + ai + 2, k + 3)).astype(t)
    B = rng.uniform(-1, 1, (n + bi + 1, k + 3)).astype(t)
    Cm = rng.uniform(-1, 1, (m + ci + 3, n + 2)).astype(t)
    D0 = rng.uniform(-1, 1, (m + di + 1, n + 4)).astype(t)
    cA, cB, cC, cD = HostCmMat(A, t), HostCmMat(B, t), HostCmMat(Cm, t), HostCmMat(D0, t)
    getattr(lib, "blasfeo_cm_%sgemm_nt" % prec)(m, n, k, _cm_real(prec, alpha), cA.ref, ai, 1, cB.ref, bi, 2,
                                                _cm_real(prec, beta), cC.ref, ci, 1, cD.ref, di, 3)
    H = lambda M: HostMat(*M.shape, dtype=t).set(M)
    pD = H(D0)
    orc.gemm_nt(prec, m, n, k, alpha, H(A), ai, 1, H(B), bi, 2, beta, H(Cm), ci, 1, pD, di, 3)
    assert relfro(cD.a, pD.get()) <= CM_TOL[prec]
    assert _outside_same(cD.a, D0, di, 3, m, n)


@pytest.mark.parametrize("mk", [(16, 32, 0), (13, 7, 1)])
def test_cm_reference_syrk_ln_writes_lower_block(mk):
    import ctypes as C
    from oracle.pyoracle import HostCmMat, HostMat
    lib = _cm_ref()
    orc = oracle_api()
    m, k, off = mk
    rng = np.random.default_rng(m + 100 * k)
    A = rng.standard_normal((m + off + 1, k))
    Cm = rng.standard_normal((m + off, m + off))
    D0 = rng.standard_normal((m + off + 2, m + off + 1))
    cA, cC, cD = HostCmMat(A), HostCmMat(Cm), HostCmMat(D0)
    lib.blasfeo_cm_dsyrk_ln(m, k, C.c_double(0.7), cA.ref, off, 0, cA.ref, off + 1, 0, C.c_double(1.3), cC.ref, off,
                            off, cD.ref, off + 1, off)
    hA, pD = HostMat(*A.shape).set(A), HostMat(*D0.shape).set(D0)
    orc.syrk_ln("d", m, k, 0.7, hA, off, 0, hA, off + 1, 0, 1.3, HostMat(*Cm.shape).set(Cm), off, off, pD, off + 1, off)
    assert relfro(cD.a, pD.get()) <= 1e-13
    assert _outside_same(cD.a, D0, off + 1, off, m, m, lower=True)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mn", [(13, 21), (40, 7), (64, 64)])
def test_cm_reference_trsm_rltn_is_panel_major_trsm(prec, mn):
    import ctypes as C
    from oracle.pyoracle import HostCmMat, HostMat
    lib = _cm_ref()
    orc = oracle_api()
    m, n = mn
    rng = np.random.default_rng(m * 3 + n)
    t = CM_NP[prec]
    Abig = rng.standard_normal((n + 2, n + 1))
    Abig[2:2 + n, 1:1 + n] = np.linalg.cholesky(spd(rng, n))
    Abig = Abig.astype(t)
    B = rng.standard_normal((m + 1, n + 3)).astype(t)
    D0 = rng.standard_normal((m + 3, n + 2)).astype(t)
    cA, cB, cD = HostCmMat(Abig, t), HostCmMat(B, t), HostCmMat(D0, t)
    getattr(lib, "blasfeo_cm_%strsm_rltn" % prec)(m, n, _cm_real(prec, 1.0), cA.ref, 2, 1, cB.ref, 1, 3, cD.ref, 3, 2)
    H = lambda M: HostMat(*M.shape, dtype=t).set(M)
    pD = H(D0)
    orc.trsm_rltn(prec, m, n, 1.0, H(Abig), 2, 1, H(B), 1, 3, pD, 3, 2)
    assert relfro(cD.a, pD.get()) <= CM_TOL[prec] * 10
    assert _outside_same(cD.a, D0, 3, 2, m, n)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", [1, 5, 16, 33, 64])
def test_cm_reference_potrf_l_writes_lower_block_only(prec, n):
    from oracle.pyoracle import HostCmMat, HostMat
    lib = _cm_ref()
    orc = oracle_api()
    rng = np.random.default_rng(n + 7)
    t = CM_NP[prec]
    big = rng.standard_normal((n + 3, n + 2))
    big[1:1 + n, 2:2 + n] = spd(rng, n)
    big = big.astype(t)
    D0 = rng.standard_normal((n + 2, n + 4)).astype(t)
    cC, cD = HostCmMat(big, t), HostCmMat(D0, t)
    getattr(lib, "blasfeo_cm_%spotrf_l" % prec)(n, cC.ref, 1, 2, cD.ref, 2, 1)
    H = lambda M: HostMat(*M.shape, dtype=t).set(M)
    pD = H(D0)
    orc.potrf_l(prec, n, H(big), 1, 2, pD, 2, 1)
    got, want = np.tril(cD.a[2:2 + n, 1:1 + n]), np.tril(pD.get()[2:2 + n, 1:1 + n])
    assert relfro(got, want) <= CM_TOL[prec]
    assert _outside_same(cD.a, D0, 2, 1, n, n, lower=True)
    assert cD.desc.use_dA == 0


@pytest.mark.parametrize("mn", [(37, 20), (20, 37), (64, 64)])
def test_cm_reference_getrf_rp_pivots_match(mn):
    import ctypes as C
    from oracle.pyoracle import HostCmMat, HostMat
    lib = _cm_ref()
    orc = oracle_api()
    m, n = mn
    rng = np.random.default_rng(m + 3 * n)
    big = rng.standard_normal((m + 2, n + 1))
    D0 = rng.standard_normal((m + 1, n + 3))
    cC, cD = HostCmMat(big), HostCmMat(D0)
    piv = np.zeros(min(m, n) + 8, dtype=np.int32)
    lib.blasfeo_cm_dgetrf_rp(m, n, cC.ref, 2, 1, cD.ref, 1, 3, piv.ctypes.data_as(C.POINTER(C.c_int)))
    pD = HostMat(*D0.shape).set(D0)
    ppiv = orc.getrf_rp("d", m, n, HostMat(*big.shape).set(big), 2, 1, pD, 1, 3)
    assert np.array_equal(piv[:min(m, n)], ppiv)
    assert relfro(cD.a, pD.get()) <= 1e-12
    assert _outside_same(cD.a, D0, 1, 3, m, n)


def test_riccati_solve_oracle_vs_golden_and_kkt():
    """The oracle's Riccati factorization + solve (tests/ric_oracle.py composing
    the oracle routines) reproduces the compiled reference's outputs of
    d_back_ric_trs_libstr (golden cfg4_trs.npz) and solves the LQ problem's KKT
    system."""
    from tests.ric_oracle import ric_trf, ric_trs, kkt_residual
    g = np.load(os.path.join(GOLD, "cfg4_trs.npz"))
    orc = oracle_api()
    N, nx, nu = 30, 12, 4
    RSQ = np.broadcast_to(np.eye(16), (N + 1, 16, 16)).copy()
    for p in range(2):
        BA, b, rq = g["BA%d" % p], g["b%d" % p], g["rq%d" % p]
        L = ric_trf(orc, BA, RSQ, N, nx, nu)
        ux, pi = ric_trs(orc, L, BA, b, rq, N, nx, nu)
        for k in range(N + 1):
            assert relfro(ux[k], g["ux%d" % p][k][:len(ux[k])]) <= 1e-14, (p, k)
        assert relfro(np.stack(pi), g["pi%d" % p]) <= 1e-14
        rs, rd = kkt_residual(BA, RSQ, b, rq, ux, pi, N, nx, nu)
        assert max(np.abs(r).max() for r in rs + rd) <= 1e-12
