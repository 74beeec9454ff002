"""GPU parity of the batched entry points (uniform *_batch and variable-size
*_vbatch) and of the fused factor+solve kernels, against the CPU oracle run
instance by instance on the same seeded inputs."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro, spd, tol

pytestmark = pytest.mark.gpu
NP = {"d": np.float64, "s": np.float32}
TOL = {"d": 1e-13, "s": 2e-5}


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


def sync():
    import torch
    torch.cuda.synchronize()


def batch_of(bf, prec, arr):
    b, m, n = arr.shape
    B = (bf.DMatBatch if prec == "d" else bf.SMatBatch)(m, n, b)
    return B.pack_all(arr)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", [4, 16, 23, 53, 64, 96, 150])
def test_potrf_batch(bf, orc, prec, n):
    import torch
    rng = np.random.default_rng(n)
    nb = 37
    S = np.stack([spd(rng, n) for _ in range(nb)])
    dC = batch_of(bf, prec, S)
    dD = batch_of(bf, prec, np.zeros_like(S))
    info = torch.full((nb,), -7, dtype=torch.int32, device="cuda")
    st = getattr(bf.lib, "blasfeo_%spotrf_l_batch" % prec)(nb, n, dC.ref, 0, 0, dD.ref, 0, 0,
                                                         C.c_void_p(info.data_ptr()), None)
    assert st == 0
    sync()
    got = dD.unpack_all()
    dg = dD.diag_all(n)
    assert (info.cpu().numpy() == 0).all()
    for b in range(0, nb, 6):
        hC, hD = host(n, n, prec, S[b]), host(n, n, prec)
        orc.potrf_l(prec, n, hC, 0, 0, hD, 0, 0)
        assert relfro(got[b], hD.get()) <= TOL[prec]
        assert relfro(dg[b], hD.diag(n)) <= tol(prec, 10)


@pytest.mark.parametrize("prec", ["d", "s"])
def test_potrf_batch_info(bf, prec):
    import torch
    rng = np.random.default_rng(1)
    n, nb = 12, 5
    S = np.stack([spd(rng, n) for _ in range(nb)])
    S[2, 7, 7] = -5.0
    dC, dD = batch_of(bf, prec, S), batch_of(bf, prec, np.zeros_like(S))
    info = torch.zeros(nb, dtype=torch.int32, device="cuda")
    getattr(bf.lib, "blasfeo_%spotrf_l_batch" % prec)(nb, n, dC.ref, 0, 0, dD.ref, 0, 0, C.c_void_p(info.data_ptr()), None)
    sync()
    inf = info.cpu().numpy()
    assert inf[2] == 8 and (np.delete(inf, 2) == 0).all()


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("mnk", [(16, 16, 16), (5, 9, 3), (64, 48, 33)])
def test_gemm_syrk_trsm_batch(bf, orc, prec, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m + n + k)
    nb = 11
    A = rng.standard_normal((nb, m, k))
    B = rng.standard_normal((nb, n, k))
    Cm = rng.standard_normal((nb, m, n))
    dA, dB, dC, dD = (batch_of(bf, prec, A), batch_of(bf, prec, B), batch_of(bf, prec, Cm),
                      batch_of(bf, prec, np.zeros((nb, m, n))))
    st = getattr(bf.lib, "blasfeo_%sgemm_nt_batch" % prec)(nb, m, n, k, 1.25, dA.ref, 0, 0, dB.ref, 0, 0, -0.5,
                                                          dC.ref, 0, 0, dD.ref, 0, 0, None)
    assert st == 0
    sync()
    got = dD.unpack_all()
    for b in (0, nb // 2, nb - 1):
        hA, hB, hC, hD = host(m, k, prec, A[b]), host(n, k, prec, B[b]), host(m, n, prec, Cm[b]), host(m, n, prec)
        orc.gemm_nt(prec, m, n, k, 1.25, hA, 0, 0, hB, 0, 0, -0.5, hC, 0, 0, hD, 0, 0)
        assert relfro(got[b], hD.get()) <= TOL[prec]
    # syrk on A (m x k): D = A A^T lower
    Cs = rng.standard_normal((nb, m, m))
    dCs, dDs = batch_of(bf, prec, Cs), batch_of(bf, prec, np.zeros((nb, m, m)))
    getattr(bf.lib, "blasfeo_%ssyrk_ln_batch" % prec)(nb, m, k, 1.0, dA.ref, 0, 0, dA.ref, 0, 0, 1.0, dCs.ref, 0, 0,
                                                      dDs.ref, 0, 0, None)
    sync()
    gs = dDs.unpack_all()
    for b in (0, nb - 1):
        hA, hC, hD = host(m, k, prec, A[b]), host(m, m, prec, Cs[b]), host(m, m, prec)
        orc.syrk_ln(prec, m, k, 1.0, hA, 0, 0, hA, 0, 0, 1.0, hC, 0, 0, hD, 0, 0)
        assert relfro(np.tril(gs[b]), np.tril(hD.get())) <= TOL[prec]
    # trsm with a batch of factors
    S = np.stack([spd(rng, n) for _ in range(nb)])
    X = rng.standard_normal((nb, m, n))
    dS, dL = batch_of(bf, prec, S), batch_of(bf, prec, np.zeros_like(S))
    getattr(bf.lib, "blasfeo_%spotrf_l_batch" % prec)(nb, n, dS.ref, 0, 0, dL.ref, 0, 0, None, None)
    dX, dY = batch_of(bf, prec, X), batch_of(bf, prec, np.zeros_like(X))
    getattr(bf.lib, "blasfeo_%strsm_rltn_batch" % prec)(nb, m, n, 1.0, dL.ref, 0, 0, dX.ref, 0, 0, dY.ref, 0, 0, None)
    sync()
    gy = dY.unpack_all()
    for b in (0, nb - 1):
        hS, hL = host(n, n, prec, S[b]), host(n, n, prec)
        orc.potrf_l(prec, n, hS, 0, 0, hL, 0, 0)
        hX, hY = host(m, n, prec, X[b]), host(m, n, prec)
        orc.trsm_rltn(prec, m, n, 1.0, hL, 0, 0, hX, 0, 0, hY, 0, 0)
        assert relfro(gy[b], hY.get()) <= tol(prec, 10)


@pytest.mark.parametrize("prec", ["d", "s"])
def test_getrf_geqrf_batch(bf, orc, prec):
    import torch
    rng = np.random.default_rng(21)
    nb, m, n = 9, 24, 24
    M = rng.standard_normal((nb, m, n))
    dC, dD = batch_of(bf, prec, M), batch_of(bf, prec, np.zeros_like(M))
    piv = torch.zeros(nb * n, dtype=torch.int32, device="cuda")
    getattr(bf.lib, "blasfeo_%sgetrf_rp_batch" % prec)(nb, m, n, dC.ref, 0, 0, dD.ref, 0, 0, C.c_void_p(piv.data_ptr()),
                                                       None, None)
    sync()
    got, gp = dD.unpack_all(), piv.cpu().numpy().reshape(nb, n)
    for b in range(nb):
        hC, hD = host(m, n, prec, M[b]), host(m, n, prec)
        pr = orc.getrf_rp(prec, m, n, hC, 0, 0, hD, 0, 0)
        assert np.array_equal(gp[b], pr)
        assert relfro(got[b], hD.get()) <= tol(prec, 100)
    Q = rng.standard_normal((nb, 2 * n, n))
    dQ, dR = batch_of(bf, prec, Q), batch_of(bf, prec, np.zeros_like(Q))
    getattr(bf.lib, "blasfeo_%sgeqrf_batch" % prec)(nb, 2 * n, n, dQ.ref, 0, 0, dR.ref, 0, 0, None)
    sync()
    gr, gt = dR.unpack_all(), dR.diag_all(n)
    for b in range(nb):
        hC, hD = host(2 * n, n, prec, Q[b]), host(2 * n, n, prec)
        orc.geqrf(prec, 2 * n, n, hC, 0, 0, hD, 0, 0)
        assert relfro(gr[b], hD.get()) <= tol(prec, 50)
        assert relfro(gt[b], hD.diag(n)) <= tol(prec, 50)


def _vb_setup(bf, mats):
    return bf.descriptor_array(mats)


def test_vbatch_potrf_gemm_getrf_geqrf(bf, orc):
    import torch
    rng = np.random.default_rng(33)
    ns = [4, 17, 64, 5, 100, 33, 250, 1]
    nb = len(ns)
    S = [spd(rng, n) for n in ns]
    Cs = [bf.DMat(n, n).pack(s) for n, s in zip(ns, S)]
    Ds = [bf.DMat(n, n) for n in ns]
    dC, dD = _vb_setup(bf, Cs), _vb_setup(bf, Ds)
    nv = torch.tensor(ns, dtype=torch.int32, device="cuda")
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dpotrf_l_vbatch(nb, C.c_void_p(nv.data_ptr()), max(ns), C.c_void_p(dC.data_ptr()),
                                        C.c_void_p(dD.data_ptr()), C.c_void_p(info.data_ptr()), None)
    assert st == 0
    sync()
    assert (info.cpu().numpy() == 0).all()
    for n, s, d in zip(ns, S, Ds):
        hC, hD = host(n, n, "d", s), host(n, n, "d")
        orc.potrf_l("d", n, hC, 0, 0, hD, 0, 0)
        assert relfro(np.tril(d.unpack()), np.tril(hD.get())) <= 1e-13
    # gemm vbatch with uneven m, n, k
    ms, nn, ks = [3, 40, 17, 64], [5, 20, 33, 64], [7, 1, 40, 64]
    As = [rng.standard_normal((m, k)) for m, k in zip(ms, ks)]
    Bs = [rng.standard_normal((n, k)) for n, k in zip(nn, ks)]
    dAs = [bf.DMat(m, k).pack(a) for m, k, a in zip(ms, ks, As)]
    dBs = [bf.DMat(n, k).pack(b) for n, k, b in zip(nn, ks, Bs)]
    dDs = [bf.DMat(m, n) for m, n in zip(ms, nn)]
    t = lambda v: torch.tensor(v, dtype=torch.int32, device="cuda")
    mv, nv2, kv = t(ms), t(nn), t(ks)
    aA, aB, aD = _vb_setup(bf, dAs), _vb_setup(bf, dBs), _vb_setup(bf, dDs)
    st = bf.lib.blasfeo_dgemm_nt_vbatch(4, C.c_void_p(mv.data_ptr()), C.c_void_p(nv2.data_ptr()),
                                        C.c_void_p(kv.data_ptr()), max(ms), max(nn), max(ks), 1.0,
                                        C.c_void_p(aA.data_ptr()), C.c_void_p(aB.data_ptr()), 0.0,
                                        C.c_void_p(aD.data_ptr()), C.c_void_p(aD.data_ptr()), None)
    assert st == 0
    sync()
    for a, b, d in zip(As, Bs, dDs):
        assert relfro(d.unpack(), a @ b.T) <= 1e-14
    # getrf / geqrf vbatch
    Ms = [rng.standard_normal((n, n)) for n in ns]
    Gc = [bf.DMat(n, n).pack(x) for n, x in zip(ns, Ms)]
    Gd = [bf.DMat(n, n) for n in ns]
    piv = torch.zeros(nb * max(ns), dtype=torch.int32, device="cuda")
    aC, aD2 = _vb_setup(bf, Gc), _vb_setup(bf, Gd)
    nv3 = t(ns)
    st = bf.lib.blasfeo_dgetrf_rp_vbatch(nb, C.c_void_p(nv3.data_ptr()), C.c_void_p(nv3.data_ptr()), max(ns), max(ns),
                                         C.c_void_p(aC.data_ptr()), C.c_void_p(aD2.data_ptr()),
                                         C.c_void_p(piv.data_ptr()), max(ns), None, None)
    assert st == 0
    sync()
    pv = piv.cpu().numpy().reshape(nb, max(ns))
    for i, (n, x, d) in enumerate(zip(ns, Ms, Gd)):
        hC, hD = host(n, n, "d", x), host(n, n, "d")
        pr = orc.getrf_rp("d", n, n, hC, 0, 0, hD, 0, 0)
        assert np.array_equal(pv[i, :n], pr)
        assert relfro(d.unpack(), hD.get()) <= 1e-13


def _posv_inputs(bf, rng, ns, cond=1e6):
    import torch
    As, bs, mats, bvecs, xvecs = [], [], [], [], []
    for n in ns:
        q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        lam = 10.0 ** rng.uniform(0, np.log10(cond), n)
        a = (q * lam) @ q.T
        a = 0.5 * (a + a.T)
        b = rng.standard_normal(n)
        As.append(a)
        bs.append(b)
        mats.append(bf.DMat(n, n).pack(a))
        bvecs.append(bf.DVec(n).pack(b))
        xvecs.append(bf.DVec(n))
    return As, bs, mats, bvecs, xvecs


@pytest.mark.parametrize("mixed", [False, True])
def test_posv_vbatch(bf, orc, mixed):
    import torch
    rng = np.random.default_rng(77)
    # every size class of both solvers, and its edges (n = 4k, 4k + 1, 16k, 16k + 1)
    ns = [4, 5, 16, 31, 64, 97, 128, 150, 190, 200, 233, 256, 1, 240, 17, 63, 65, 129, 176, 177, 224, 225, 255]
    As, bs, mats, bvecs, xvecs = _posv_inputs(bf, rng, ns)
    dA, db, dx = bf.descriptor_array(mats), bf.vector_array(bvecs), bf.vector_array(xvecs)
    nb = len(ns)
    nv = torch.tensor(ns, dtype=torch.int32, device="cuda")
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    iters = torch.zeros(nb, dtype=torch.int32, device="cuda")
    berr = torch.zeros(nb, dtype=torch.float64, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    if mixed:
        st = bf.lib.blasfeo_dsposv_l_vbatch(nb, P(nv), max(ns), P(dA), P(db), P(dx), 30, 1e-12, P(iters), P(berr),
                                            P(info), None, 0, None)
    else:
        st = bf.lib.blasfeo_dposv_l_vbatch(nb, P(nv), max(ns), P(dA), P(db), P(dx), P(info), None, 0, None)
    assert st == 0
    sync()
    inf = info.cpu().numpy()
    assert (inf == 0).all(), inf
    kb = berr.cpu().numpy()
    for i, (n, a, b, xv) in enumerate(zip(ns, As, bs, xvecs)):
        x = xv.unpack()
        r = b - a @ x
        be = np.abs(r).max() / (np.abs(a).sum(1).max() * np.abs(x).max())
        assert be <= 1e-12, (n, be)
        if mixed:
            # the solver's own FP64 residual (the stopping test) agrees with
            # the host's: same definition; the two summation orders differ by
            # at most n eps ||A|| ||x|| in each residual entry
            assert abs(kb[i] - be) <= 0.1 * be + n * 2.2e-16, (n, kb[i], be)
        if not mixed:
            # the factor path matches the oracle's dpotrf_l + dtrsv_lnn + dtrsv_ltn
            from oracle.pyoracle import HostVec
            hC, hL = host(n, n, "d", a), host(n, n, "d")
            orc.potrf_l("d", n, hC, 0, 0, hL, 0, 0)
            hb, hy, hx = HostVec(n).set(b), HostVec(n), HostVec(n)
            orc.trsv_lnn("d", n, hL, 0, 0, hb, 0, hy, 0)
            orc.trsv_ltn("d", n, hL, 0, 0, hy, 0, hx, 0)
            xr = hx.get()
            # two backward-stable solvers differ by ~cond*eps in x
            assert relfro(x, xr) <= 1e-6


@pytest.mark.parametrize("mixed", [False, True])
def test_posv_vbatch_caller_workspace(bf, mixed):
    # a caller-provided workspace of blasfeo_dposv_worksize_n bytes is enough
    # (plain systems above n = 128 take the blocked path with per-CTA factor
    # slots), one byte less is rejected before any device work
    import torch
    rng = np.random.default_rng(91)
    ns = [3, 100, 129, 200, 256, 57]
    As, bs, mats, bvecs, xvecs = _posv_inputs(bf, rng, ns)
    dA, db, dx = bf.descriptor_array(mats), bf.vector_array(bvecs), bf.vector_array(xvecs)
    nb = len(ns)
    nv = torch.tensor(ns, dtype=torch.int32, device="cuda")
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    need = bf.lib.blasfeo_dposv_worksize_n(nb, max(ns), 1 if mixed else 0)
    assert need >= bf.lib.blasfeo_dposv_worksize(nb)
    work = torch.zeros(need, dtype=torch.uint8, device="cuda")

    def call(nbytes):
        if mixed:
            return bf.lib.blasfeo_dsposv_l_vbatch(nb, P(nv), max(ns), P(dA), P(db), P(dx), 30, 1e-12, None, None,
                                                  P(info), P(work), nbytes, None)
        return bf.lib.blasfeo_dposv_l_vbatch(nb, P(nv), max(ns), P(dA), P(db), P(dx), P(info), P(work), nbytes, None)
    assert call(need - 1) == 3  # BLASFEO_B200_ENOMEM
    assert call(need) == 0
    sync()
    assert (info.cpu().numpy() == 0).all()
    for n, a, b, xv in zip(ns, As, bs, xvecs):
        x = xv.unpack()
        assert np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max()) <= 1e-12, n
