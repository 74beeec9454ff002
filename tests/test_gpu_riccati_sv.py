"""GPU parity of the batched Riccati solve (examples/example_d_riccati_recursion.c
d_back_ric_trs_libstr), the feedback gains and the mixed-precision LQ solve:
against the golden outputs of the compiled reference, the oracle on
time-varying problems, and the KKT residual of the LQ problem."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
P = lambda t: C.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    return blasfeo_b200


def problems(rng, nbt, N, nx, nu):
    m = nx + nu
    BA = np.zeros((nbt, N, 16, nx))
    RSQ = np.zeros((nbt, N + 1, 16, 16))
    b = np.zeros((nbt, N, 16))
    rq = np.zeros((nbt, N + 1, 16))
    for p in range(nbt):
        for k in range(N + 1):
            G = rng.standard_normal((m, m))
            RSQ[p, k, :m, :m] = G @ G.T / m + np.eye(m)
            rq[p, k, :m if k < N else nx] = rng.standard_normal(m if k < N else nx)
            if k < N:
                BA[p, k, :m] = rng.standard_normal((m, nx)) / np.sqrt(nx)
                b[p, k, :nx] = rng.standard_normal(nx)
    return BA, RSQ, b, rq


def device(bf, BA, RSQ, b, rq):
    import torch
    nbt, N, _, nx = BA.shape
    sBA = bf.DMatBatch(16, nx, nbt * N).pack_all(BA.reshape(nbt * N, 16, nx))
    sRSQ = bf.DMatBatch(16, 16, nbt * (N + 1)).pack_all(RSQ.reshape(nbt * (N + 1), 16, 16))
    db = torch.from_numpy(b.reshape(-1)).cuda()
    drq = torch.from_numpy(rq.reshape(-1)).cuda()
    ux = torch.zeros(nbt * (N + 1) * 16, dtype=torch.float64, device="cuda")
    pi = torch.zeros(nbt * N * 16, dtype=torch.float64, device="cuda")
    return sBA, sRSQ, db, drq, ux, pi


def factor_and_solve(bf, BA, RSQ, b, rq, nx, nu):
    import torch
    nbt, N = BA.shape[:2]
    sBA, sRSQ, db, drq, ux, pi = device(bf, BA, RSQ, b, rq)
    sL = bf.DMatBatch(16, 16, nbt * (N + 1))
    info = torch.full((nbt,), -9, dtype=torch.int32, device="cuda")
    assert bf.lib.blasfeo_dric_trf_batch(nbt, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, P(info), None) == 0
    assert bf.lib.blasfeo_dric_trs_batch(nbt, N, nx, nu, sBA.ref, sL.ref, P(db), 16, P(drq), 16, P(ux), 16, P(pi), 16,
                                         None) == 0
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    return sL, ux.cpu().numpy().reshape(nbt, N + 1, 16), pi.cpu().numpy().reshape(nbt, N, 16)


def test_trs_vs_golden_reference(bf):
    g = np.load(os.path.join(GOLD, "cfg4_trs.npz"))
    N, nx, nu = 30, 12, 4
    BA = np.stack([g["BA0"], g["BA1"]])
    RSQ = np.broadcast_to(np.eye(16), (2, N + 1, 16, 16)).copy()
    b, rq = np.stack([g["b0"], g["b1"]]), np.stack([g["rq0"], g["rq1"]])
    _, ux, pi = factor_and_solve(bf, BA, RSQ, b, rq, nx, nu)
    for p in range(2):
        assert relfro(ux[p], g["ux%d" % p]) <= 1e-13, p
        assert relfro(pi[p, :, :nx], g["pi%d" % p]) <= 1e-13, p


@pytest.mark.parametrize("dims", [(12, 4, 30), (8, 3, 7), (5, 0, 4), (13, 3, 1), (4, 4, 2)])
def test_trs_time_varying_vs_oracle_and_kkt(bf, dims):
    from tests.ric_oracle import ric_trf, ric_trs, kkt_residual
    nx, nu, N = dims
    rng = np.random.default_rng(nx * 100 + nu * 10 + N)
    nbt = 19
    BA, RSQ, b, rq = problems(rng, nbt, N, nx, nu)
    _, ux, pi = factor_and_solve(bf, BA, RSQ, b, rq, nx, nu)
    orc = oracle_api()
    m = nx + nu
    for p in (0, nbt // 2, nbt - 1):
        L = ric_trf(orc, BA[p], RSQ[p], N, nx, nu)
        uxr, pir = ric_trs(orc, L, BA[p], b[p], rq[p], N, nx, nu)
        for k in range(N + 1):
            mm = nx if k == N else m
            assert relfro(ux[p, k, :mm], uxr[k]) <= 1e-13, (p, k)
        assert relfro(pi[p, :, :nx], np.stack(pir)) <= 1e-13, p
        rs, rd = kkt_residual(BA[p], RSQ[p], b[p], rq[p], [ux[p, k] for k in range(N + 1)],
                              [pi[p, k, :nx] for k in range(N)], N, nx, nu)
        assert max(np.abs(r).max() for r in rs + rd) <= 1e-12


def test_gains(bf):
    import torch
    from tests.ric_oracle import ric_trf
    nx, nu, N = 12, 4, 6
    rng = np.random.default_rng(3)
    nbt = 9
    BA, RSQ, b, rq = problems(rng, nbt, N, nx, nu)
    sL, _, _ = factor_and_solve(bf, BA, RSQ, b, rq, nx, nu)
    sK = bf.DMatBatch(nu, nx, nbt * N)
    assert bf.lib.blasfeo_dric_gains_batch(nbt, N, nx, nu, sL.ref, sK.ref, None) == 0
    torch.cuda.synchronize()
    K = sK.unpack_all().reshape(nbt, N, nu, nx)
    orc = oracle_api()
    for p in (0, nbt - 1):
        L = ric_trf(orc, BA[p], RSQ[p], N, nx, nu)
        for k in range(N):
            Lk = np.tril(L[k].get())
            Kr = -np.linalg.solve(np.tril(Lk[:nu, :nu]).T, Lk[nu:, :nu].T)
            assert relfro(K[p, k], Kr) <= 1e-13, (p, k)
            # the gain is the minimiser of the stage's quadratic in u for fixed x
            Lkk = Lk @ Lk.T
            assert np.abs(Lkk[:nu, :nu] @ K[p, k] + Lkk[:nu, nu:]).max() <= 1e-12


@pytest.mark.parametrize("dims", [(12, 4, 30), (8, 3, 7)])
def test_mixed_lq_solve_reaches_fp64(bf, dims):
    """FP32 factorization + FP64 refinement: the KKT residual reaches the
    tolerance and the solution agrees with the FP64 solve to about cond * tol."""
    import torch
    from tests.ric_oracle import kkt_residual
    nx, nu, N = dims
    rng = np.random.default_rng(7 + N)
    nbt = 23
    BA, RSQ, b, rq = problems(rng, nbt, N, nx, nu)
    _, ux64, pi64 = factor_and_solve(bf, BA, RSQ, b, rq, nx, nu)
    sBA, sRSQ, db, drq, ux, pi = device(bf, BA, RSQ, b, rq)
    iters = torch.full((nbt,), -5, dtype=torch.int32, device="cuda")
    res = torch.zeros(nbt, dtype=torch.float64, device="cuda")
    info = torch.full((nbt,), -9, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dsric_sv_batch(nbt, N, nx, nu, sBA.ref, sRSQ.ref, P(db), 16, P(drq), 16, P(ux), 16, P(pi), 16,
                                       20, 1e-13, P(iters), P(res), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0
    assert (info.cpu().numpy() == 0).all() and (res.cpu().numpy() <= 1e-13).all()
    it = iters.cpu().numpy()
    assert (it >= 1).all() and (it <= 6).all(), it
    u, p_ = ux.cpu().numpy().reshape(nbt, N + 1, 16), pi.cpu().numpy().reshape(nbt, N, 16)
    assert relfro(u, ux64) <= 1e-11 and relfro(p_, pi64) <= 1e-11
    for q in (0, nbt - 1):
        rs, rd = kkt_residual(BA[q], RSQ[q], b[q], rq[q], [u[q, k] for k in range(N + 1)],
                              [p_[q, k, :nx] for k in range(N)], N, nx, nu)
        assert max(np.abs(r).max() for r in rs + rd) <= 1e-12
    # without refinement steps the FP32 factor alone stays far from the tolerance
    st = bf.lib.blasfeo_dsric_sv_batch(nbt, N, nx, nu, sBA.ref, sRSQ.ref, P(db), 16, P(drq), 16, P(ux), 16, P(pi), 16,
                                       0, 1e-13, P(iters), P(res), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0 and (info.cpu().numpy() == -1).all() and (iters.cpu().numpy() == 0).all()
    assert (res.cpu().numpy() > 1e-9).all()


def test_rejects_bad_arguments(bf):
    a = bf.dmat_batch()
    assert bf.lib.blasfeo_dric_trs_batch(1, 0, 4, 2, C.byref(a), C.byref(a), None, 16, None, 16, None, 16, None, 16,
                                         None) == 1
    assert bf.lib.blasfeo_dric_trs_batch(1, 3, 14, 4, C.byref(a), C.byref(a), None, 16, None, 16, None, 16, None, 16,
                                         None) == 4
