"""GPU parity of the batched Riccati factorization against the golden
fixtures of the compiled reference (examples/example_d_riccati_recursion.c
recursion) and against the oracle on time-varying problems."""
import os
import sys

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    return blasfeo_b200


def build(bf, prec, BAs, RSQs):
    """BAs: (batch, N, 16, nx); RSQs: (batch, N+1, 16, 16) -> device slabs."""
    nbt, N, m, nx = BAs.shape
    Bt = bf.DMatBatch if prec == "d" else bf.SMatBatch
    sBA = Bt(16, nx, nbt * N).pack_all(BAs.reshape(nbt * N, 16, nx))
    sRSQ = Bt(16, 16, nbt * (N + 1)).pack_all(RSQs.reshape(nbt * (N + 1), 16, 16))
    sL = Bt(16, 16, nbt * (N + 1))
    return sBA, sRSQ, sL


def run(bf, prec, BAs, RSQs, nx, nu):
    import ctypes as C
    import torch
    nbt, N = BAs.shape[:2]
    sBA, sRSQ, sL = build(bf, prec, BAs, RSQs)
    info = torch.full((nbt,), -9, dtype=torch.int32, device="cuda")
    f = bf.lib.blasfeo_dric_trf_batch if prec == "d" else bf.lib.blasfeo_sric_trf_batch
    st = f(nbt, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, C.c_void_p(info.data_ptr()), None)
    torch.cuda.synchronize()
    assert st == 0
    return sL.unpack_all().reshape(nbt, N + 1, 16, 16), info.cpu().numpy()


def problem_mats(A, B, N, nx, nu):
    BA = np.vstack([B.T, A.T])
    BA16 = np.zeros((16, nx))
    BA16[: nu + nx] = BA
    BAs = np.broadcast_to(BA16, (N, 16, nx)).copy()
    RSQ = np.eye(16)
    RSQs = np.broadcast_to(RSQ, (N + 1, 16, 16)).copy()
    return BAs, RSQs


def test_riccati_vs_golden_reference(bf):
    g = np.load(os.path.join(GOLD, "cfg4.npz"))
    N, nx, nu = 30, 12, 4
    BAs, RSQs = zip(*[problem_mats(g["A%d" % p], g["B%d" % p], N, nx, nu) for p in range(2)])
    L, info = run(bf, "d", np.stack(BAs), np.stack(RSQs), nx, nu)
    assert (info == 0).all()
    for p in range(2):
        for k in range(N + 1):
            m = nx if k == N else nx + nu
            assert relfro(np.tril(L[p, k, :m, :m]), g["L%d" % p][k][:m, :m]) <= 1e-13, (p, k)


def oracle_riccati(orc, BA, RSQ, N, nx, nu):
    """Time-varying recursion with the oracle's dtrmm_rlnn + dsyrk_dpotrf_ln."""
    from oracle.pyoracle import HostMat
    m = nu + nx
    Ls = [None] * (N + 1)
    hQ, hL = HostMat(nx, nx).set(RSQ[N][:nx, :nx]), HostMat(nx, nx)
    orc.potrf_l("d", nx, hQ, 0, 0, hL, 0, 0)
    Ls[N] = np.tril(hL.get())
    prev, off = hL, 0
    for k in range(N - 1, -1, -1):
        hBA, hW, hR, hLk = HostMat(m, nx).set(BA[k][:m]), HostMat(m, nx), HostMat(m, m).set(RSQ[k][:m, :m]), HostMat(m, m)
        orc.trmm_rlnn("d", m, nx, 1.0, prev, off, off, hBA, 0, 0, hW, 0, 0)
        orc.syrk_potrf_ln("d", m, nx, hW, 0, 0, hW, 0, 0, hR, 0, 0, hLk, 0, 0)
        Ls[k] = np.tril(hLk.get())
        prev, off = hLk, nu
    return Ls


@pytest.mark.parametrize("dims", [(12, 4, 30), (8, 3, 7), (5, 0, 4), (13, 3, 1), (4, 4, 0)])
def test_riccati_time_varying_vs_oracle(bf, dims):
    nx, nu, N = dims
    orc = oracle_api()
    rng = np.random.default_rng(nx * 100 + nu * 10 + N)
    nbt = 37
    m = nx + nu
    BAs = np.zeros((nbt, max(N, 1), 16, nx))
    RSQs = np.zeros((nbt, N + 1, 16, 16))
    for b in range(nbt):
        for k in range(N + 1):
            G = rng.standard_normal((m, m))
            RSQs[b, k, :m, :m] = G @ G.T / m + np.eye(m)
            if k < N:
                BAs[b, k, :m] = rng.standard_normal((m, nx)) / np.sqrt(nx)
    if N == 0:
        BAs = BAs[:, :0]
    L, info = run(bf, "d", BAs if N > 0 else np.zeros((nbt, 0, 16, nx)), RSQs, nx, nu)
    assert (info == 0).all()
    for b in (0, nbt // 2, nbt - 1):
        Ls = oracle_riccati(orc, BAs[b], RSQs[b], N, nx, nu)
        for k in range(N + 1):
            mm = nx if k == N else m
            assert relfro(np.tril(L[b, k, :mm, :mm]), Ls[k]) <= 1e-13, (b, k)
    # single precision: error against the FP64 factor stays at FP32 level
    Ls32, info32 = run(bf, "s", BAs.astype(np.float32), RSQs.astype(np.float32), nx, nu)
    assert (info32 == 0).all()
    assert relfro(np.tril(Ls32[:, 0, :m, :m]), np.tril(L[:, 0, :m, :m])) <= 1e-5


def test_riccati_reports_bad_pivot(bf):
    nx, nu, N = 4, 2, 3
    nbt = 3
    BAs = np.zeros((nbt, N, 16, nx))
    RSQs = np.broadcast_to(np.eye(16), (nbt, N + 1, 16, 16)).copy()
    RSQs[1, 1, 2, 2] = -10.0  # stage 1 of problem 1: indefinite
    L, info = run(bf, "d", BAs, RSQs, nx, nu)
    assert info[0] == 0 and info[2] == 0
    assert info[1] == 16 * (N - 1) + 3


def run_il(bf, BAs, RSQs, nx, nu):
    """The interleaved-slab factorization: stage-major slabs (stage k of
    problem b at instance k * bs + b, bs = batch rounded up to 16)."""
    import ctypes as C
    import torch
    from blasfeo_b200.api import DMatBatchIL
    nbt, N = BAs.shape[:2]
    bs = (nbt + 15) // 16 * 16
    ba = np.zeros((max(N, 1) * bs, 16, nx))
    rsq = np.zeros(((N + 1) * bs, 16, 16))
    for k in range(N):
        ba[k * bs: k * bs + nbt] = BAs[:, k]
    for k in range(N + 1):
        rsq[k * bs: k * bs + nbt] = RSQs[:, k]
    iBA = DMatBatchIL(16, nx, len(ba)).from_batch(bf.DMatBatch(16, nx, len(ba)).pack_all(ba))
    iRSQ = DMatBatchIL(16, 16, len(rsq)).from_batch(bf.DMatBatch(16, 16, len(rsq)).pack_all(rsq))
    iL = DMatBatchIL(16, 16, len(rsq))
    info = torch.full((nbt,), -9, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dric_trf_batch_il(nbt, N, nx, nu, iBA.ref, iRSQ.ref, iL.ref, C.c_void_p(info.data_ptr()),
                                          None)
    assert st == 0
    out = iL.to_batch(bf.DMatBatch(16, 16, len(rsq)))
    torch.cuda.synchronize()
    Lall, dall = out.unpack_all(), out.diag_all(16)
    L = np.stack([Lall[k * bs: k * bs + nbt] for k in range(N + 1)], axis=1)
    dA = np.stack([dall[k * bs: k * bs + nbt] for k in range(N + 1)], axis=1)
    return L, dA, info.cpu().numpy()


def test_riccati_il_vs_golden_reference(bf):
    g = np.load(os.path.join(GOLD, "cfg4.npz"))
    N, nx, nu = 30, 12, 4
    BAs, RSQs = zip(*[problem_mats(g["A%d" % p], g["B%d" % p], N, nx, nu) for p in range(2)])
    L, _, info = run_il(bf, np.stack(BAs), np.stack(RSQs), nx, nu)
    assert (info == 0).all()
    for p in range(2):
        for k in range(N + 1):
            m = nx if k == N else nx + nu
            assert relfro(np.tril(L[p, k, :m, :m]), g["L%d" % p][k][:m, :m]) <= 1e-13, (p, k)


@pytest.mark.parametrize("dims", [(12, 4, 30, 53), (8, 3, 7, 16), (5, 0, 4, 9), (13, 3, 1, 40), (4, 4, 0, 21)])
def test_riccati_il_vs_back_to_back_and_oracle(bf, dims):
    """Batches with partial groups and partial warps, nu = 0, N = 0 and N = 1,
    and one problem with an indefinite stage (same info as the back-to-back
    kernel)."""
    nx, nu, N, nbt = dims
    rng = np.random.default_rng(nx * 1000 + nu * 100 + N + nbt)
    m = nx + nu
    BAs = np.zeros((nbt, N, 16, nx))
    RSQs = np.zeros((nbt, N + 1, 16, 16))
    for b in range(nbt):
        for k in range(N + 1):
            G = rng.standard_normal((m, m))
            RSQs[b, k, :m, :m] = G @ G.T / m + np.eye(m)
            if k < N:
                BAs[b, k, :m] = rng.standard_normal((m, nx)) / np.sqrt(nx)
    bad_b = nbt // 3
    RSQs[bad_b, N // 2, 1, 1] = -50.0
    L, dA, info = run_il(bf, BAs, RSQs, nx, nu)
    L2, info2 = run(bf, "d", BAs, RSQs, nx, nu)
    assert np.array_equal(info, info2)
    assert info[bad_b] > 0 and (np.delete(info, bad_b) == 0).all()
    for k in range(N + 1):
        mm = nx if k == N else m
        ok = info == 0
        assert relfro(np.tril(L[ok, k, :mm, :mm]), np.tril(L2[ok, k, :mm, :mm])) <= 1e-13, k
        assert relfro(dA[ok, k, :mm], 1.0 / np.diagonal(L2[ok, k, :mm, :mm], axis1=1, axis2=2)) <= 1e-13, k
    orc = oracle_api()
    for b in (0, nbt - 1):
        if info[b]:
            continue
        Ls = oracle_riccati(orc, BAs[b], RSQs[b], N, nx, nu)
        for k in range(N + 1):
            mm = nx if k == N else m
            assert relfro(np.tril(L[b, k, :mm, :mm]), Ls[k]) <= 1e-13, (b, k)


def test_riccati_il_rejects(bf):
    from blasfeo_b200.api import DMatBatchIL
    f = bf.lib.blasfeo_dric_trf_batch_il
    BA, R = DMatBatchIL(16, 12, 2 * 16), DMatBatchIL(16, 16, 3 * 16)
    assert f(10, 2, 12, 4, BA.ref, R.ref, R.ref, None, None) == 0
    assert f(10, 2, 13, 4, BA.ref, R.ref, R.ref, None, None) == 4     # nu + nx > 16
    assert f(10, 2, 11, 4, BA.ref, R.ref, R.ref, None, None) == 1     # BAbt not 16 x nx
    assert f(17, 2, 12, 4, BA.ref, R.ref, R.ref, None, None) == 1     # slabs shorter than (N+1) * 32
    assert f(0, 2, 12, 4, BA.ref, R.ref, R.ref, None, None) == 0
