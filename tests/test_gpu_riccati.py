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
