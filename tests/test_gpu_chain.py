"""GPU parity of the fused n=16 chain (syrk -> +shift I -> potrf -> trsm ->
gemm) against the golden fixtures of the compiled reference, against the
oracle, and against the same chain built from the batched entry points and
replayed as a CUDA graph."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.helpers import oracle_api, relfro

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    return blasfeo_b200


def _batch(bf, arr):
    b, m, n = arr.shape
    return bf.DMatBatch(m, n, b).pack_all(arr)


def _run_fused(bf, A, R, Cm, G, shift=16.0):
    import torch
    nb, m, k = A.shape
    dA, dR, dC, dG = _batch(bf, A), _batch(bf, R), _batch(bf, Cm), _batch(bf, G)
    dL, dX, dD = bf.DMatBatch(m, m, nb), bf.DMatBatch(m, m, nb), bf.DMatBatch(m, m, nb)
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    st = bf.lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(nb, m, k, shift, dA.ref, dR.ref, dC.ref, dG.ref, dL.ref,
                                                       dX.ref, dD.ref, C.c_void_p(info.data_ptr()), None)
    torch.cuda.synchronize()
    assert st == 0
    assert (info.cpu().numpy() == 0).all()
    return dL, dX, dD


def test_chain_vs_golden_reference_outputs(bf):
    g = np.load(os.path.join(GOLD, "cfg2.npz"))
    dL, dX, dD = _run_fused(bf, g["A"], g["R"], g["C"], g["G"])
    L, X, D = dL.unpack_all(), dX.unpack_all(), dD.unpack_all()
    for b in range(g["A"].shape[0]):
        assert relfro(np.tril(L[b]), g["L"][b]) <= 1e-13
        assert relfro(X[b], g["X"][b]) <= 1e-13
        assert relfro(D[b], g["D"][b]) <= 1e-13


def test_chain_random_batch_vs_oracle_and_inverse_diag(bf):
    rng = np.random.default_rng(8)
    nb, m, k = 1000, 16, 32
    A = rng.standard_normal((nb, m, k))
    R, Cm, G = (rng.standard_normal((nb, m, m)) for _ in range(3))
    dL, dX, dD = _run_fused(bf, A, R, Cm, G)
    L, X, D, dg = dL.unpack_all(), dX.unpack_all(), dD.unpack_all(), dL.diag_all(m)
    for b in (0, 1, 499, 999):
        S = A[b] @ A[b].T + 16 * np.eye(m)
        Lr = np.linalg.cholesky(S)
        assert relfro(np.tril(L[b]), Lr) <= 1e-13
        assert relfro(dg[b], 1 / np.diag(Lr)) <= 1e-13
        Xr = np.linalg.solve(Lr, R[b].T).T
        assert relfro(X[b], Xr) <= 1e-13
        assert relfro(D[b], Cm[b] - Xr @ G[b].T) <= 1e-13
    # upper triangle of L untouched (left as allocated: zeros)
    assert np.abs(np.triu(L, 1)).max() == 0.0


def test_chain_odd_k_and_graph_of_unfused_calls(bf):
    import torch
    rng = np.random.default_rng(9)
    nb, m, k = 300, 16, 13
    A = rng.standard_normal((nb, m, k))
    R, Cm, G = (rng.standard_normal((nb, m, m)) for _ in range(3))
    dL, dX, dD = _run_fused(bf, A, R, Cm, G, shift=3.0)
    # the same chain from the batched entry points, captured as one CUDA graph
    lib = bf.lib
    uA = _batch(bf, A)
    uS0 = _batch(bf, np.broadcast_to(3.0 * np.eye(m), (nb, m, m)).copy())
    uS = bf.DMatBatch(m, m, nb)
    uL, uR, uX = bf.DMatBatch(m, m, nb), _batch(bf, R), bf.DMatBatch(m, m, nb)
    uC, uG, uD = _batch(bf, Cm), _batch(bf, G), bf.DMatBatch(m, m, nb)
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    h = C.c_void_p(s.cuda_stream)
    with torch.cuda.graph(graph, stream=s):
        lib.blasfeo_dsyrk_ln_batch(nb, m, k, 1.0, uA.ref, 0, 0, uA.ref, 0, 0, 1.0, uS0.ref, 0, 0, uS.ref, 0, 0, h)
        lib.blasfeo_dpotrf_l_batch(nb, m, uS.ref, 0, 0, uL.ref, 0, 0, None, h)
        lib.blasfeo_dtrsm_rltn_batch(nb, m, m, 1.0, uL.ref, 0, 0, uR.ref, 0, 0, uX.ref, 0, 0, h)
        lib.blasfeo_dgemm_nt_batch(nb, m, m, m, -1.0, uX.ref, 0, 0, uG.ref, 0, 0, 1.0, uC.ref, 0, 0, uD.ref, 0, 0, h)
    graph.replay()
    torch.cuda.synchronize()
    assert relfro(np.tril(dL.unpack_all()), np.tril(uL.unpack_all())) <= 1e-13
    assert relfro(dX.unpack_all(), uX.unpack_all()) <= 1e-13
    assert relfro(dD.unpack_all(), uD.unpack_all()) <= 1e-13
    # replaying again gives the same result (every output is written from unchanged inputs)
    graph.replay()
    torch.cuda.synchronize()
    assert relfro(dD.unpack_all(), uD.unpack_all()) <= 1e-13


def test_chain_rejects_unsupported(bf):
    a = bf.dmat_batch()
    assert bf.lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(1, 12, 8, 1.0, C.byref(a), C.byref(a), C.byref(a),
                                                         C.byref(a), C.byref(a), C.byref(a), C.byref(a), None,
                                                         None) == 4
