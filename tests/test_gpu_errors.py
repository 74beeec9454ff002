"""Error paths that need a GPU but fault nothing: the bounded mbarrier wait
running out (a wait on data that no copy delivers), and iterative refinement
that is not allowed enough steps to reach its tolerance."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = lambda t: C.c_void_p(t.data_ptr())


def test_bounded_wait_times_out_and_gpu_stays_usable():
    import torch
    import blasfeo_b200 as bf
    lib = bf.lib
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    try:
        lib.blasfeo_b200_set_wait_limit(64)  # a few microseconds
        assert lib.blasfeo_b200_check_wait_timeout(P(status), None) == 0
        torch.cuda.synchronize()
        assert int(status.item()) == -3
    finally:
        lib.blasfeo_b200_set_wait_limit(0)
    # with the default limit the same kernel still reports the timeout (nothing is ever delivered)
    # only when it runs out; the context is healthy: a bulk-copy kernel runs normally afterwards
    from blasfeo_b200.api import DMatBatch
    from blasfeo_b200.workloads import fill_batch
    nb = 64
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    A = DMatBatch(16, 32, nb)
    fill_batch(A, torch.randn((nb, 16, 32), generator=g, dtype=torch.float64, device="cuda"))
    R, Cm, G = (DMatBatch(16, 16, nb) for _ in range(3))
    for M in (R, Cm, G):
        fill_batch(M, torch.randn((nb, 16, 16), generator=g, dtype=torch.float64, device="cuda"))
    L, X, D = (DMatBatch(16, 16, nb) for _ in range(3))
    info = torch.full((nb,), 9, dtype=torch.int32, device="cuda")
    st = lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(nb, 16, 32, 16.0, A.ref, R.ref, Cm.ref, G.ref, L.ref, X.ref, D.ref,
                                                   P(info), None)
    torch.cuda.synchronize()
    assert st == 0 and (info.cpu().numpy() == 0).all()
    a = A.unpack_all()
    Lr = np.linalg.cholesky(a[0] @ a[0].T + 16 * np.eye(16))
    assert np.abs(np.tril(L.unpack_all()[0]) - Lr).max() <= 1e-12


@pytest.mark.parametrize("max_iter", [0, 1])
def test_refinement_without_enough_steps_reports_minus_one(max_iter):
    """cond(A) up to 1e6: the FP32 factor's first solve leaves a backward error
    far above 1e-12, so with no refinement step allowed every system ends with
    info = -1, iters = 0 and berr > tol; with one step allowed a system either
    converged in that step (info 0) or reports info = -1, iters = 1 and
    berr > tol, and most do not converge.  With the default 30 steps every
    system converges."""
    import torch
    import blasfeo_b200 as bf
    from blasfeo_b200.workloads import spd_config3
    lib = bf.lib
    num = 40
    W = spd_config3(num, seed=21, nmin=60, nmax=200, logcond=6.0)
    info = torch.full((num,), 9, dtype=torch.int32, device="cuda")
    iters = torch.full((num,), -5, dtype=torch.int32, device="cuda")
    berr = torch.zeros(num, dtype=torch.float64, device="cuda")
    st = lib.blasfeo_dsposv_l_vbatch(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), max_iter, 1e-12,
                                     P(iters), P(berr), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0
    inf, it, be = info.cpu().numpy(), iters.cpu().numpy(), berr.cpu().numpy()
    failed = inf == -1
    assert ((inf == 0) | failed).all(), inf
    assert failed.sum() > num // 2, inf
    assert (it[failed] == max_iter).all() and (be[failed] > 1e-12).all(), (it, be)
    assert (it[~failed] <= max_iter).all() and (be[~failed] <= 1e-12).all(), (it, be)
    if max_iter == 0:
        assert failed.all()
    st = lib.blasfeo_dsposv_l_vbatch(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12,
                                     P(iters), P(berr), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0 and (info.cpu().numpy() == 0).all() and (berr.cpu().numpy() <= 1e-12).all()
