"""GPU parity of the tensor-core engine of blasfeo_dsposv_l_vbatch (trailing
matrix in tensor memory, 3xTF32 tcgen05.mma updates, FP64 diagonal blocks,
FP64 residual and refinement) through the C ABI: backward error against the
FP64 matrix on the host, the reference's silent-zero pivot rule on
indefinite input, and agreement with the SIMT engine on the uneven-size
workload (n ~ U{4..256}, cond up to 1e6)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = lambda t: C.c_void_p(t.data_ptr())


@pytest.fixture
def bf():
    import blasfeo_b200
    blasfeo_b200.set_sync(True)
    prev = blasfeo_b200.set_posv_engine(blasfeo_b200.POSV_TENSOR)
    yield blasfeo_b200
    blasfeo_b200.set_posv_engine(prev)


def _solve(bf, mats, bvecs, xvecs, ns, max_iter=30, tol=1e-12):
    import torch
    nb = len(ns)
    dA, db, dx = bf.descriptor_array(mats), bf.vector_array(bvecs), bf.vector_array(xvecs)
    nv = torch.tensor(ns, dtype=torch.int32, device="cuda")
    info = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    iters = torch.full((nb,), -9, dtype=torch.int32, device="cuda")
    berr = torch.full((nb,), -1.0, dtype=torch.float64, device="cuda")
    st = bf.lib.blasfeo_dsposv_l_vbatch(nb, P(nv), max(ns), P(dA), P(db), P(dx), max_iter, tol, P(iters), P(berr),
                                        P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0
    return info.cpu().numpy(), iters.cpu().numpy(), berr.cpu().numpy()


def _spd(rng, n, cond):
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = 10.0 ** rng.uniform(0, np.log10(cond), n)
    a = (q * lam) @ q.T
    return 0.5 * (a + a.T)


def _berr(a, b, x):
    return np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max())


def test_tensor_engine_sizes(bf):
    # every padding case of the 16-column blocks and both 128-row TMEM halves
    rng = np.random.default_rng(5)
    ns = [1, 2, 4, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 143, 144, 145, 200, 239, 240, 241, 255,
          256, 3, 128, 256]
    As = [_spd(rng, n, 1e6) for n in ns]
    bs = [rng.standard_normal(n) for n in ns]
    mats = [bf.DMat(n, n).pack(a) for n, a in zip(ns, As)]
    bvecs = [bf.DVec(n).pack(b) for n, b in zip(ns, bs)]
    xvecs = [bf.DVec(n) for n in ns]
    info, iters, berr = _solve(bf, mats, bvecs, xvecs, ns)
    assert (info == 0).all(), info
    assert (berr <= 1e-12).all(), berr
    assert (iters >= 0).all() and (iters <= 30).all(), iters
    for n, a, b, xv, be in zip(ns, As, bs, xvecs, berr):
        x = xv.unpack()
        e = _berr(a, b, x)
        assert e <= 1e-12, (n, e)
        # the device's backward error is the same quantity (up to the rounding
        # of the residual itself, visible at the 1e-16 level)
        assert abs(e - be) <= 0.05 * max(e, be) + 1e-16, (n, e, be)


def test_tensor_engine_converges_fast_on_wellconditioned(bf):
    # a 3xTF32 factor is FP32-accurate: cond ~ 10 needs at most two corrections
    rng = np.random.default_rng(6)
    ns = [16, 80, 160, 256]
    As = [_spd(rng, n, 10.0) for n in ns]
    bs = [rng.standard_normal(n) for n in ns]
    mats = [bf.DMat(n, n).pack(a) for n, a in zip(ns, As)]
    bvecs = [bf.DVec(n).pack(b) for n, b in zip(ns, bs)]
    xvecs = [bf.DVec(n) for n in ns]
    info, iters, berr = _solve(bf, mats, bvecs, xvecs, ns)
    assert (info == 0).all() and (berr <= 1e-12).all()
    assert (iters <= 2).all(), iters


@pytest.mark.parametrize("n,k", [(16, 0), (16, 15), (40, 17), (130, 129), (256, 200)])
def test_tensor_engine_indefinite_pivot(bf, n, k):
    # identity with one negative diagonal entry: the first non-positive pivot is
    # column k, reported as info = k + 1 (reference rule: pivot and its
    # reciprocal set to zero, no error raised)
    a = np.eye(n)
    a[k, k] = -1.0
    b = np.ones(n)
    mats, bvecs, xvecs = [bf.DMat(n, n).pack(a)], [bf.DVec(n).pack(b)], [bf.DVec(n)]
    info, _, _ = _solve(bf, mats, bvecs, xvecs, [n])
    assert info[0] == k + 1, info


def test_tensor_engine_matches_simt_engine_uneven_batch(bf):
    import torch
    from blasfeo_b200.workloads import spd_config3
    num = 600
    W = spd_config3(num, seed=21)
    out = {}
    for eng in (bf.POSV_SIMT, bf.POSV_TENSOR):
        bf.set_posv_engine(eng)
        W.x.zero_()
        info = torch.full((num,), -9, dtype=torch.int32, device="cuda")
        berr = torch.zeros(num, dtype=torch.float64, device="cuda")
        st = bf.lib.blasfeo_dsposv_l_vbatch(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12,
                                            None, P(berr), P(info), None, 0, None)
        torch.cuda.synchronize()
        assert st == 0
        assert (info.cpu().numpy() == 0).all(), eng
        assert (berr.cpu().numpy() <= 1e-12).all(), eng
        out[eng] = W.x.clone()
    # both solutions are backward stable to 1e-12: they agree to ~cond * 1e-12
    d = (out[bf.POSV_SIMT] - out[bf.POSV_TENSOR]).norm().item() / out[bf.POSV_SIMT].norm().item()
    assert d <= 1e-5, d
    for i in np.argsort(W.ns)[-4:]:
        assert _berr(W.matrix(int(i)), W.rhs[int(i)], W.solution(int(i))) <= 1e-12


def test_engine_switch_rejects_unknown(bf):
    assert bf.lib.blasfeo_b200_set_posv_engine(7) != 0
    assert bf.lib.blasfeo_b200_get_posv_engine() == bf.POSV_TENSOR
