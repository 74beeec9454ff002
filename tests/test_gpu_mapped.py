"""GPU tests of the mixed SPD solver for inputs in mapped host memory
(blasfeo_dsposv_l_vbatch_mapped, the `e2e` path of the benchmark): the same
solutions as the device path on the same systems, backward errors within the
tolerance, and a caller workspace that is too small refused before any
device work."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    import blasfeo_b200 as bf
    from blasfeo_b200.workloads import spd_config3
    W = spd_config3(num=600, seed=21)
    P = lambda t: C.c_void_p(t.data_ptr())
    info = torch.zeros(600, dtype=torch.int32, device="cuda")
    berr = torch.zeros(600, dtype=torch.float64, device="cuda")
    st = bf.lib.blasfeo_dsposv_l_vbatch(600, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12,
                                        None, P(berr), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0 and bool((info == 0).all().item())
    xdev = W.x.cpu().numpy().copy()
    return bf, W, xdev


def _mapped(bf, W, work=None, work_bytes=0):
    import torch
    H = W.mapped_copy()
    info = torch.full((len(W.ns),), -9, dtype=torch.int32).pin_memory()
    berr = torch.zeros(len(W.ns), dtype=torch.float64).pin_memory()
    P = lambda t: C.c_void_p(t.data_ptr())
    st = bf.lib.blasfeo_dsposv_l_vbatch_mapped(len(W.ns), P(H.n), W.max_n, P(H.desc), P(H.bdesc), P(H.xdesc), 30,
                                               1e-12, None, P(berr), P(info), work, work_bytes, None)
    torch.cuda.synchronize()
    return st, H, info.numpy().copy(), berr.numpy().copy()


def test_mapped_matches_device_path(setup):
    bf, W, xdev = setup
    st, H, info, berr = _mapped(bf, W)
    assert st == 0
    assert (info == 0).all()
    assert berr.max() <= 1e-12
    x = H.x.numpy()
    assert np.linalg.norm(x - xdev) <= 1e-13 * np.linalg.norm(xdev)
    # the largest system re-checked on the host in FP64
    i = int(np.argmax(W.ns))
    a, b = W.matrix(i), W.rhs[i]
    xi = H.solution(i, len(b))
    assert np.abs(b - a @ xi).max() / (np.abs(a).sum(1).max() * np.abs(xi).max()) <= 1e-12


def test_mapped_small_workspace_refused(setup):
    import torch
    bf, W, _ = setup
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    st, H, info, _ = _mapped(bf, W, C.c_void_p(small.data_ptr()), small.numel())
    assert st == 3  # BLASFEO_B200_ENOMEM, before any device work
    assert (info == -9).all()
    assert not H.x.numpy().any()
