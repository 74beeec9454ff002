"""GPU test of blasfeo_dsposv_l_vbatch_noalloc, the allocation-free entry point.

It exists for callers that cannot allocate device memory while they run
(embedded / real-time solvers whose memory is fixed at start-up, code that
cannot take cudaMalloc's device-wide synchronisation) and that pass no
workspace: its scratch is a static device array owned by the library.  The
test calls it through the C ABI twice in a row and checks both results
against the allocating entry point on the same inputs.  The file name sorts
last so that a run stopping at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(num, seed):
    from blasfeo_b200.workloads import spd_config3
    return spd_config3(num, seed=seed)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import blasfeo_b200 as bf
    lib = bf.lib
    P = lambda t: C.c_void_p(t.data_ptr())
    num = 300
    W = _inputs(num, seed=11)
    info = torch.full((num,), -9, dtype=torch.int32, device="cuda")
    berr = torch.zeros(num, dtype=torch.float64, device="cuda")
    st = lib.blasfeo_dsposv_l_vbatch(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12, None,
                                     P(berr), P(info), None, 0, None)
    torch.cuda.synchronize()
    assert st == 0 and (info.cpu().numpy() == 0).all()
    x_ref = W.x.clone()
    for call in range(2):
        W.x.zero_()
        info.fill_(-9)
        berr.zero_()
        st = lib.blasfeo_dsposv_l_vbatch_noalloc(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30,
                                                 1e-12, None, P(berr), P(info), None)
        torch.cuda.synchronize()
        assert st == 0, (call, st)
        assert (info.cpu().numpy() == 0).all(), call
        assert (berr.cpu().numpy() <= 1e-12).all(), call
        diff = (W.x - x_ref).norm().item() / x_ref.norm().item()
        assert diff <= 1e-12, (call, diff)
    # spot check against the host: backward error of the largest system
    i = int(np.argmax(W.ns))
    a, b, x = W.matrix(i), W.rhs[i], W.solution(i)
    assert np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max()) <= 1e-12


def test_noalloc_rejects_oversize_requests():
    import blasfeo_b200 as bf
    lib = bf.lib
    ENOTSUP = 4
    big = 65536 + 1
    assert lib.blasfeo_dsposv_l_vbatch_noalloc(big, None, 16, None, None, None, 30, 1e-12, None, None, None,
                                               None) == ENOTSUP
    assert lib.blasfeo_dsposv_l_vbatch_noalloc(10, None, 257, None, None, None, 30, 1e-12, None, None, None,
                                               None) == ENOTSUP
    # the static array is exactly the scratch the allocating entry point asks for at the limit
    assert lib.blasfeo_dsposv_noalloc_scratch_bytes() == lib.blasfeo_dposv_worksize(65536)


def _noalloc_call(lib, W, num, berr, info):
    P = lambda t: C.c_void_p(t.data_ptr())
    return lib.blasfeo_dsposv_l_vbatch_noalloc(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12,
                                               None, P(berr), P(info), None)


def test_noalloc_largest_size_and_tensor_engine_allocate_nothing():
    """Systems up to the documented limit n = 256, on both engines of the
    solver, from a host thread that has never called the library (so it owns no
    library workspace): the device's free memory is the same before and after
    the calls, and the results match the allocating entry point."""
    import threading
    import torch
    import blasfeo_b200 as bf
    from blasfeo_b200.workloads import spd_config3
    lib = bf.lib
    P = lambda t: C.c_void_p(t.data_ptr())
    num = 120
    W = spd_config3(num, seed=13, nmin=200, nmax=256)  # seed 13 draws n = 256 twice
    assert W.max_n == 256
    info = torch.full((num,), -9, dtype=torch.int32, device="cuda")
    berr = torch.zeros(num, dtype=torch.float64, device="cuda")
    assert lib.blasfeo_dsposv_l_vbatch(num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12, None,
                                       P(berr), P(info), None, 0, None) == 0
    torch.cuda.synchronize()
    x_ref = W.x.clone()
    # first call on this device (looks up the static array's address; loads the module)
    assert _noalloc_call(lib, W, num, berr, info) == 0
    # and a first call of the tensor-memory engine: under the driver's lazy
    # module loading a kernel's first launch may map memory for its code, which
    # is not an allocation of the entry point (the same call is repeated below)
    assert lib.blasfeo_b200_set_posv_engine(2) == 0
    assert _noalloc_call(lib, W, num, berr, info) == 0
    assert lib.blasfeo_b200_set_posv_engine(0) == 0
    torch.cuda.synchronize()
    out = {}

    def worker():
        try:
            torch.cuda.set_device(0)
            free = []
            for engine in (1, 2):  # SIMT, then the tensor-memory engine (the setting is per host thread)
                assert lib.blasfeo_b200_set_posv_engine(engine) == 0
                W.x.zero_()
                info.fill_(-9)
                torch.cuda.synchronize()
                # free memory right around the call (torch's own first kernel
                # launches on this thread stay outside the window)
                f0 = torch.cuda.mem_get_info()[0]
                st = _noalloc_call(lib, W, num, berr, info)
                torch.cuda.synchronize()
                free.append((f0, torch.cuda.mem_get_info()[0]))
                out[engine] = (st, info.cpu().numpy().copy(), berr.cpu().numpy().copy(),
                               ((W.x - x_ref).norm() / x_ref.norm()).item())
            out["free"] = free
        except Exception as ex:  # reported by the main thread
            out["error"] = repr(ex)

    t = threading.Thread(target=worker)
    t.start()
    t.join()
    assert "error" not in out, out.get("error")
    for engine in (1, 2):
        st, inf, be, diff = out[engine]
        assert st == 0 and (inf == 0).all() and (be <= 1e-12).all(), engine
        # SIMT is the allocating call's engine: the same arithmetic, the same x.  The
        # tensor-memory engine rounds differently; both solutions are backward stable
        # to 1e-12, so they agree to about cond(A) * 1e-12 = 1e-6 (cond up to 1e6)
        assert diff <= (1e-12 if engine == 1 else 1e-5), (engine, diff)
    for free0, free1 in out["free"]:
        assert free0 == free1, (free0, free1)
