"""Single-routine cases for profiling one kernel under ncu (small, seeded).

Usage: python -m blasfeo_b200.profile_cases OP N BATCH REPS [NMIN]
  gemm  N BATCH REPS       blasfeo_dgemm_nt_batch, n = m = k = N, A, B ~ U[-1,1], beta = 0
  potrf N BATCH REPS       blasfeo_dpotrf_l_batch on C = G G^T / N + I, G ~ N(0,1)
  posv  N BATCH REPS NMIN  blasfeo_dposv_l_vbatch on the uneven SPD workload with n ~ U{NMIN..N}
  sposv N BATCH REPS NMIN  blasfeo_dsposv_l_vbatch (mixed precision), same inputs
  ric   N BATCH REPS       blasfeo_dric_trf_batch, horizon N, nx = 12, nu = 4, BATCH problems
                           (A = I + 0.1 N(0,1) scaled to spectral radius 0.95, B ~ N(0,1)/sqrt(12), Q = R = I)
Each call goes through the C ABI; REPS calls back to back, then a check of info.
"""
import ctypes as C, sys, os
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import torch
import blasfeo_b200 as bf
from blasfeo_b200.workloads import fill_batch, to_panel_major, spd_config3
lib = bf.lib
dev = torch.device("cuda")
op, n, batch, reps = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4])
P = lambda t: C.c_void_p(t.data_ptr())
if op == "gemm":
    A, B, D = bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch)
    fill_batch(A, torch.rand((batch, n, n), dtype=torch.float64, device=dev) * 2 - 1)
    fill_batch(B, torch.rand((batch, n, n), dtype=torch.float64, device=dev) * 2 - 1)
    for _ in range(reps):
        assert lib.blasfeo_dgemm_nt_batch(batch, n, n, n, 1.0, A.ref, 0, 0, B.ref, 0, 0, 0.0, D.ref, 0, 0, D.ref, 0, 0, None) == 0
elif op == "potrf":
    Cm, L = bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch)
    pm, cn, st = Cm.s.pm, Cm.s.cn, Cm.s.stride
    for s0 in range(0, batch, 4096):
        s1 = min(batch, s0 + 4096)
        G = torch.randn((s1 - s0, n, n), dtype=torch.float64, device=dev)
        S = G @ G.transpose(1, 2) / n + torch.eye(n, dtype=torch.float64, device=dev)
        Cm.buf[s0 * st * 8: s1 * st * 8].view(torch.float64).view(s1 - s0, st)[:, : pm * cn] = to_panel_major(S, pm, cn)
    info = torch.zeros(batch, dtype=torch.int32, device=dev)
    for _ in range(reps):
        assert lib.blasfeo_dpotrf_l_batch(batch, n, Cm.ref, 0, 0, L.ref, 0, 0, P(info), None) == 0
    torch.cuda.synchronize()
    assert bool((info == 0).all().item())
elif op in ("posv", "sposv"):
    lo = int(sys.argv[5]) if len(sys.argv) > 5 else n
    W = spd_config3(batch, nmin=lo, nmax=n, seed=3, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device=dev)
    for _ in range(reps):
        if op == "posv":
            st = lib.blasfeo_dposv_l_vbatch(batch, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), P(info), None, 0, None)
        else:
            st = lib.blasfeo_dsposv_l_vbatch(batch, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30, 1e-12, None, None, P(info), None, 0, None)
        assert st == 0
    torch.cuda.synchronize()
    assert bool((info == 0).all().item())
elif op == "ric":
    import numpy as np
    N, nx, nu = n, 12, 4
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    A = torch.eye(nx, dtype=torch.float64, device=dev) + 0.1 * torch.randn((batch, nx, nx), generator=g, dtype=torch.float64, device=dev)
    A = A * (0.95 / torch.linalg.eigvals(A.cpu()).abs().max(dim=1).values.to(dev))[:, None, None]
    B = torch.randn((batch, nx, nu), generator=g, dtype=torch.float64, device=dev) / np.sqrt(nx)
    BA = torch.zeros((batch, 16, nx), dtype=torch.float64, device=dev)
    BA[:, :nu] = B.transpose(1, 2)
    BA[:, nu:] = A.transpose(1, 2)
    sBA, sRSQ, sL = bf.DMatBatch(16, nx, batch * N), bf.DMatBatch(16, 16, batch * (N + 1)), bf.DMatBatch(16, 16, batch * (N + 1))
    fill_batch(sBA, BA[:, None].expand(batch, N, 16, nx).reshape(batch * N, 16, nx).contiguous())
    fill_batch(sRSQ, torch.eye(16, dtype=torch.float64, device=dev).expand(batch * (N + 1), 16, 16).contiguous())
    info = torch.zeros(batch, dtype=torch.int32, device=dev)
    for _ in range(reps):
        assert lib.blasfeo_dric_trf_batch(batch, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, P(info), None) == 0
    torch.cuda.synchronize()
    assert bool((info == 0).all().item())
torch.cuda.synchronize()
print("ok", op, n, batch)
