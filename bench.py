#!/usr/bin/env python
"""Benchmark: solved instances/s at FP64-level residual, mixed vs plain FP64.

Workload (one "step"): 20,000 independent SPD systems A x = b, n drawn
uniformly from 4..256 (seeded), A = Q diag(lambda) Q^T with Q from the QR of an
N(0,1) matrix and log10(lambda) ~ U[0,6], b ~ N(0,1); every system solved to
||b - A x||_inf <= 1e-12 ||A||_inf ||x||_inf.

  value : mixed-precision path (blasfeo_dsposv_l_vbatch: FP32 factor with FP64
          diagonal blocks + FP64 iterative refinement), inputs resident in HBM
  plain : plain FP64 path (blasfeo_dposv_l_vbatch), same inputs
  e2e   : the mixed path through blasfeo_dsposv_l_vbatch_mapped with every input
          in pinned host memory (matrices, right-hand sides, sizes,
          descriptors): the kernels read the lower triangles over the host link
          and write x back to host memory inside the timed region
  fp64_batched : plain FP64 batched dgemm_nt and dpotrf_l on uniform batches
          (n = 64, 128, 256, inputs larger than L2) against the FP64 roofline
  fused_kernels : the fused n=16 chain (100,000 instances) and the batched
          Riccati factorization (4,096 problems, N=30), GB/s against HBM
  learned_dispatch : the mixed-op stream (gemm/potrf/getrf/geqrf, sizes 4..384):
          regret of the MLP cost model's variant picks against the exhaustive
          autotuner, next to the built-in rule, and GFLOP/s of the stream
  cpu_baseline / --impl reference : the reference's own CPU path
          (blasfeo_dpotrf_l + blasfeo_dtrsv_lnn + blasfeo_dtrsv_ltn, BLASFEO
          compiled from source) on the host cores, threads over instances.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 launch one process per GPU with torch.distributed.run; every rank
solves its own batch (weak scaling, no data-path collective).

Single-routine cases for profiling one kernel under ncu (small, seeded; every
call goes through the C ABI, REPS calls back to back, then a check of info):
  python bench.py --case gemm  N BATCH REPS        blasfeo_dgemm_nt_batch, m = n = k = N, A, B ~ U[-1,1], beta = 0
  python bench.py --case potrf N BATCH REPS        blasfeo_dpotrf_l_batch on C = G G^T / N + I, G ~ N(0,1)
  python bench.py --case posv  N BATCH REPS NMIN   blasfeo_dposv_l_vbatch, uneven SPD systems n ~ U{NMIN..N}
  python bench.py --case sposv N BATCH REPS NMIN   blasfeo_dsposv_l_vbatch (mixed precision), same inputs
  python bench.py --case ric   N BATCH REPS        blasfeo_dric_trf_batch, horizon N, nx = 12, nu = 4
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solved instances/s at FP64-level residual, mixed vs plain FP64, same B200"
UNIT = "systems/s"
NUM = 20000
TOL = 1e-12
MAX_ITER = 30
WORKLOAD = ("uneven SPD batch: 20,000 systems, n~U{4..256}, A=Q diag(lambda) Q^T, log10(lambda)~U[0,6], "
            "b~N(0,1), refine to ||r||/(||A|| ||x||) <= 1e-12")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--num", type=int, default=NUM)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 batched dgemm/dpotrf roofline legs")
    ap.add_argument("--case", nargs="+", metavar="ARG",
                    help="run one profiling case instead of the benchmark: OP N BATCH REPS [NMIN | M]")
    return ap.parse_args()


def rank_seed(rank):
    """Seed of a rank's systems: every replica solves its own batch of the
    distribution (rank 0's is the batch the reference arm solves)."""
    return 1000 + rank


def reduce_max_ms(ms, world, dist, device):
    """The job's time of a step: the maximum over the ranks (the slowest replica
    finishes the job); the same collective on every rank."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(world, num, ms):
    """Whole-job systems/s: every rank solves `num` systems in `ms` (the max over ranks)."""
    return world * num / (ms * 1e-3)


def run_case(argv):
    """One routine on a small seeded workload, for an ncu capture of its kernel."""
    import torch
    import blasfeo_b200 as bf
    from blasfeo_b200.workloads import fill_batch, to_panel_major, spd_config3
    lib = bf.lib
    dev = torch.device("cuda")
    op, n, batch, reps = argv[0], int(argv[1]), int(argv[2]), int(argv[3])
    P = lambda t: C.c_void_p(t.data_ptr())
    if op == "gemm":
        A, B, D = bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch)
        fill_batch(A, torch.rand((batch, n, n), dtype=torch.float64, device=dev) * 2 - 1)
        fill_batch(B, torch.rand((batch, n, n), dtype=torch.float64, device=dev) * 2 - 1)
        for _ in range(reps):
            bf.check(lib.blasfeo_dgemm_nt_batch(batch, n, n, n, 1.0, A.ref, 0, 0, B.ref, 0, 0, 0.0, D.ref, 0, 0,
                                                D.ref, 0, 0, None))
    elif op == "potrf":
        Cm, L = bf.DMatBatch(n, n, batch), bf.DMatBatch(n, n, batch)
        pm, cn, st = Cm.s.pm, Cm.s.cn, Cm.s.stride
        for s0 in range(0, batch, 4096):
            s1 = min(batch, s0 + 4096)
            G = torch.randn((s1 - s0, n, n), dtype=torch.float64, device=dev)
            S = G @ G.transpose(1, 2) / n + torch.eye(n, dtype=torch.float64, device=dev)
            Cm.buf[s0 * st * 8: s1 * st * 8].view(torch.float64).view(s1 - s0, st)[:, : pm * cn] = \
                to_panel_major(S, pm, cn)
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        for _ in range(reps):
            bf.check(lib.blasfeo_dpotrf_l_batch(batch, n, Cm.ref, 0, 0, L.ref, 0, 0, P(info), None))
        torch.cuda.synchronize()
        assert bool((info == 0).all().item())
    elif op in ("posv", "sposv"):
        lo = int(argv[4]) if len(argv) > 4 else n
        W = spd_config3(batch, nmin=lo, nmax=n, seed=3, device="cuda")
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        for _ in range(reps):
            if op == "posv":
                st = lib.blasfeo_dposv_l_vbatch(batch, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc),
                                                P(info), None, 0, None)
            else:
                st = lib.blasfeo_dsposv_l_vbatch(batch, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30,
                                                 1e-12, None, None, P(info), None, 0, None)
            bf.check(st)
        torch.cuda.synchronize()
        assert bool((info == 0).all().item())
    elif op in ("ric", "ric_il"):
        N, nx, nu = n, 12, 4
        g = torch.Generator(device=dev)
        g.manual_seed(4)
        A = torch.eye(nx, dtype=torch.float64, device=dev) + 0.1 * torch.randn((batch, nx, nx), generator=g,
                                                                              dtype=torch.float64, device=dev)
        A = A * (0.95 / torch.linalg.eigvals(A.cpu()).abs().max(dim=1).values.to(dev))[:, None, None]
        B = torch.randn((batch, nx, nu), generator=g, dtype=torch.float64, device=dev) / np.sqrt(nx)
        BA = torch.zeros((batch, 16, nx), dtype=torch.float64, device=dev)
        BA[:, :nu] = B.transpose(1, 2)
        BA[:, nu:] = A.transpose(1, 2)
        sBA = bf.DMatBatch(16, nx, batch * N)
        sRSQ, sL = bf.DMatBatch(16, 16, batch * (N + 1)), bf.DMatBatch(16, 16, batch * (N + 1))
        fill_batch(sBA, BA[:, None].expand(batch, N, 16, nx).reshape(batch * N, 16, nx).contiguous())
        fill_batch(sRSQ, torch.eye(16, dtype=torch.float64, device=dev).expand(batch * (N + 1), 16, 16).contiguous())
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        if op == "ric_il":
            # stage-major interleaved slabs: stage k of problem b at instance k * bs + b
            from blasfeo_b200.api import DMatBatchIL
            bs = (batch + 15) // 16 * 16
            ba = torch.zeros((N * bs, 16, nx), dtype=torch.float64, device=dev)
            ba.view(N, bs, 16, nx)[:, :batch] = BA[None]
            tBA, tRSQ = bf.DMatBatch(16, nx, N * bs), bf.DMatBatch(16, 16, (N + 1) * bs)
            fill_batch(tBA, ba)
            fill_batch(tRSQ, torch.eye(16, dtype=torch.float64, device=dev).expand((N + 1) * bs, 16, 16).contiguous())
            sBA, sRSQ = DMatBatchIL(16, nx, N * bs).from_batch(tBA), DMatBatchIL(16, 16, (N + 1) * bs).from_batch(tRSQ)
            sL = DMatBatchIL(16, 16, (N + 1) * bs)
            f = lib.blasfeo_dric_trf_batch_il
        else:
            f = lib.blasfeo_dric_trf_batch
        for _ in range(reps):
            bf.check(f(batch, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, P(info), None))
        torch.cuda.synchronize()
        assert bool((info == 0).all().item())
    elif op == "cfg3":
        # the headline call on `batch` systems of the benchmark's distribution
        from blasfeo_b200.workloads import SpdBatch
        W = SpdBatch(*gen_config3(batch, 1000, "cuda"))
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        for _ in range(reps):
            bf.check(lib.blasfeo_dsposv_l_vbatch(batch, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), 30,
                                                 1e-12, None, None, P(info), None, 0, None))
        torch.cuda.synchronize()
        assert bool((info == 0).all().item())
    elif op in ("getrf", "geqrf"):
        # m x n instances (m = the optional fifth argument, default n)
        m = int(argv[4]) if len(argv) > 4 else n
        A, D = bf.DMatBatch(m, n, batch), bf.DMatBatch(m, n, batch)
        fill_batch(A, torch.rand((batch, m, n), dtype=torch.float64, device=dev) * 2 - 1)
        ipiv = torch.zeros(batch * min(m, n), dtype=torch.int32, device=dev)
        for _ in range(reps):
            if op == "getrf":
                bf.check(lib.blasfeo_dgetrf_rp_batch(batch, m, n, A.ref, 0, 0, D.ref, 0, 0, P(ipiv), None, None))
            else:
                bf.check(lib.blasfeo_dgeqrf_batch(batch, m, n, A.ref, 0, 0, D.ref, 0, 0, None))
    elif op in ("chain", "chain_il"):
        from blasfeo_b200.api import DMatBatchIL
        g = torch.Generator(device=dev)
        g.manual_seed(2)
        sl = {}
        for name, (r, c) in (("A", (16, 32)), ("R", (16, 16)), ("C", (16, 16)), ("G", (16, 16))):
            sl[name] = bf.DMatBatch(r, c, batch)
            fill_batch(sl[name], torch.randn((batch, r, c), generator=g, dtype=torch.float64, device=dev))
        outs = [bf.DMatBatch(16, 16, batch) for _ in range(3)]
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        if op == "chain_il":
            sl = {k: DMatBatchIL(v.m, v.n, batch).from_batch(v) for k, v in sl.items()}
            outs = [DMatBatchIL(16, 16, batch) for _ in range(3)]
            f = lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il
        else:
            f = lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch
        for _ in range(reps):
            bf.check(f(batch, 16, 32, 16.0, *(sl[k].ref for k in "ARCG"), *(o.ref for o in outs), P(info), None))
        torch.cuda.synchronize()
        assert bool((info == 0).all().item())
    elif op == "potrf_il":
        from blasfeo_b200.api import DMatBatchIL
        A = torch.randn((batch, n, 2 * n), dtype=torch.float64, device=dev)
        Cm = bf.DMatBatch(n, n, batch)
        fill_batch(Cm, A @ A.transpose(1, 2) + n * torch.eye(n, dtype=torch.float64, device=dev))
        Ci, Di = DMatBatchIL(n, n, batch).from_batch(Cm), DMatBatchIL(n, n, batch)
        for _ in range(reps):
            bf.check(lib.blasfeo_dpotrf_l_batch_il(batch, n, Ci.ref, Di.ref, None, None))
    else:
        raise SystemExit("unknown case %r" % op)
    torch.cuda.synchronize()
    print("ok", op, n, batch, flush=True)
    return 0


# ---------------------------------------------------------------------------
# CPU side: the reference (or the oracle port) on the host cores
# ---------------------------------------------------------------------------
def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def cpu_library():
    """(ctypes lib, prefix, kind, name): compiled reference if present, else the oracle port."""
    from oracle import pyoracle
    flags = _cpu_flags()
    for target in (["haswell"] if {"avx2", "fma"} <= flags else []) + ["generic"]:
        if pyoracle.ref_available(target):
            return pyoracle.ref_lib(target), "blasfeo_d", "reference", "BLASFEO 0.1.4.2 HP " + target
    from tests.helpers import ensure_oracle
    ensure_oracle()
    return pyoracle.oracle_lib(), "oracle_d_", "port", "oracle restatement (C, scalar loops)"


def physical_cpus():
    """One logical CPU per physical core among the CPUs this process may run
    on (sysfs topology: core_id and physical_package_id), so that P threads of
    the CPU baseline land on P different cores."""
    allowed = sorted(os.sched_getaffinity(0))
    seen, pick = set(), []
    for c in allowed:
        base = "/sys/devices/system/cpu/cpu%d/topology/" % c
        try:
            core = open(base + "core_id").read().strip()
            pkg = open(base + "physical_package_id").read().strip()
        except OSError:
            return allowed
        if (pkg, core) not in seen:
            seen.add((pkg, core))
            pick.append(c)
    return pick


def gen_config3(num, seed, device):
    """The benchmark's systems: n ~ U{4..256} (numpy, seeded); per size,
    A = Q diag(lambda) Q^T with Q from the QR of an N(0,1) matrix and
    log10(lambda) ~ U[0,6] (torch generator with the same seed, on `device`);
    b ~ N(0,1).  Returns (ns, {n: (indices, A tensor)}, [b]).  Both arms call
    this with the same seed, so the GPU arm and the reference arm solve the
    same systems."""
    import torch
    rng = np.random.default_rng(seed)
    ns = rng.integers(4, 257, size=num).astype(np.int32)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    mats = {}
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        G = torch.randn((len(idx), int(n), int(n)), generator=g, dtype=torch.float64, device=device)
        Q, _ = torch.linalg.qr(G)
        lam = 10.0 ** (torch.rand((len(idx), int(n)), generator=g, dtype=torch.float64, device=device) * 6.0)
        A = (Q * lam[:, None, :]) @ Q.transpose(1, 2)
        mats[int(n)] = (idx, 0.5 * (A + A.transpose(1, 2)))
    rhs = [rng.standard_normal(int(n)) for n in ns]
    return ns, mats, rhs


def _memsize_dmat(m, n):
    """blasfeo_memsize_dmat (auxiliary/d_aux_lib4.c:1519): pm*cn + dA rounded to 16, in bytes, 64-byte rounded."""
    pm, cn = (m + 3) // 4 * 4, (n + 3) // 4 * 4
    return ((pm * cn + (min(m, n) + 15) // 16 * 16) * 8 + 63) // 64 * 64


class HostSystems:
    """The systems of gen_config3 in host memory, each matrix laid out as
    blasfeo_create_dmat lays it out (panel-major, panel size 4), with BLASFEO
    descriptors for the CPU library."""

    def __init__(self, ns, mats, rhs):
        import torch
        from oracle.pyoracle import DMat, DVec
        self.ns = np.asarray(ns, dtype=np.int32)
        num = len(ns)
        size = {int(n): _memsize_dmat(int(n), int(n)) // 8 for n in np.unique(self.ns)}
        offs = np.zeros(num, dtype=np.int64)
        acc = 0
        for i, n in enumerate(self.ns):
            offs[i] = acc
            acc += size[int(n)]
        # the reference's AVX kernels need 64-byte aligned panel-major storage
        from oracle.pyoracle import _aligned_zeros
        self.slab = _aligned_zeros(acc + 8, np.float64)
        for n, (idx, X) in mats.items():
            pm = (n + 3) // 4 * 4
            pad = torch.zeros((len(idx), pm, pm), dtype=torch.float64, device=X.device)
            pad[:, :n, :n] = X
            P = pad.reshape(len(idx), pm // 4, 4, pm).permute(0, 1, 3, 2).reshape(len(idx), pm * pm).cpu().numpy()
            for r, i in enumerate(idx):
                self.slab[offs[i]:offs[i] + pm * pm] = P[r]
        self.mats_by_n = mats
        vlen = (self.ns + 3) // 4 * 4
        voff = np.concatenate([[0], np.cumsum(vlen)[:-1]]).astype(np.int64)
        self.b = _aligned_zeros(int(vlen.sum()) + 4, np.float64)
        self.x = _aligned_zeros(int(vlen.sum()) + 4, np.float64)
        for i, r in enumerate(rhs):
            self.b[voff[i]:voff[i] + len(r)] = r
        self.rhs, self.voff = rhs, voff
        base, bb, xb = self.slab.ctypes.data, self.b.ctypes.data, self.x.ctypes.data
        A, bv, xv = (DMat * num)(), (DVec * num)(), (DVec * num)()
        for i, n in enumerate(self.ns):
            n = int(n)
            pm = (n + 3) // 4 * 4
            a = A[i]
            a.mem = a.pA = base + int(offs[i]) * 8
            a.dA = a.pA + pm * pm * 8
            a.m = a.n = n
            a.pm = a.cn = pm
            a.use_dA = 0
            a.memsize = size[n] * 8
            for v, p in ((bv[i], bb), (xv[i], xb)):
                v.mem = v.pa = p + int(voff[i]) * 8
                v.m, v.pm, v.memsize = n, pm, pm * 8
        self.A, self.bv, self.xv = A, bv, xv
        self.nvec = (C.c_int * num)(*[int(v) for v in self.ns])
        self.num = num

    def backward_error(self, i):
        n = int(self.ns[i])
        idx, X = self.mats_by_n[n]
        a = X[int(np.nonzero(idx == i)[0][0])].cpu().numpy()
        x = self.x[self.voff[i]:self.voff[i] + n]
        b = self.rhs[i]
        return float(np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max()))


class CpuRun:
    """The reference's CPU path (dpotrf_l + dtrsv_lnn + dtrsv_ltn per system,
    oracle/cpu_bench.c) over HostSystems with P threads on P physical cores."""

    def __init__(self, systems):
        self.lib, self.prefix, self.kind, self.name = cpu_library()
        self.drv = cpu_driver()
        self.sys = systems
        f = lambda s: C.cast(getattr(self.lib, self.prefix + s), C.c_void_p)
        self.fp = (f("potrf_l"), f("trsv_lnn"), f("trsv_ltn"))
        self.cpus = physical_cpus()

    def run(self, threads):
        S = self.sys
        old = os.sched_getaffinity(0)
        os.sched_setaffinity(0, self.cpus[:max(1, threads)])
        try:
            return self.drv.cpu_posv_batch(threads, S.num, int(S.ns.max()), S.nvec, S.A, S.bv, S.xv, *self.fp)
        finally:
            os.sched_setaffinity(0, old)

    def check(self, k=8):
        return max(self.sys.backward_error(i) for i in range(0, self.sys.num, max(1, self.sys.num // k)))


DESC_DTYPE_CPU = np.dtype([("mem", "<u8"), ("pA", "<u8"), ("dA", "<u8"), ("m", "<i4"), ("n", "<i4"),
                           ("pm", "<i4"), ("cn", "<i4"), ("use_dA", "<i4"), ("memsize", "<i4")])


def cpu_driver():
    d = os.path.join(ROOT, "oracle")
    so = os.path.join(d, "libcpu_bench.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", d, "cpubench"], check=True)
    drv = C.CDLL(so)
    for f in ("cpu_posv_batch", "cpu_chain_batch", "cpu_ric_trf_batch"):
        getattr(drv, f).restype = C.c_double
    drv.cpu_chain_batch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double] + [C.c_void_p, C.c_longlong] * 7 + \
        [C.c_void_p] * 5
    drv.cpu_ric_trf_batch.argtypes = [C.c_int] * 5 + [C.c_void_p, C.c_longlong] * 3 + [C.c_void_p] * 3
    return drv


def cpu_baseline(systems, passes=5, p1_passes=3, warmup=3):
    """Median wall time of `passes` passes over all systems with one thread per
    physical core (after `warmup` passes, as the reference arm), and of
    `p1_passes` passes on one core."""
    cr = CpuRun(systems)
    P = len(cr.cpus)
    for _ in range(warmup):
        cr.run(P)
    tp = float(np.median([cr.run(P) for _ in range(passes)]))
    t1 = float(np.median([cr.run(1) for _ in range(p1_passes)]))
    n = systems.num
    return {"value": n / tp, "unit": UNIT, "cores": P, "kind": cr.kind,
            "sample": "the same %d systems as the GPU arm (seed 1000), %s, dpotrf_l+dtrsv_lnn+dtrsv_ltn per system, "
                      "one thread per physical core (%d of %d logical CPUs), median of %d passes after 3 warm-up passes; worst sampled "
                      "backward error %.1e" % (n, cr.name, P, len(os.sched_getaffinity(0)), passes, cr.check()),
            "p1": {"value": n / t1, "cores": 1, "sample": "same systems, one core, median of %d passes" % p1_passes},
            "ms_per_pass": 1e3 * tp}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0"))) if torch.cuda.is_available() else "cpu"
    # the GPU arm's systems (seed 1000 for rank 0); the device only generates them
    systems = HostSystems(*gen_config3(args.num, 1000, dev))
    cr = CpuRun(systems)
    P = len(cr.cpus)
    for _ in range(args.warmup):
        cr.run(P)
    ts = [cr.run(P) for _ in range(args.steps)]
    total = float(np.sum(ts))
    val = args.num * args.steps / total
    t1 = float(np.median([cr.run(1) for _ in range(2)]))
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "systems": args.num, "seed": 1000, "library": cr.name,
                       "same_systems_as_gpu_arm": True},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": P, "kind": cr.kind,
                             "sample": "all %d systems per step (the GPU arm's, seed 1000), %s, one thread per "
                                       "physical core; median pass %.1f ms; worst sampled backward error %.1e"
                                       % (args.num, cr.name, 1e3 * float(np.median(ts)), cr.check()),
                             "p1": {"value": args.num / t1, "cores": 1}},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampler over the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        mhz = [float(s[0]) for s in self.samples if len(s) >= 7 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 7 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples if len(s) >= 7 for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def main():
    args = parse()
    if args.case:
        return run_case(args.case)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    import blasfeo_b200 as bf
    from blasfeo_b200.workloads import SpdBatch
    lib = bf.lib
    P = lambda t: C.c_void_p(t.data_ptr())
    dev = torch.device("cuda", local)
    systems = gen_config3(args.num, rank_seed(rank), dev)
    W = SpdBatch(*systems, device=dev)
    # the CPU baseline solves the very same systems from host memory
    host_sys = HostSystems(*systems) if (rank == 0 and world == 1 and not args.no_cpu) else None
    del systems
    info = torch.zeros(args.num, dtype=torch.int32, device=dev)
    iters = torch.zeros(args.num, dtype=torch.int32, device=dev)
    berr = torch.zeros(args.num, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = C.c_void_p(stream.cuda_stream)

    def mixed():
        return lib.blasfeo_dsposv_l_vbatch(args.num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), MAX_ITER,
                                           TOL, P(iters), P(berr), P(info), None, 0, sh)

    def plain():
        return lib.blasfeo_dposv_l_vbatch(args.num, P(W.nvec), W.max_n, P(W.desc), P(W.bdesc), P(W.xdesc), P(info),
                                          None, 0, sh)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            bf.check(fn())
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return reduce_max_ms(e0.elapsed_time(e1) / steps, world, dist, dev)

    # ---- correctness gate (not timed): every system at FP64-level residual ----
    bf.check(mixed())
    torch.cuda.synchronize()
    inf_ = info.cpu().numpy()
    be = berr.cpu().numpy()
    it = iters.cpu().numpy()
    ok_mixed = bool((inf_ == 0).all() and (be <= TOL).all())
    rng = np.random.default_rng(rank)
    worst = 0.0
    for i in rng.choice(args.num, size=min(16, args.num), replace=False):
        a, b, x = W.matrix(i), W.rhs[i], W.solution(i)
        worst = max(worst, np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max()))
    bf.check(plain())
    torch.cuda.synchronize()
    ok_plain = bool((info.cpu().numpy() == 0).all())
    worst_plain = 0.0
    for i in rng.choice(args.num, size=min(16, args.num), replace=False):
        a, b, x = W.matrix(i), W.rhs[i], W.solution(i)
        worst_plain = max(worst_plain, np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max()))
    if not ok_mixed or worst > TOL or worst_plain > TOL:
        print("residual gate failed: mixed ok=%s (max berr %.2e, sampled %.2e), plain ok=%s (sampled %.2e)"
              % (ok_mixed, be.max(), worst, ok_plain, worst_plain), file=sys.stderr)
        return 2

    # ---- timed: mixed (headline value) and plain FP64 ----
    clk = Clocks(local)
    clk.start()
    time.sleep(0.3)
    ms_mixed = timed(mixed, args.steps, args.warmup)
    ms_plain = timed(plain, args.steps, args.warmup)
    clocks = clk.stop()
    nclass = 9  # classify + size classes (upper bound of launches per call)
    value = aggregate_value(world, args.num, ms_mixed)
    plain_value = aggregate_value(world, args.num, ms_plain)

    # ---- e2e: everything in pinned host memory, kernels read it over the host link ----
    e2e = None
    try:
        e2e = run_e2e(args, W, lib, torch, dev, stream, barrier, world)
    except Exception as ex:  # reported, never silently replaced
        e2e = {"value": None, "unit": UNIT, "error": repr(ex)}

    peak_bw = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_bw = float(json.load(f)["hbm_gbs"])
        peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        peak_bw = 6650.0
        peak_src = "fallback 6.65 TB/s"
    fp32_peak = lib.blasfeo_b200_measure_fma_peak(b"s"[0], 4096)
    fp64_peak = lib.blasfeo_b200_measure_fma_peak(b"d"[0], 2048)
    bytes_pass = W.lower_bytes()
    flops = W.chol_flops()
    achieved = bytes_pass / (ms_mixed * 1e-3) / 1e9
    # DRAM bytes of one call: ncu capture of the same call on 2,000 systems of
    # this distribution (summary under profiles/, k_posv_f32_cfg3_2000_dram):
    # 185,359,872 B of DRAM traffic against 178,497,336 algorithmic bytes,
    # scaled to this call by its algorithmic bytes
    traffic = bytes_pass * (185359872.0 / 178497336.0)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak_bw, "unit": "GB/s", "frac": achieved / peak_bw,
                "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same "
                "call on 2,000 systems of the distribution, scaled by algorithmic bytes (ratio 1.038)",
                "peak_source": peak_src,
                "kernel": "k_posv<float,true> (all size classes of one blasfeo_dsposv_l_vbatch call)",
                "algorithmic_bytes_per_launch": bytes_pass,
                "fp32_simt": {"achieved_gflops": flops / (ms_mixed * 1e-3) / 1e9, "peak_gflops": fp32_peak,
                              "frac": flops / (ms_mixed * 1e-3) / 1e9 / fp32_peak if fp32_peak > 0 else None}}
    plain_roof = {"achieved_gflops": flops / (ms_plain * 1e-3) / 1e9, "fp64_peak_gflops": fp64_peak,
                  "frac": flops / (ms_plain * 1e-3) / 1e9 / fp64_peak if fp64_peak > 0 else None,
                  "hbm_frac": bytes_pass / (ms_plain * 1e-3) / 1e9 / peak_bw}
    fp64 = None
    if not args.no_fp64:
        try:
            fp64 = fp64_batched(lib, torch, dev, stream, fp64_peak, peak_bw)
        except Exception as ex:  # reported, never silently replaced
            fp64 = {"error": repr(ex)}
    others = None
    if not args.no_fp64:
        try:
            others = other_configs(lib, torch, dev, stream, peak_bw, cpu=(rank == 0 and not args.no_cpu))
        except Exception as ex:  # reported, never silently replaced
            others = {"error": repr(ex)}
    single = None
    if not args.no_fp64 and rank == 0:
        try:
            single = single_dropin(torch, stream, fp64_peak, peak_bw)
        except Exception as ex:  # reported, never silently replaced
            single = {"error": repr(ex)}
        if not args.no_cpu:
            try:
                single["cpu_reference"] = cpu_single_dropin()
            except Exception as ex:
                single["cpu_reference"] = {"error": repr(ex)}
    dispatch = None
    if not args.no_fp64 and rank == 0:
        try:
            dispatch = learned_dispatch(cpu=not args.no_cpu)
        except Exception as ex:  # reported, never silently replaced
            dispatch = {"error": repr(ex)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(host_sys)
        except Exception as ex:
            cpu = {"value": None, "error": repr(ex)}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 factor + f64 refinement", "data": "synthetic",
            "config": {"workload": WORKLOAD, "systems_per_gpu": args.num, "max_iter": MAX_ITER, "tol": TOL,
                       "l2": "inputs larger than L2 (%.2f GB FP64 matrices per GPU vs 126 MB L2)" % (W.total_bytes / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_plain, "roofline": plain_roof},
            "mixed_vs_plain": value / plain_value,
            "refinement": {"mean_steps": float(it.mean()), "max_steps": int(it.max()), "max_berr": float(be.max()),
                           "sampled_host_residual": worst, "sampled_host_residual_plain": worst_plain},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "fp64_batched": fp64,
            "fused_kernels": others, "single_dropin": single, "learned_dispatch": dispatch,
            "gpu_launches": (args.steps * nclass) * 2}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def fp64_batched(lib, torch, dev, stream, fp64_peak, peak_bw, sizes=(64, 128, 256)):
    """Plain FP64 batched dgemm_nt (D = A B^T, beta = 0) and dpotrf_l on uniform
    batches larger than L2, per size: GFLOP/s (LAPACK flop counts), fraction of
    the measured FP64 FMA peak and of the roofline min(peak, AI * HBM) with
    algorithmic bytes = inputs read once + outputs written once (gemm: A, B, D;
    potrf: lower triangle in and out)."""
    from blasfeo_b200.workloads import fp64_roofline_batches
    sh = C.c_void_p(stream.cuda_stream)
    out = {"peak_gflops": fp64_peak, "peak_source": "blasfeo_b200_measure_fma_peak('d'), same run", "hbm_gbs": peak_bw}

    def tm(fn, reps=5):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for n in sizes:
        w = fp64_roofline_batches(n, device=dev)
        bg, A, B, D = w["gemm"]
        ms = tm(lambda: lib.blasfeo_dgemm_nt_batch(bg, n, n, n, 1.0, A.ref, 0, 0, B.ref, 0, 0, 0.0, D.ref, 0, 0, D.ref,
                                                   0, 0, sh))
        fl, by = 2.0 * n ** 3 * bg, 3.0 * n * n * 8 * bg
        g = fl / ms / 1e6
        roof = min(fp64_peak, fl / by * peak_bw)
        out["dgemm_nt_n%d" % n] = {"batch": bg, "ms": ms, "gflops": g, "frac_of_peak": g / fp64_peak,
                                   "roofline_gflops": roof, "frac_of_roofline": g / roof}
        bp, Cm, L = w["potrf"]
        info = torch.zeros(bp, dtype=torch.int32, device=dev)
        ms = tm(lambda: lib.blasfeo_dpotrf_l_batch(bp, n, Cm.ref, 0, 0, L.ref, 0, 0, C.c_void_p(info.data_ptr()), sh))
        torch.cuda.synchronize()
        if not bool((info == 0).all().item()):
            raise RuntimeError("dpotrf_l batch reported a non-positive pivot at n=%d" % n)
        fl, by = (n ** 3 / 3.0 + n * n / 2.0 + n / 6.0) * bp, 2.0 * n * (n + 1) / 2 * 8 * bp
        g = fl / ms / 1e6
        roof = min(fp64_peak, fl / by * peak_bw)
        out["dpotrf_l_n%d" % n] = {"batch": bp, "ms": ms, "gflops": g, "frac_of_peak": g / fp64_peak,
                                   "roofline_gflops": roof, "frac_of_roofline": g / roof}
        del w, A, B, D, Cm, L
        torch.cuda.empty_cache()
    return out


SINGLE_N = 64


def _single_inputs():
    """Config 1 inputs, seed 0: A, B 64x64 ~ U[-1,1]; S = G G^T / 64 + I with
    G ~ N(0,1); R 64x64 ~ N(0,1), the trsm right-hand side."""
    import numpy as np
    n = SINGLE_N
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, (n, n))
    B = rng.uniform(-1, 1, (n, n))
    G = rng.standard_normal((n, n))
    S = G @ G.T / n + np.eye(n)
    R = rng.standard_normal((n, n))
    return A, B, S, R


def single_dropin(torch, stream, fp64_peak, peak_bw):
    """Config 1: one 64x64 instance per call through the single-instance C ABI
    (device-resident panel-major matrices): dgemm_nt 64x64x64 (alpha 1, beta 0),
    dpotrf_l of S, dtrsm_rltn of R with that factor (which reuses the cached
    inverse diagonal).  Microseconds per call: back-to-back asynchronous calls
    timed with CUDA events (device time plus launch; the calls are made from
    Python through ctypes), the same calls each synchronised (what a caller with
    CPU semantics waits), and the three calls as one CUDA graph replay.  For
    form: flops, algorithmic bytes and the roofline time max(flops / FP64 peak,
    bytes / HBM bandwidth) of each call."""
    import blasfeo_b200 as bf
    from blasfeo_b200.api import DMat
    n = SINGLE_N
    A, B, S, R = _single_inputs()
    dA, dB, dS, dL, dR, dX, dD = (DMat(n, n).pack(M) for M in (A, B, S, S, R, R, A))
    lib = bf.lib
    ref = lambda M: M.ref
    calls = {
        "dgemm_nt_64": lambda: lib.blasfeo_dgemm_nt(n, n, n, 1.0, ref(dA), 0, 0, ref(dB), 0, 0, 0.0, ref(dD), 0, 0,
                                                    ref(dD), 0, 0),
        "dpotrf_l_64": lambda: lib.blasfeo_dpotrf_l(n, ref(dS), 0, 0, ref(dL), 0, 0),
        "dtrsm_rltn_64": lambda: lib.blasfeo_dtrsm_rltn(n, n, 1.0, ref(dL), 0, 0, ref(dR), 0, 0, ref(dX), 0, 0),
    }
    work = {"dgemm_nt_64": (2.0 * n ** 3, 3 * n * n * 8),
            "dpotrf_l_64": (n ** 3 / 3 + n * n / 2 + n / 6, 2 * n * n * 8),
            "dtrsm_rltn_64": (float(n ** 3), 3 * n * n * 8)}
    bf.set_stream(stream)
    out = {"n": n}
    reps = 2000
    try:
        for name, f in calls.items():
            bf.set_sync(False)
            for _ in range(50):
                f()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                f()
            e1.record(stream)
            torch.cuda.synchronize()
            us_async = e0.elapsed_time(e1) * 1e3 / reps
            bf.set_sync(True)
            t0 = time.perf_counter()
            for _ in range(reps // 4):
                f()
            us_sync = (time.perf_counter() - t0) * 1e6 / (reps // 4)
            fl, by = work[name]
            roof_us = max(fl / (fp64_peak * 1e9), by / (peak_bw * 1e9)) * 1e6
            out[name] = {"us_async": us_async, "us_sync": us_sync, "flops": fl, "bytes": by,
                         "flop_per_byte": fl / by, "roofline_us": roof_us,
                         "gflops_async": fl / (us_async * 1e-6) / 1e9}
            assert lib.blasfeo_b200_last_error() == 0
        # the three calls (factor, solve, update) as one graph
        bf.set_sync(False)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        with torch.cuda.graph(g, stream=cap, capture_error_mode="relaxed"):
            bf.set_stream(cap)
            for f in calls.values():
                f()
        bf.set_stream(stream)
        for _ in range(20):
            g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        out["graph_3calls_us"] = e0.elapsed_time(e1) * 1e3 / reps
        del g
        # the measured floor: the same timing of an empty kernel launched from
        # Python, and the potrf through every kernel variant of the batched
        # routine with one instance (0-3: a CTA of 64-512 threads per instance,
        # 4: global memory, 5: one warp on the FP64 tensor cores)
        def tm_async(f, r=reps):
            for _ in range(50):
                f()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(r):
                f()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) * 1e3 / r
        with torch.cuda.stream(stream):
            out["empty_kernel_us"] = tm_async(lambda: torch.cuda._sleep(0))
        from blasfeo_b200.api import descriptor_array
        arrS, arrL = descriptor_array([dS]), descriptor_array([dL])
        nv = torch.tensor([n], dtype=torch.int32, device=dS.buf.device)
        sh = C.c_void_p(stream.cuda_stream)
        out["dpotrf_l_64_by_variant_us"] = {
            str(v): tm_async(lambda: lib.blasfeo_dpotrf_l_vbatch_variant(1, C.c_void_p(nv.data_ptr()), n,
                                                                         C.c_void_p(arrS.data_ptr()),
                                                                         C.c_void_p(arrL.data_ptr()), None, v, sh))
            for v in range(int(lib.blasfeo_b200_num_variants(1)))}
    finally:
        bf.set_sync(True)
        bf.set_stream(None)
    return out


def cpu_single_dropin(reps=2000):
    """Config 1 on the host: the same three calls through the compiled reference
    (BLASFEO HP, Haswell build, one core), microseconds per call."""
    import numpy as np
    from oracle.pyoracle import Api, HostMat, ref_available
    kind = "reference" if ref_available("haswell") else "port"
    api = Api("hp", "haswell") if kind == "reference" else Api("oracle")
    n = SINGLE_N
    A, B, S, R = _single_inputs()
    hA, hB, hS, hR = (HostMat(n, n).set(M) for M in (A, B, S, R))
    hD, hL, hX = HostMat(n, n), HostMat(n, n), HostMat(n, n)
    calls = {
        "dgemm_nt_64": lambda: api.gemm_nt("d", n, n, n, 1.0, hA, 0, 0, hB, 0, 0, 0.0, hD, 0, 0, hD, 0, 0),
        "dpotrf_l_64": lambda: api.potrf_l("d", n, hS, 0, 0, hL, 0, 0),
        "dtrsm_rltn_64": lambda: api.trsm_rltn("d", n, n, 1.0, hL, 0, 0, hR, 0, 0, hX, 0, 0),
    }
    out = {"kind": kind, "cores": 1}
    for name, f in calls.items():
        for _ in range(50):
            f()
        t0 = time.perf_counter()
        for _ in range(reps):
            f()
        out[name + "_us"] = (time.perf_counter() - t0) * 1e6 / reps
    return out


def other_configs(lib, torch, dev, stream, peak_bw, cpu=True):
    """The two fused HBM-bound kernels on their own workloads (seeded, inputs
    larger than L2), per instance: algorithmic bytes (inputs read once, outputs
    written once) and flops as in the design record.
      chain:    100,000 instances, n = 16: S = A A^T + 16 I (A 16x32), L = chol(S),
                X = R L^-T, D = C - X G^T (R, C, G 16x16 ~ N(0,1)); one launch on
                batch-interleaved slabs (the leg's number; also replayed as a
                CUDA graph), the back-to-back kernel on the same instances beside;
      riccati:  4,096 problems, N = 30, nx = 12, nu = 4, A = I + 0.1 N(0,1) scaled
                to spectral radius 0.95, B ~ N(0,1)/sqrt(nx), Q = I, R = I, S = 0,
                P_N = I; the whole backward factorization in one launch, FP64 and FP32."""
    import numpy as np
    from blasfeo_b200.api import DMatBatch, SMatBatch
    from blasfeo_b200.workloads import fill_batch
    sh = C.c_void_p(stream.cuda_stream)
    g = torch.Generator(device=dev)
    g.manual_seed(2)

    def tm(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    nb = 100000
    slabs = {}
    for name, (r, c) in (("A", (16, 32)), ("R", (16, 16)), ("C", (16, 16)), ("G", (16, 16))):
        slabs[name] = DMatBatch(r, c, nb)
        fill_batch(slabs[name], torch.randn((nb, r, c), generator=g, dtype=torch.float64, device=dev))
    L, X, D = DMatBatch(16, 16, nb), DMatBatch(16, 16, nb), DMatBatch(16, 16, nb)
    info = torch.zeros(nb, dtype=torch.int32, device=dev)
    ms = tm(lambda: lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(nb, 16, 32, 16.0, slabs["A"].ref, slabs["R"].ref,
                                                             slabs["C"].ref, slabs["G"].ref, L.ref, X.ref, D.ref,
                                                             C.c_void_p(info.data_ptr()), sh))
    if not bool((info == 0).all().item()):
        raise RuntimeError("chain reported a non-positive pivot")
    by, fl = 15424.0 * nb, 22.8e3 * nb
    out["chain_n16"] = {"instances": nb, "ms": ms, "instances_per_s": nb / ms * 1e3, "gbs": by / ms / 1e6,
                        "frac_of_hbm": by / ms / 1e6 / peak_bw, "gflops": fl / ms / 1e6,
                        "bytes_per_instance": 15424, "flops_per_instance": 22.8e3}
    if cpu:
        try:
            out["chain_n16"]["cpu_reference"] = cpu_chain_leg(nb, slabs, L, X, D)
        except Exception as ex:  # reported, never silently replaced
            out["chain_n16"]["cpu_reference"] = {"error": repr(ex)}
    # the configuration's layout is the batch-interleaved one: its kernel is the
    # leg's number, the back-to-back kernel on the same instances beside it
    try:
        il = chain_interleaved(lib, torch, stream, peak_bw, tm, nb, slabs, L, X, D, ms)
        b2b = {k: out["chain_n16"].pop(k) for k in ("ms", "instances_per_s", "gbs", "frac_of_hbm", "gflops")}
        out["chain_n16"].update({"layout": "batch-interleaved (blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il)",
                                 "ms": il["ms"], "instances_per_s": il["instances_per_s"], "gbs": il["gbs"],
                                 "frac_of_hbm": il["frac_of_hbm"], "gflops": fl / il["ms"] / 1e6,
                                 "graph_replay_ms": il.get("graph_replay_ms"),
                                 "relfro_vs_back_to_back_first_2000": il["relfro_vs_back_to_back_first_2000"],
                                 "back_to_back": dict(b2b, kernel="blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch"),
                                 "speedup_vs_back_to_back": il["speedup_vs_back_to_back"]})
    except Exception as ex:  # reported, never silently replaced
        out["chain_n16"]["interleaved"] = {"error": repr(ex)}
    del slabs, L, X, D
    torch.cuda.empty_cache()
    try:
        out["potrf_n16_layouts"] = potrf_layouts(lib, torch, dev, stream, peak_bw, g, tm)
    except Exception as ex:  # reported, never silently replaced
        out["potrf_n16_layouts"] = {"error": repr(ex)}

    nbt, N, nx, nu = 4096, 30, 12, 4
    out.update(riccati_legs(lib, torch, dev, stream, peak_bw, g, tm, nbt, N, nx, nu, cpu))
    torch.cuda.empty_cache()
    return out


def chain_interleaved(lib, torch, stream, peak_bw, tm, nb, slabs, L, X, D, ms_b2b):
    """The same 100,000 chain instances on batch-interleaved slabs
    (blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il, a quad of lanes per instance);
    the conversions happen outside the timed region.  Same algorithmic bytes
    as the back-to-back leg; outputs compared with the back-to-back call's."""
    import numpy as np
    from blasfeo_b200.api import DMatBatch, DMatBatchIL
    sh = C.c_void_p(stream.cuda_stream)
    ins = [DMatBatchIL(slabs[n].m, slabs[n].n, nb).from_batch(slabs[n], sh) for n in "ARCG"]
    outs = [DMatBatchIL(16, 16, nb) for _ in range(3)]
    info = torch.zeros(nb, dtype=torch.int32, device=ins[0].buf.device)
    call_on = lambda h: lib.blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il(nb, 16, 32, 16.0, *(x.ref for x in ins),
                                                                      *(x.ref for x in outs),
                                                                      C.c_void_p(info.data_ptr()), h)
    ms = tm(lambda: call_on(sh))
    # the same launch captured in a CUDA graph (on a stream of its own: the
    # legacy stream cannot be captured) and replayed on the leg's stream
    try:
        cap = torch.cuda.Stream()
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=cap, capture_error_mode="relaxed"):
            call_on(C.c_void_p(cap.cuda_stream))
        with torch.cuda.stream(stream):
            graph_ms = tm(gr.replay)
        del gr
    except Exception as ex:  # reported beside the direct launch
        graph_ms = {"error": repr(ex)}
    if not bool((info == 0).all().item()):
        raise RuntimeError("interleaved chain reported a non-positive pivot")
    diff = {}
    for name, il, ref in (("L", outs[0], L), ("X", outs[1], X), ("D", outs[2], D)):
        back = il.to_batch(DMatBatch(16, 16, nb), sh)
        torch.cuda.synchronize()
        a_, b_ = back.unpack_all()[:2000], ref.unpack_all()[:2000]
        if name == "L":
            a_, b_ = np.tril(a_), np.tril(b_)
        diff[name] = float(np.linalg.norm(a_ - b_) / np.linalg.norm(b_))
    by = 15424.0 * nb
    return {"ms": ms, "instances_per_s": nb / ms * 1e3, "gbs": by / ms / 1e6, "frac_of_hbm": by / ms / 1e6 / peak_bw,
            "speedup_vs_back_to_back": ms_b2b / ms, "relfro_vs_back_to_back_first_2000": diff,
            "graph_replay_ms": graph_ms}


def potrf_layouts(lib, torch, dev, stream, peak_bw, g, tm, nb=100000, n=16):
    """potrf_l of 100,000 SPD 16 x 16 instances (the factor step of the n = 16
    chain, S = A A^T + 16 I with A 16 x 32 ~ N(0,1)) on the back-to-back slab
    (blasfeo_dpotrf_l_batch: one warp per instance, FP64 tensor cores) and on the
    batch-interleaved slab (blasfeo_dpotrf_l_batch_il: a lane pair per instance);
    algorithmic bytes = lower triangle in and out plus the inverse diagonal."""
    from blasfeo_b200.api import DMatBatch, DMatBatchIL
    from blasfeo_b200.workloads import fill_batch
    A = torch.randn((nb, n, 2 * n), generator=g, dtype=torch.float64, device=dev)
    S = A @ A.transpose(1, 2) + n * torch.eye(n, dtype=torch.float64, device=dev)
    C0, D0 = DMatBatch(n, n, nb), DMatBatch(n, n, nb)
    fill_batch(C0, S)
    Ci, Di = DMatBatchIL(n, n, nb).from_batch(C0), DMatBatchIL(n, n, nb)
    sh = C.c_void_p(stream.cuda_stream)
    ms_b = tm(lambda: lib.blasfeo_dpotrf_l_batch(nb, n, C0.ref, 0, 0, D0.ref, 0, 0, None, sh))
    ms_i = tm(lambda: lib.blasfeo_dpotrf_l_batch_il(nb, n, Ci.ref, Di.ref, None, sh))
    out = DMatBatch(n, n, nb)
    Di.to_batch(out)
    torch.cuda.synchronize()
    a_, b_ = np.tril(out.unpack_all()), np.tril(D0.unpack_all())
    by = (2 * n * (n + 1) / 2 + n) * 8 * nb
    res = {"instances": nb}
    for name, ms in (("back_to_back", ms_b), ("interleaved", ms_i)):
        res[name] = {"ms": ms, "instances_per_s": nb / ms * 1e3, "gbs": by / ms / 1e6, "frac_of_hbm": by / ms / 1e6 / peak_bw}
    res["winner"] = "interleaved" if ms_i < ms_b else "back_to_back"
    res["relfro_between_layouts"] = float(np.linalg.norm(a_ - b_) / np.linalg.norm(b_))
    return res


def riccati_interleaved(lib, torch, sh, peak_bw, tm, nbt, N, nx, nu, BAs, RSQ, L_b2b, ms_b2b):
    """The FP64 factorization of the same problems on stage-major
    batch-interleaved slabs (blasfeo_dric_trf_batch_il, a quad of lanes per
    problem; stage k of problem b at instance k * bs + b); conversions outside
    the timed region; factors compared with the back-to-back call's."""
    import numpy as np
    from blasfeo_b200.api import DMatBatch, DMatBatchIL
    from blasfeo_b200.workloads import fill_batch
    dev = BAs.device
    bs = (nbt + 15) // 16 * 16
    ba = torch.zeros((N * bs, 16, nx), dtype=torch.float64, device=dev)
    ba.view(N, bs, 16, nx)[:, :nbt] = BAs.reshape(nbt, N, 16, nx).transpose(0, 1)
    rsq = torch.zeros(((N + 1) * bs, 16, 16), dtype=torch.float64, device=dev)
    rsq.view(N + 1, bs, 16, 16)[:, :nbt] = RSQ.reshape(nbt, N + 1, 16, 16).transpose(0, 1)
    tBA, tRSQ = DMatBatch(16, nx, N * bs), DMatBatch(16, 16, (N + 1) * bs)
    fill_batch(tBA, ba.contiguous())
    fill_batch(tRSQ, rsq.contiguous())
    iBA, iRSQ = DMatBatchIL(16, nx, N * bs).from_batch(tBA, sh), DMatBatchIL(16, 16, (N + 1) * bs).from_batch(tRSQ, sh)
    iL = DMatBatchIL(16, 16, (N + 1) * bs)
    info = torch.zeros(nbt, dtype=torch.int32, device=dev)
    ms = tm(lambda: lib.blasfeo_dric_trf_batch_il(nbt, N, nx, nu, iBA.ref, iRSQ.ref, iL.ref, C.c_void_p(info.data_ptr()),
                                                  sh))
    if not bool((info == 0).all().item()):
        raise RuntimeError("interleaved Riccati factorization reported a non-positive pivot")
    back = iL.to_batch(DMatBatch(16, 16, (N + 1) * bs), sh)
    torch.cuda.synchronize()
    Lil = back.unpack_all().reshape(N + 1, bs, 16, 16)[:, :nbt].transpose(1, 0, 2, 3)
    m = nu + nx  # the written blocks: m x m at stages < N, nx x nx at stage N
    a_ = np.concatenate([np.tril(Lil[:, :N, :m, :m]).ravel(), np.tril(Lil[:, N, :nx, :nx]).ravel()])
    b_ = np.concatenate([np.tril(L_b2b[:, :N, :m, :m]).ravel(), np.tril(L_b2b[:, N, :nx, :nx]).ravel()])
    by = (16 * nx + 16 * 16 + 136) * 8 * N * nbt
    return {"ms": ms, "problems_per_s": nbt / ms * 1e3, "gbs": by / ms / 1e6, "frac_of_hbm": by / ms / 1e6 / peak_bw,
            "speedup_vs_back_to_back": ms_b2b / ms,
            "relfro_vs_back_to_back": float(np.linalg.norm(a_ - b_) / np.linalg.norm(b_))}


def riccati_legs(lib, torch, dev, stream, peak_bw, g, tm, nbt, N, nx, nu, cpu):
    """Config 4: 4,096 LQR problems, N = 30, nx = 12, nu = 4; A = I + 0.1 N(0,1)
    scaled to spectral radius 0.95, B ~ N(0,1)/sqrt(nx), Q = R = I, S = 0,
    P_N = I; for the solves, linear terms rq_k ~ N(0,1), b_k ~ N(0,1).
      riccati_d_N30 / riccati_s_N30: the backward factorization in one launch
        (FP64 / FP32);
      lq_solve_d_N30: FP64 factorization + Riccati solve (ux_k, pi_k);
      lq_solve_mixed_N30: FP32 factorization + FP64 refinement on the KKT residual;
    errors of P_0, K_k (all stages) and of the refined solution against the
    FP64 reference (the compiled reference's factors when the CPU leg runs,
    else this library's FP64 factors)."""
    from blasfeo_b200.api import DMatBatch, SMatBatch
    from blasfeo_b200.workloads import fill_batch
    P = lambda t: C.c_void_p(t.data_ptr())
    sh = C.c_void_p(stream.cuda_stream)
    out = {}
    A = torch.eye(nx, dtype=torch.float64, device=dev) + 0.1 * torch.randn((nbt, nx, nx), generator=g,
                                                                          dtype=torch.float64, device=dev)
    rho = torch.linalg.eigvals(A.cpu()).abs().max(dim=1).values.to(dev)
    A = A * (0.95 / rho)[:, None, None]
    B = torch.randn((nbt, nx, nu), generator=g, dtype=torch.float64, device=dev) / np.sqrt(nx)
    BA = torch.zeros((nbt, 16, nx), dtype=torch.float64, device=dev)
    BA[:, :nu] = B.transpose(1, 2)
    BA[:, nu:nu + nx] = A.transpose(1, 2)
    BAs = BA[:, None].expand(nbt, N, 16, nx).reshape(nbt * N, 16, nx)
    RSQ = torch.eye(16, dtype=torch.float64, device=dev).expand(nbt * (N + 1), 16, 16)
    m = nx + nu
    b = torch.zeros((nbt, N, 16), dtype=torch.float64, device=dev)
    b[:, :, :nx] = torch.randn((nbt, N, nx), generator=g, dtype=torch.float64, device=dev)
    rq = torch.zeros((nbt, N + 1, 16), dtype=torch.float64, device=dev)
    rq[:, :N, :m] = torch.randn((nbt, N, m), generator=g, dtype=torch.float64, device=dev)
    rq[:, N, :nx] = torch.randn((nbt, nx), generator=g, dtype=torch.float64, device=dev)
    Ls = {}
    slabs = {}
    for prec, Bt, dt in (("d", DMatBatch, torch.float64), ("s", SMatBatch, torch.float32)):
        sBA, sRSQ, sL = Bt(16, nx, nbt * N), Bt(16, 16, nbt * (N + 1)), Bt(16, 16, nbt * (N + 1))
        fill_batch(sBA, BAs.to(dt).contiguous())
        fill_batch(sRSQ, RSQ.to(dt).contiguous())
        info = torch.zeros(nbt, dtype=torch.int32, device=dev)
        f = lib.blasfeo_dric_trf_batch if prec == "d" else lib.blasfeo_sric_trf_batch
        ms = tm(lambda: f(nbt, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, P(info), sh))
        if not bool((info == 0).all().item()):
            raise RuntimeError("Riccati factorization reported a non-positive pivot")
        esz = 8 if prec == "d" else 4
        by = (16 * nx + 16 * 16 + 136) * esz * N * nbt   # BAbt_k and RSQ_k in, lower L_k out per stage
        out["riccati_%s_N30" % prec] = {"problems": nbt, "ms": ms, "problems_per_s": nbt / ms * 1e3,
                                        "gbs": by / ms / 1e6, "frac_of_hbm": by / ms / 1e6 / peak_bw,
                                        "gflops": 7.1e3 * N * nbt / ms / 1e6}
        Ls[prec] = sL.unpack_all().reshape(nbt, N + 1, 16, 16)
        slabs[prec] = (sBA, sRSQ, sL)
    sBA, sRSQ, sL = slabs["d"]
    # the FP64 factorization's number is the faster layout's (stage-major
    # batch-interleaved slabs, bit-equal factors); the back-to-back kernel, whose
    # factors the error and CPU legs below use, beside it
    try:
        il = riccati_interleaved(lib, torch, sh, peak_bw, tm, nbt, N, nx, nu, BAs, RSQ, Ls["d"],
                                 out["riccati_d_N30"]["ms"])
        r = out["riccati_d_N30"]
        b2b = {k: r.pop(k) for k in ("ms", "problems_per_s", "gbs", "frac_of_hbm", "gflops")}
        r.update({"layout": "stage-major batch-interleaved (blasfeo_dric_trf_batch_il)", "ms": il["ms"],
                  "problems_per_s": il["problems_per_s"], "gbs": il["gbs"], "frac_of_hbm": il["frac_of_hbm"],
                  "gflops": 7.1e3 * N * nbt / il["ms"] / 1e6,
                  "relfro_vs_back_to_back": il["relfro_vs_back_to_back"],
                  "back_to_back": dict(b2b, kernel="blasfeo_dric_trf_batch"),
                  "speedup_vs_back_to_back": il["speedup_vs_back_to_back"]})
    except Exception as ex:  # reported, never silently replaced
        out["riccati_d_N30"]["interleaved"] = {"error": repr(ex)}
    if cpu:
        try:
            out["riccati_d_N30"]["cpu_reference"], Ls["ref"] = cpu_riccati_leg(nbt, N, nx, nu, sBA, sRSQ, sL)
        except Exception as ex:  # reported, never silently replaced
            out["riccati_d_N30"]["cpu_reference"] = {"error": repr(ex)}
    # FP64 factorization + solve
    bflat, rqflat = b.reshape(-1).contiguous(), rq.reshape(-1).contiguous()
    ux = torch.zeros(nbt * (N + 1) * 16, dtype=torch.float64, device=dev)
    pi = torch.zeros(nbt * N * 16, dtype=torch.float64, device=dev)
    info = torch.zeros(nbt, dtype=torch.int32, device=dev)

    def solve64():
        lib.blasfeo_dric_trf_batch(nbt, N, nx, nu, sBA.ref, sRSQ.ref, sL.ref, P(info), sh)
        return lib.blasfeo_dric_trs_batch(nbt, N, nx, nu, sBA.ref, sL.ref, P(bflat), 16, P(rqflat), 16, P(ux), 16,
                                          P(pi), 16, sh)
    ms64 = tm(solve64)
    ux64, pi64 = ux.clone(), pi.clone()
    ms_trs = tm(lambda: lib.blasfeo_dric_trs_batch(nbt, N, nx, nu, sBA.ref, sL.ref, P(bflat), 16, P(rqflat), 16,
                                                   P(ux), 16, P(pi), 16, sh))
    out["lq_solve_d_N30"] = {"problems": nbt, "ms": ms64, "problems_per_s": nbt / ms64 * 1e3, "trs_ms": ms_trs}
    # mixed: FP32 factorization + FP64 refinement
    iters = torch.zeros(nbt, dtype=torch.int32, device=dev)
    res = torch.zeros(nbt, dtype=torch.float64, device=dev)
    TOLR = 1e-13
    msm = tm(lambda: lib.blasfeo_dsric_sv_batch(nbt, N, nx, nu, sBA.ref, sRSQ.ref, P(bflat), 16, P(rqflat), 16, P(ux),
                                                16, P(pi), 16, 20, TOLR, P(iters), P(res), P(info), None, 0, sh))
    torch.cuda.synchronize()
    rel = lambda a_, b_: float((a_ - b_).norm().item() / b_.norm().item())
    out["lq_solve_mixed_N30"] = {
        "problems": nbt, "ms": msm, "problems_per_s": nbt / msm * 1e3, "vs_fp64_solve": ms64 / msm,
        "converged": bool((info == 0).all().item()), "tol_rel_kkt_residual": TOLR,
        "mean_refinement_steps": float(iters.double().mean().item()), "max_rel_kkt_residual": float(res.max().item()),
        "solution_relfro_vs_fp64": {"ux": rel(ux, ux64), "pi": rel(pi, pi64)}}
    ref = Ls.get("ref", Ls["d"])
    for prec in ("d", "s"):
        out["riccati_%s_N30" % prec]["error_vs_fp64_reference"] = riccati_errors(Ls[prec], ref, nx, nu, N)
    out["riccati_d_N30"]["error_reference"] = "compiled reference (CPU)" if "ref" in Ls else "this library's FP64"
    return out


def riccati_gains(L, nx, nu):
    """From a stage factor L = [[Luu, 0], [Lxu, Lxx]] (problems x 16 x 16):
    P = Lxx Lxx^T and K = -Luu^{-T} Lxu^T (the feedback u = K x)."""
    Luu, Lxu, Lxx = L[:, :nu, :nu], L[:, nu:nu + nx, :nu], L[:, nu:nu + nx, nu:nu + nx]
    P = np.tril(Lxx) @ np.transpose(np.tril(Lxx), (0, 2, 1))
    K = -np.linalg.solve(np.transpose(np.tril(Luu), (0, 2, 1)), np.transpose(Lxu, (0, 2, 1)))
    return P, K


def riccati_errors(L, ref, nx, nu, N):
    """Max over problems of the relative Frobenius error of P_0, and of K_k
    over all problems and stages k < N."""
    e = lambda a, b: float((np.linalg.norm(a - b, axis=(1, 2)) / np.linalg.norm(b, axis=(1, 2))).max())
    P, _ = riccati_gains(np.asarray(L[:, 0], dtype=np.float64), nx, nu)
    Pr, _ = riccati_gains(ref[:, 0], nx, nu)
    kerr = 0.0
    for k in range(N):
        _, K = riccati_gains(np.asarray(L[:, k], dtype=np.float64), nx, nu)
        _, Kr = riccati_gains(ref[:, k], nx, nu)
        kerr = max(kerr, e(K, Kr))
    return {"P0_relfro_max": e(P, Pr), "K_relfro_max_all_stages": kerr}


def _host_slab(B):
    """Host copy of a device uniform-batch slab (same layout, 64-byte aligned as
    the reference's AVX kernels need): (array, pointer to instance 0, stride)."""
    from oracle.pyoracle import _aligned_zeros
    src = B.buf.cpu().numpy().view(np.float64)
    h = _aligned_zeros(src.size, np.float64)
    h[:] = src
    off = (B.s.pA - B.buf.data_ptr()) // 8
    return h, h.ctypes.data + 8 * off, B.s.stride


def _cpu_times(fn, passes=5, p1_passes=3):
    cpus = physical_cpus()
    old = os.sched_getaffinity(0)
    try:
        os.sched_setaffinity(0, cpus)
        fn(len(cpus))
        tp = float(np.median([fn(len(cpus)) for _ in range(passes)]))
        os.sched_setaffinity(0, cpus[:1])
        t1 = float(np.median([fn(1) for _ in range(p1_passes)]))
    finally:
        os.sched_setaffinity(0, old)
    return len(cpus), tp, t1


def cpu_chain_leg(nb, slabs, L, X, D):
    """The n = 16 chain through the compiled reference (dsyrk_ln + ddiare +
    dpotrf_l + dtrsm_rltn + dgemm_nt per instance) on host copies of the GPU
    leg's input slabs; instances/s at P = all physical cores and P = 1, and the
    GPU results' relative error against the reference's."""
    lib, prefix, kind, name = cpu_library()
    drv = cpu_driver()
    f = lambda s_: C.cast(getattr(lib, prefix + s_), C.c_void_p)
    hin = {k: _host_slab(v) for k, v in slabs.items()}
    hout = {k: _host_slab(v) for k, v in (("L", L), ("X", X), ("D", D))}
    for h, _, _ in hout.values():
        h[:] = 0.0
    args = [hin[k][1:] for k in "ARCG"] + [hout[k][1:] for k in "LXD"]
    flat = [a for pr in args for a in pr]

    def run(P):
        return drv.cpu_chain_batch(P, nb, 32, 16.0, *flat, f("syrk_ln"), f("diare"), f("potrf_l"), f("trsm_rltn"),
                                   f("gemm_nt"))
    P, tp, t1 = _cpu_times(run)
    errs = {}
    for k, B in (("L", L), ("X", X), ("D", D)):
        g = B.unpack_all()
        h = hout[k][0]
        pm, cn, st = B.s.pm, B.s.cn, B.s.stride
        off = (B.s.pA - B.buf.data_ptr()) // 8
        r = h[off: off + nb * st].reshape(nb, st)[:, :pm * cn].reshape(nb, pm // 4, cn, 4).transpose(0, 1, 3, 2)
        r = r.reshape(nb, pm, cn)[:, :16, :16]
        if k == "L":
            g, r = np.tril(g), np.tril(r)
        errs[k] = float(np.linalg.norm(g - r) / np.linalg.norm(r))
    return {"kind": kind, "library": name, "instances_per_s": nb / tp, "cores": P,
            "p1_instances_per_s": nb / t1, "median_pass_ms": 1e3 * tp,
            "sample": "the GPU leg's %d instances (host copies of its slabs)" % nb,
            "gpu_vs_reference_relfro": errs}


def cpu_riccati_leg(nbt, N, nx, nu, sBA, sRSQ, sL):
    """The Riccati factorization through the compiled reference
    (examples/example_d_riccati_recursion.c:115-143: dpotrf_l, then per stage
    dtrmm_rlnn + dsyrk_dpotrf_ln) on host copies of the GPU leg's FP64 slabs;
    problems/s at P = all physical cores and P = 1; returns (report, the
    reference's L as problems x (N+1) x 16 x 16)."""
    lib, prefix, kind, name = cpu_library()
    drv = cpu_driver()
    f = lambda s_: C.cast(getattr(lib, prefix + s_), C.c_void_p)
    hBA, hRSQ, hL = _host_slab(sBA), _host_slab(sRSQ), _host_slab(sL)
    hL[0][:] = 0.0

    def run(P):
        return drv.cpu_ric_trf_batch(P, nbt, N, nx, nu, *hBA[1:], *hRSQ[1:], *hL[1:], f("potrf_l"), f("trmm_rlnn"),
                                     f("syrk_potrf_ln") if prefix == "oracle_d_" else f("syrk_dpotrf_ln"))
    P, tp, t1 = _cpu_times(run)
    pm, cn, st = sL.s.pm, sL.s.cn, sL.s.stride
    off = (sL.s.pA - sL.buf.data_ptr()) // 8
    tot = nbt * (N + 1)
    r = hL[0][off: off + tot * st].reshape(tot, st)[:, :pm * cn].reshape(tot, pm // 4, cn, 4).transpose(0, 1, 3, 2)
    Lref = r.reshape(tot, pm, cn)[:, :16, :16].reshape(nbt, N + 1, 16, 16)
    g = sL.unpack_all().reshape(nbt, N + 1, 16, 16)
    m = nu + nx
    err = float(np.linalg.norm(np.tril(g[:, :N, :m, :m]) - np.tril(Lref[:, :N, :m, :m])) /
                np.linalg.norm(np.tril(Lref[:, :N, :m, :m])))
    rep = {"kind": kind, "library": name, "problems_per_s": nbt / tp, "cores": P, "p1_problems_per_s": nbt / t1,
           "median_pass_ms": 1e3 * tp, "sample": "the GPU leg's %d problems (host copies of its FP64 slabs)" % nbt,
           "gpu_fp64_vs_reference_relfro": err}
    return rep, Lref


def learned_dispatch(n_ops=1_000_000, train_frac=0.3, seed=5, budget_s=150.0, cpu=True):
    """Config 5, the mixed-op stream: ops drawn 40% gemm_nt, 25% potrf_l, 20%
    getrf_rp, 15% geqrf (m = 2n), sizes log-uniform in 4..384 (geqrf n in
    4..192), batched into launches of log-uniform 256..8192 instances, until
    the launches hold n_ops instances.  The exhaustive autotuner times every
    kernel variant of every launch; the MLP cost model is trained by the
    library's CUDA kernels on the first train_frac of the launches and
    installed in the library, which then dispatches the held-out launches
    itself (variant -1; each new launch shape runs the model once on the
    device).  Reported: regret of the library's picks, of the built-in rule and
    of a fixed variant against the exhaustive best, on the held-out launches;
    end-to-end GFLOP/s of the whole stream under each policy; the compiled
    reference on the host cores for a sample of launches.  If the sweep
    exceeds budget_s the stream is cut there and the ops actually covered are
    reported."""
    import torch
    import blasfeo_b200 as bf
    from blasfeo_b200 import autotune as at
    from blasfeo_b200.costmodel import CostModel
    lib = bf.lib
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    recs, launches_kept, ops = [], [], 0
    while ops < n_ops and time.perf_counter() - t0 < budget_s:
        op, batch, m, n, k = at.sample_launch(rng)
        batch = min(batch, n_ops - ops) if n_ops - ops >= 256 else batch
        L = at.Launch(op, batch, m[:batch], n[:batch], k[:batch], seed=len(recs))
        times = [min(L.time(v, 1), L.time(v, 1)) for v in range(at.NVAR[op])]
        heur = min(L.time(-1, 1), L.time(-1, 1))
        recs.append({"op": op, "batch": batch, "feat": L.feature_rows(), "times": np.array(times), "heur": heur,
                     "flops": L.flops})
        ops += batch
        nbytes = 8.0 * float(np.sum(L.m * L.k + L.n * L.k + L.m * L.n))
        if len(launches_kept) < 12 and len(recs) % 7 == 1 and nbytes < 3e8:
            launches_kept.append(L)  # a sample for the CPU leg
        else:
            del L
    sweep_s = time.perf_counter() - t0
    ntr = max(4, int(len(recs) * train_frac))
    X, y = at.training_set(recs[:ntr])
    cm = CostModel(at.NFEAT, seed=0)
    cm.fit(X, y, epochs=200, lr=2e-3, batch=256)
    test = recs[ntr:]
    picks = [cm.pick(r["feat"]) for r in test]
    out = {"ops": ops, "launches": len(recs), "train_launches": ntr, "test_launches": len(test),
           "complete": ops >= n_ops, "sweep_s": sweep_s,
           "ops_by_kind": {op_: int(sum(r["batch"] for r in recs if r["op"] == op_)) for op_ in at.OPS}}
    for name, pk in (("mlp", picks), ("rule", [-1] * len(test)), ("variant0", [0] * len(test))):
        mean, tot = at.regret(test, pk)
        out["regret_" + name] = {"mean_per_launch": mean, "total_time": tot}
    # the library dispatching the held-out launches itself with the installed model
    rng2 = np.random.default_rng(seed)
    lib_t, lib_match = 0.0, 0
    try:
        cm.install()
        # rebuild the held-out launches (same draws) and time variant -1 through the library
        idx = 0
        ops2 = 0
        while idx < len(recs):
            op, batch, m, n, k = at.sample_launch(rng2)
            batch = min(batch, n_ops - ops2) if n_ops - ops2 >= 256 else batch
            ops2 += batch
            if idx >= ntr:
                L = at.Launch(op, batch, m[:batch], n[:batch], k[:batch], seed=idx)
                P_ = lambda t_: C.c_void_p(t_.data_ptr())
                pk = lib.blasfeo_b200_dispatch_pick(at.OPS.index(op), batch, P_(L.mv), P_(L.nv), P_(L.kv), L.maxm,
                                                   L.maxn, L.maxk, None)
                lib_match += int(pk == picks[idx - ntr])
                lib_t += min(L.time(-1, 1), L.time(-1, 1))
                del L
            idx += 1
    finally:
        CostModel.uninstall()
    best_test = sum(float(r["times"].min()) for r in test)
    out["regret_library_dispatch"] = {"total_time": lib_t / best_test - 1.0 if best_test > 0 else None,
                                      "picks_equal_to_model_argmin": lib_match, "of": len(test)}
    fl = sum(r["flops"] for r in recs)
    # whole stream: the training launches run with the exhaustive best (that is what was measured for them)
    t_best = sum(float(r["times"].min()) for r in recs)
    t_rule = sum(float(r["heur"]) for r in recs)
    t_v0 = sum(float(r["times"][0]) for r in recs)
    t_mlp = sum(float(r["times"].min()) for r in recs[:ntr]) + sum(float(r["times"][p]) for r, p in zip(test, picks))
    out["stream_gflops"] = {"exhaustive": fl / t_best / 1e6, "mlp": fl / t_mlp / 1e6, "rule": fl / t_rule / 1e6,
                            "variant0": fl / t_v0 / 1e6, "total_gflop": fl / 1e9}
    out["by_op_exhaustive"] = {op_: {"ms": sum(float(r["times"].min()) for r in recs if r["op"] == op_),
                                     "gflop": sum(r["flops"] for r in recs if r["op"] == op_) / 1e9}
                               for op_ in at.OPS}
    for v in out["by_op_exhaustive"].values():
        v["gflops"] = v["gflop"] / (v["ms"] * 1e-3) if v["ms"] > 0 else None
    if cpu:
        try:
            out["cpu_reference"] = cpu_ops_leg(launches_kept, {r_["op"]: 0 for r_ in recs})
        except Exception as ex:  # reported, never silently replaced
            out["cpu_reference"] = {"error": repr(ex)}
    del launches_kept
    torch.cuda.empty_cache()
    return out


def cpu_ops_leg(launches, _ops):
    """The compiled reference on host copies of a sample of the stream's
    launches (blasfeo_dgemm_nt / dpotrf_l / dgetrf_rp per instance; dgeqrf from
    the GENERIC build, whose HP Haswell version crashes on unaligned stack
    buffers), one thread per physical core; GFLOP/s of the sample, and the same
    sample's GPU time under the exhaustive best variants."""
    from blasfeo_b200 import autotune as at
    from oracle.pyoracle import DMat, ref_lib, ref_available
    lib_, prefix, kind, name = cpu_library()
    gen = ref_lib("generic") if ref_available("generic") else lib_
    drv = cpu_driver()
    drv.cpu_ops_batch.restype = C.c_double
    f = lambda L_, s_: C.cast(getattr(L_, prefix + s_), C.c_void_p)
    fl, tc, tg = 0.0, 0.0, 0.0
    keep = []
    for L in launches:
        def host(slab, rows, cols):
            from oracle.pyoracle import _aligned_zeros
            src = slab.buf.cpu().numpy()
            h = _aligned_zeros(src.size, np.float64)
            h[:] = src
            d = slab.desc.cpu().numpy().view(DESC_DTYPE_CPU).copy()
            shift = h.ctypes.data - slab.buf.data_ptr()
            for fld in ("mem", "pA", "dA"):
                d[fld] = (d[fld].astype(np.int64) + shift).astype(np.uint64)
            arr = (DMat * len(d)).from_buffer_copy(d.tobytes())
            keep.append((h, arr))
            return arr
        A = host(L.A, L.m, L.n)
        B = host(L.B, L.n, L.k) if L.op == "gemm_nt" else A
        D = host(L.D, L.m, L.n)
        iv = lambda a: (C.c_int * len(a))(*[int(v) for v in a])
        mm, nn, kk = iv(L.m), iv(L.n), iv(L.k)
        opi = at.OPS.index(L.op)
        geq = (C.cast(getattr(gen, "blasfeo_dgeqrf_worksize"), C.c_void_p), C.cast(getattr(gen, "blasfeo_dgeqrf"),
                                                                                   C.c_void_p))
        run = lambda P_: drv.cpu_ops_batch(P_, opi, L.batch, mm, nn, kk, A, B, D, f(lib_, "gemm_nt"),
                                           f(lib_, "potrf_l"), f(lib_, "getrf_rp"), geq[0], geq[1], L.maxm, L.maxn)
        P_, tp, _ = _cpu_times(run, passes=3, p1_passes=1)
        tc += tp
        fl += L.flops
        tg += min(L.time(v, 1) for v in range(at.NVAR[L.op])) * 1e-3
    return {"kind": kind, "library": name, "cores": P_, "launches": len(launches), "gflops": fl / tc / 1e9,
            "gpu_gflops_same_sample": fl / tg / 1e9,
            "sample": "%d launches of the stream (host copies of their slabs), %.2f GFLOP" % (len(launches), fl / 1e9)}


def run_e2e(args, W, lib, torch, dev, stream, barrier, world):
    """Mixed path with all inputs in pinned host memory (mapped into the GPU's
    address space): blasfeo_dsposv_l_vbatch_mapped reads the lower triangles
    over the host link and writes x to host memory."""
    P = lambda t: C.c_void_p(t.data_ptr())
    H = W.mapped_copy()
    hx, hn, hdesc, hbd, hxd = H.x, H.n, H.desc, H.bdesc, H.xdesc
    hinfo = torch.zeros(args.num, dtype=torch.int32).pin_memory()
    sh = C.c_void_p(stream.cuda_stream)

    def call():
        return lib.blasfeo_dsposv_l_vbatch_mapped(args.num, P(hn), W.max_n, P(hdesc), P(hbd), P(hxd), MAX_ITER, TOL,
                                                  None, None, P(hinfo), None, 0, sh)
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    if not (hinfo.numpy() == 0).all():
        raise RuntimeError("mapped solve: %d systems not converged" % int((hinfo.numpy() != 0).sum()))
    xs = hx.numpy()
    i = 0
    a, b = W.matrix(i), W.rhs[i]
    x = xs[W.voff[i]:W.voff[i] + len(b)]
    res = np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max())
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    barrier()
    import torch.distributed as dist
    ms = reduce_max_ms(e0.elapsed_time(e1) / args.steps, world, dist, dev)
    n = W.ns.astype(np.int64)
    h2d = int((n * (n + 1) // 2 * 8).sum() + W.b.numel() * 8 + hn.numel() * 4 + hdesc.numel() + hbd.numel() * 2)
    d2h = int(n.sum() * 8)
    return {"value": aggregate_value(world, args.num, ms), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "host_wall_ms_per_step": wall * 1e3,
            "path": "blasfeo_dsposv_l_vbatch_mapped, all inputs in pinned host memory",
            "host_link_gbs": (h2d + d2h) / (ms * 1e-3) / 1e9, "residual_system0": float(res)}


if __name__ == "__main__":
    sys.exit(main())
