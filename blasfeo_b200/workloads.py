"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations, laid out in device memory for the batched entry
points (panel-major instances in one slab, descriptor arrays on the device).

Input generation uses torch on the GPU (QR factorizations and products to
build the SPD matrices); it is setup, never part of a timed region.
"""
import ctypes as C

import numpy as np

from . import lib, dmat, dvec

DESC_DTYPE = np.dtype([("mem", "<u8"), ("pA", "<u8"), ("dA", "<u8"), ("m", "<i4"), ("n", "<i4"), ("pm", "<i4"),
                       ("cn", "<i4"), ("use_dA", "<i4"), ("memsize", "<i4")])
VDESC_DTYPE = np.dtype([("mem", "<u8"), ("pa", "<u8"), ("m", "<i4"), ("pm", "<i4"), ("memsize", "<i4"),
                        ("pad", "<i4")])
assert DESC_DTYPE.itemsize == C.sizeof(dmat) and VDESC_DTYPE.itemsize == C.sizeof(dvec)


def memsize_dmat(m, n):
    return int(lib.blasfeo_memsize_dmat(m, n))


def to_panel_major(X, pm, cn):
    """(B, m, n) tensor -> (B, pm*cn) panel-major (panel size 4), zero padded."""
    import torch
    B, m, n = X.shape
    pad = torch.zeros((B, pm, cn), dtype=X.dtype, device=X.device)
    pad[:, :m, :n] = X
    return pad.reshape(B, pm // 4, 4, cn).permute(0, 1, 3, 2).reshape(B, pm * cn)


def from_panel_major(P, m, n, pm, cn):
    B = P.shape[0]
    return P[:, : pm * cn].reshape(B, pm // 4, cn, 4).permute(0, 1, 3, 2).reshape(B, pm, cn)[:, :m, :n]


class SpdBatch:
    """Variable-size batch of SPD systems A x = b in device memory.

    Systems of equal size are stored contiguously in one FP64 slab (each one
    laid out exactly like blasfeo_create_dmat would); ``desc`` is the device
    array of struct blasfeo_dmat descriptors in the original (random) order,
    ``bdesc`` / ``xdesc`` the struct blasfeo_dvec arrays of b and x.
    """

    def __init__(self, ns, mats_by_n, rhs, device="cuda"):
        import torch
        self.ns = np.asarray(ns, dtype=np.int32)
        num = len(ns)
        sizes = np.array([memsize_dmat(int(n), int(n)) for n in range(int(self.ns.max()) + 1)])
        order = np.argsort(self.ns, kind="stable")
        per = sizes[self.ns[order]]
        offs_sorted = np.concatenate([[0], np.cumsum(per)[:-1]])
        self.offsets = np.empty(num, dtype=np.int64)
        self.offsets[order] = offs_sorted
        self.total_bytes = int(per.sum())
        self.slab = torch.zeros(self.total_bytes // 8 + 8, dtype=torch.float64, device=device)
        base = self.slab.data_ptr()
        for n, (idx, X) in mats_by_n.items():
            # equal-size systems are contiguous in the slab, in ascending index order
            pm = cn = (n + 3) // 4 * 4
            stride = int(sizes[n]) // 8
            o = int(self.offsets[idx[0]]) // 8
            view = self.slab[o:o + len(idx) * stride].view(len(idx), stride)
            view[:, : pm * cn] = to_panel_major(X, pm, cn)
        d = np.zeros(num, dtype=DESC_DTYPE)
        pmv = (self.ns + 3) // 4 * 4
        d["mem"] = base + self.offsets
        d["pA"] = base + self.offsets
        d["dA"] = base + self.offsets + pmv.astype(np.int64) * pmv * 8
        d["m"] = self.ns
        d["n"] = self.ns
        d["pm"] = pmv
        d["cn"] = pmv
        d["memsize"] = sizes[self.ns]
        self.desc = torch.from_numpy(d.view(np.uint8).copy()).to(device)
        # right-hand sides and solutions: one FP64 vector per system, 4-padded
        vlen = (self.ns + 3) // 4 * 4
        voff = np.concatenate([[0], np.cumsum(vlen)[:-1]]).astype(np.int64)
        self.voff, self.vlen = voff, vlen
        self.b = torch.zeros(int(vlen.sum()) + 4, dtype=torch.float64, device=device)
        self.x = torch.zeros_like(self.b)
        bflat = np.zeros(int(vlen.sum()) + 4)
        for i, r in enumerate(rhs):
            bflat[voff[i]:voff[i] + len(r)] = r
        self.b.copy_(torch.from_numpy(bflat))
        self.rhs = rhs
        self.bdesc = self._vdesc(self.b)
        self.xdesc = self._vdesc(self.x)
        self.nvec = torch.from_numpy(self.ns.copy()).to(device)
        self.max_n = int(self.ns.max())

    def _vdesc(self, t):
        import torch
        v = np.zeros(len(self.ns), dtype=VDESC_DTYPE)
        v["mem"] = t.data_ptr() + self.voff * 8
        v["pa"] = t.data_ptr() + self.voff * 8
        v["m"] = self.ns
        v["pm"] = self.vlen
        v["memsize"] = self.vlen * 8
        return torch.from_numpy(v.view(np.uint8).copy()).to(t.device)

    def solution(self, i):
        n = int(self.ns[i])
        o = int(self.voff[i])
        return self.x[o:o + n].cpu().numpy()

    def matrix(self, i):
        n = int(self.ns[i])
        pm = (n + 3) // 4 * 4
        o = int(self.offsets[i]) // 8
        P = self.slab[o:o + pm * pm].reshape(1, -1)
        return from_panel_major(P, n, n, pm, pm)[0].cpu().numpy()

    def mapped_copy(self):
        """The same systems in pinned host memory (for blasfeo_dsposv_l_vbatch_mapped):
        matrices, b, x, sizes and descriptors, every pointer a host address."""
        return MappedSpdBatch(self)

    def lower_bytes(self):
        """Algorithmic HBM bytes of one solve pass: lower triangle of A, b and x (FP64)."""
        n = self.ns.astype(np.int64)
        return int((n * (n + 1) // 2 * 8 + 16 * n).sum())

    def chol_flops(self):
        n = self.ns.astype(np.float64)
        return float((n ** 3 / 3 + n ** 2 / 2 + n / 6 + 4 * n ** 2).sum())


class MappedSpdBatch:
    """Pinned host copy of an SpdBatch: slab, b, x, n and the descriptor arrays
    (struct blasfeo_dmat / blasfeo_dvec with host pointers)."""

    def __init__(self, W):
        import torch
        self.slab = torch.empty(W.slab.numel(), dtype=torch.float64, pin_memory=True)
        self.slab.copy_(W.slab)
        self.b = torch.empty(W.b.numel(), dtype=torch.float64, pin_memory=True)
        self.b.copy_(W.b)
        self.x = torch.zeros(W.b.numel(), dtype=torch.float64).pin_memory()
        self.n = torch.from_numpy(W.ns.copy()).pin_memory()
        d = W.desc.cpu().numpy().view(DESC_DTYPE).copy()
        shift = self.slab.data_ptr() - W.slab.data_ptr()
        for f in ("mem", "pA", "dA"):
            d[f] = d[f] + np.uint64(shift) if shift >= 0 else d[f] - np.uint64(-shift)
        self.desc = torch.from_numpy(d.view(np.uint8).copy()).pin_memory()

        def vd(t):
            v = np.zeros(len(W.ns), dtype=VDESC_DTYPE)
            v["mem"] = t.data_ptr() + W.voff * 8
            v["pa"] = t.data_ptr() + W.voff * 8
            v["m"] = W.ns
            v["pm"] = W.vlen
            v["memsize"] = W.vlen * 8
            return torch.from_numpy(v.view(np.uint8).copy()).pin_memory()
        self.bdesc, self.xdesc = vd(self.b), vd(self.x)
        self.voff = W.voff

    def solution(self, i, n):
        o = int(self.voff[i])
        return self.x[o:o + n].numpy().copy()


def spd_config3(num=20000, nmin=4, nmax=256, logcond=6.0, seed=0, device="cuda"):
    """Uneven SPD batch: n ~ U{nmin..nmax}; A = Q diag(lambda) Q^T, Q from the QR of
    an N(0,1) matrix, log10(lambda) ~ U[0, logcond]; b ~ N(0,1)."""
    import torch
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=num).astype(np.int32)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    mats = {}
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        B = len(idx)
        G = torch.randn((B, int(n), int(n)), generator=g, dtype=torch.float64, device=device)
        Q, _ = torch.linalg.qr(G)
        lam = 10.0 ** (torch.rand((B, int(n)), generator=g, dtype=torch.float64, device=device) * logcond)
        A = (Q * lam[:, None, :]) @ Q.transpose(1, 2)
        A = 0.5 * (A + A.transpose(1, 2))
        mats[int(n)] = (idx, A)
    rhs = [rng.standard_normal(int(n)) for n in ns]
    return SpdBatch(ns, mats, rhs, device=device)


def fill_batch(B, X):
    """Write a (batch, m, n) FP64 tensor into the uniform-batch slab B (api.DMatBatch), on the device."""
    b = X.shape[0]
    pm, cn, st = B.s.pm, B.s.cn, B.s.stride
    view = B.buf[: b * st * 8].view(X.dtype).view(b, st)
    view[:, : pm * cn] = to_panel_major(X, pm, cn)


def fp64_roofline_batches(n, target_bytes=2.0e9, seed=0, device="cuda"):
    """Uniform batches for the FP64 batched-routine rooflines at size n (inputs
    larger than L2): gemm_nt operands A, B (U[-1,1]) and output D; potrf_l
    input C = G G^T / n + I (G ~ N(0,1)) and output L."""
    import torch
    from .api import DMatBatch
    g = torch.Generator(device=device)
    g.manual_seed(seed + n)
    bg = max(64, int(target_bytes / (3 * n * n * 8)))
    A, B, D = DMatBatch(n, n, bg), DMatBatch(n, n, bg), DMatBatch(n, n, bg)
    fill_batch(A, torch.rand((bg, n, n), generator=g, dtype=torch.float64, device=device) * 2 - 1)
    fill_batch(B, torch.rand((bg, n, n), generator=g, dtype=torch.float64, device=device) * 2 - 1)
    bp = max(64, int(target_bytes / (2 * n * n * 8)))
    Cm, L = DMatBatch(n, n, bp), DMatBatch(n, n, bp)
    pm, cn, st = Cm.s.pm, Cm.s.cn, Cm.s.stride
    slab = Cm.buf[: bp * st * 8].view(torch.float64).view(bp, st)
    for s0 in range(0, bp, 4096):
        s1 = min(bp, s0 + 4096)
        G = torch.randn((s1 - s0, n, n), generator=g, dtype=torch.float64, device=device)
        S = G @ G.transpose(1, 2) / n + torch.eye(n, dtype=torch.float64, device=device)
        slab[s0:s1, : pm * cn] = to_panel_major(S, pm, cn)
    return {"gemm": (bg, A, B, D), "potrf": (bp, Cm, L)}
