"""Autotuner and learned dispatch for the variable-size batched routines.

* ``sample_launch`` draws one batched launch of the mixed-op stream: an op
  (gemm_nt, potrf_l, getrf_rp, geqrf), a batch size (log-uniform 256..8192
  by default) and per-instance sizes (log-uniform 4..384; geqrf m = 2n with
  n in 4..192).
* ``Launch`` builds the device operands of one launch once (one slab per
  operand role, descriptor arrays) and runs it with any kernel variant.
* ``sweep`` times every variant of every sampled launch with CUDA events --
  the exhaustive autotuner; ``save_table``/``load_table`` persist the results
  keyed by GPU name, driver version and library build.
* ``CostModel`` (costmodel.py) is trained on those timings; ``pick`` chooses
  the variant with the smallest predicted time.  Variants never change the
  arithmetic of an element, so a pick can only change the speed.
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np

from . import lib, LIB_PATH
from .workloads import DESC_DTYPE

OPS = ("gemm_nt", "potrf_l", "getrf_rp", "geqrf")
NVAR = {op: int(lib.blasfeo_b200_num_variants(i)) for i, op in enumerate(OPS)}
MAXVAR = max(NVAR.values())
NFEAT = len(OPS) + 1 + 9 + MAXVAR


def log_uniform_int(rng, lo, hi, size):
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size))).astype(np.int64).clip(lo, hi)


def sample_launch(rng, op=None, bmin=256, bmax=8192, nmax=384):
    """(op, batch, m, n, k) with per-instance size arrays."""
    if op is None:
        op = rng.choice(OPS, p=[0.40, 0.25, 0.20, 0.15])
    batch = int(log_uniform_int(rng, bmin, bmax, 1)[0])
    if op == "gemm_nt":
        m, n, k = (log_uniform_int(rng, 4, nmax, batch) for _ in range(3))
    elif op == "geqrf":
        n = log_uniform_int(rng, 4, nmax // 2, batch)
        m, k = 2 * n, n
    else:
        n = log_uniform_int(rng, 4, nmax, batch)
        m, k = n, n
    return op, batch, m, n, k


def flops(op, m, n, k):
    m, n, k = (np.asarray(x, dtype=np.float64) for x in (m, n, k))
    if op == "gemm_nt":
        return float((2 * m * n * k).sum())
    if op == "potrf_l":
        return float((n ** 3 / 3 + n ** 2 / 2 + n / 6).sum())
    if op == "getrf_rp":
        return float((2 * n ** 3 / 3 - n ** 2 / 2 + 5 * n / 6).sum())
    return float((2 * m * n ** 2 - 2 * n ** 3 / 3 + m * n + n ** 2 + 14 * n / 3).sum())


def features(op, batch, m, n, k, variant):
    """Model input: op one-hot, log2 batch, mean/max/std of log2 m, n, k, variant one-hot."""
    f = np.zeros(NFEAT, dtype=np.float32)
    f[OPS.index(op)] = 1.0
    f[len(OPS)] = np.log2(batch) / 13.0
    o = len(OPS) + 1
    for d in (m, n, k):
        l2 = np.log2(np.maximum(np.asarray(d, dtype=np.float64), 1.0))
        f[o:o + 3] = (l2.mean() / 9.0, l2.max() / 9.0, l2.std() / 4.0)
        o += 3
    f[o + variant] = 1.0
    return f


def _memsize(m, n):
    pm = (np.asarray(m) + 3) // 4 * 4
    cn = (np.asarray(n) + 3) // 4 * 4
    dl = (np.minimum(m, n) + 15) // 16 * 16
    return ((pm * cn + dl) * 8 + 63) // 64 * 64, pm, cn


class Slab:
    """One device allocation holding a panel-major matrix per instance."""

    def __init__(self, rows, cols, device="cuda", fill=True, seed=0):
        import torch
        sizes, pm, cn = _memsize(rows, cols)
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.buf = torch.empty(int(sizes.sum()) // 8 + 8, dtype=torch.float64, device=device)
        if fill:
            g = torch.Generator(device=device)
            g.manual_seed(seed)
            self.buf.uniform_(-0.5, 0.5, generator=g)
        base = self.buf.data_ptr()
        d = np.zeros(len(rows), dtype=DESC_DTYPE)
        d["mem"] = base + offs
        d["pA"] = base + offs
        d["dA"] = base + offs + (pm * cn * 8).astype(np.int64)
        d["m"], d["n"], d["pm"], d["cn"] = rows, cols, pm, cn
        d["memsize"] = sizes
        self.desc = torch.from_numpy(d.view(np.uint8).copy()).to(device)
        self.offs, self.pm, self.cn = offs, pm, cn

    def add_to_diagonal(self, n, value):
        """A_ii += value[b] for i < n[b] (makes a uniform(-0.5,0.5) lower triangle SPD)."""
        import torch
        idx, val = [], []
        for b in range(len(n)):
            i = np.arange(int(n[b]))
            idx.append(self.offs[b] // 8 + (i - i % 4) * self.cn[b] + 4 * i + i % 4)
            val.append(np.full(len(i), float(value[b])))
        idx = torch.from_numpy(np.concatenate(idx)).to(self.buf.device)
        self.buf[idx] += torch.from_numpy(np.concatenate(val)).to(self.buf.device)


class Launch:
    def __init__(self, op, batch, m, n, k, seed=0, device="cuda"):
        import torch
        self.op, self.batch, self.m, self.n, self.k = op, batch, m, n, k
        t = lambda a: torch.from_numpy(np.asarray(a, dtype=np.int32)).to(device)
        self.mv, self.nv, self.kv = t(m), t(n), t(k)
        self.maxm, self.maxn, self.maxk = int(np.max(m)), int(np.max(n)), int(np.max(k))
        if op == "gemm_nt":
            self.A = Slab(m, k, device, seed=seed)
            self.B = Slab(n, k, device, seed=seed + 1)
            self.D = Slab(m, n, device, fill=False)
        else:
            self.A = Slab(m, n, device, seed=seed)
            if op == "potrf_l":
                self.A.add_to_diagonal(n, n.astype(np.float64))
            self.D = Slab(m, n, device, fill=False)
            self.ipiv = torch.zeros(batch * max(1, self.maxn), dtype=torch.int32, device=device)
        self.flops = flops(op, m, n, k)

    def run(self, variant, stream=None):
        P = lambda x: C.c_void_p(x.data_ptr())
        s = C.c_void_p(getattr(stream, "cuda_stream", stream) or 0)
        b = self.batch
        if self.op == "gemm_nt":
            return lib.blasfeo_dgemm_nt_vbatch_variant(b, P(self.mv), P(self.nv), P(self.kv), self.maxm, self.maxn,
                                                       self.maxk, 1.0, P(self.A.desc), P(self.B.desc), 0.0,
                                                       P(self.D.desc), P(self.D.desc), variant, s)
        if self.op == "potrf_l":
            return lib.blasfeo_dpotrf_l_vbatch_variant(b, P(self.nv), self.maxn, P(self.A.desc), P(self.D.desc), None,
                                                       variant, s)
        if self.op == "getrf_rp":
            return lib.blasfeo_dgetrf_rp_vbatch_variant(b, P(self.mv), P(self.nv), self.maxm, self.maxn,
                                                        P(self.A.desc), P(self.D.desc), P(self.ipiv), self.maxn, None,
                                                        variant, s)
        return lib.blasfeo_dgeqrf_vbatch_variant(b, P(self.mv), P(self.nv), self.maxm, self.maxn, P(self.A.desc),
                                                 P(self.D.desc), variant, s)

    def time(self, variant, reps=3):
        import torch
        st = self.run(variant)
        if st:
            raise RuntimeError("launch failed: status %d" % st)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(variant)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    def feature_rows(self):
        return np.stack([features(self.op, self.batch, self.m, self.n, self.k, v) for v in range(NVAR[self.op])])


def sweep(nlaunch, seed=0, bmin=256, bmax=8192, nmax=384, reps=3, ops=None):
    """Exhaustive autotune: time every variant of nlaunch sampled launches."""
    rng = np.random.default_rng(seed)
    recs = []
    for i in range(nlaunch):
        op = None if ops is None else ops[i % len(ops)]
        op, batch, m, n, k = sample_launch(rng, op, bmin, bmax, nmax)
        L = Launch(op, batch, m, n, k, seed=seed * 1000 + i)
        times = [L.time(v, reps) for v in range(NVAR[op])]
        heur = L.time(-1, reps)
        recs.append({"op": op, "batch": batch, "feat": L.feature_rows(), "times": np.array(times), "heur": heur,
                     "flops": L.flops, "sizes": (m, n, k)})
        del L
    return recs


def table_key():
    import torch
    p = torch.cuda.get_device_properties(0)
    h = hashlib.sha256(open(LIB_PATH, "rb").read()).hexdigest()[:16]
    drv = torch.version.cuda or "?"
    return "%s|cuda%s|%s" % (p.name, drv, h)


def save_table(recs, path):
    data = {"key": table_key(), "records": [
        {"op": r["op"], "batch": r["batch"], "times": r["times"].tolist(), "heur": r["heur"], "flops": r["flops"],
         "feat": r["feat"].tolist()} for r in recs]}
    with open(path, "w") as f:
        json.dump(data, f)


def load_table(path):
    with open(path) as f:
        data = json.load(f)
    if data.get("key") != table_key():
        return None
    return [{"op": r["op"], "batch": r["batch"], "times": np.array(r["times"]), "heur": r["heur"],
             "flops": r["flops"], "feat": np.array(r["feat"], dtype=np.float32)} for r in data["records"]]


def default_cache_path():
    d = os.path.join(os.path.expanduser("~"), ".cache", "blasfeo_b200")
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, "autotune.json")


def training_set(recs):
    X = np.concatenate([r["feat"] for r in recs]).astype(np.float32)
    y = np.concatenate([np.log(r["times"]) for r in recs]).astype(np.float32)
    return X, y


def regret(recs, picks):
    """Mean over launches of t(pick)/t(best) - 1, and the total-time regret;
    picks[i] is a variant index, or -1 for the built-in heuristic."""
    t = [r["heur"] if p < 0 else r["times"][p] for r, p in zip(recs, picks)]
    per = [ti / r["times"].min() - 1.0 for r, ti in zip(recs, t)]
    tot = sum(t) / sum(r["times"].min() for r in recs) - 1.0
    return float(np.mean(per)), float(tot)
