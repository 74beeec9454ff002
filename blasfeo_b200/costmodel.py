"""Learned cost model: an MLP (nin -> 128 -> 128 -> 128 -> 1, ReLU, FP32) that
predicts log(run time) of a batched launch for one kernel variant from the
features in autotune.features.  Training and inference run in the CUDA
kernels of libblasfeo_b200 (blasfeo_b200_mlp_forward / _grad / _adam); this
class only holds the device buffers and drives the loop."""
import ctypes as C

import numpy as np

from . import lib, check

HIDDEN = 128


class CostModel:
    def __init__(self, nin, hidden=HIDDEN, seed=0, device="cuda"):
        import torch
        self.nin, self.H = nin, hidden
        self.np = int(lib.blasfeo_b200_mlp_param_count(nin, hidden))
        rng = np.random.default_rng(seed)
        parts = []
        for fan_in, shape in [(nin, (nin, hidden)), (None, (hidden,)), (hidden, (hidden, hidden)), (None, (hidden,)),
                              (hidden, (hidden, hidden)), (None, (hidden,)), (hidden, (hidden, 1)), (None, (1,))]:
            if fan_in is None:
                parts.append(np.zeros(shape))
            else:
                lim = np.sqrt(6.0 / fan_in)  # He-uniform for ReLU layers
                parts.append(rng.uniform(-lim, lim, shape))
        p = np.concatenate([x.ravel() for x in parts]).astype(np.float32)
        assert p.size == self.np
        self.device = device
        self.params = torch.from_numpy(p).to(device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step = 0
        self.mu = 0.0
        self.sd = 1.0
        self._work = None
        self._work_b = 0

    def _ws(self, B):
        import torch
        if self._work is None or self._work_b < B:
            nb = int(lib.blasfeo_b200_mlp_work_bytes(self.H, B))
            self._work = torch.empty(nb // 4 + 16, dtype=torch.float32, device=self.device)
            self._work_b = B
        return self._work

    def grad(self, X, t):
        """Loss and gradients of the MSE between net(X) and t (device tensors)."""
        P = lambda x: C.c_void_p(x.data_ptr())
        w = self._ws(X.shape[0])
        check(lib.blasfeo_b200_mlp_grad(self.nin, self.H, P(self.params), X.shape[0], P(X), P(t), P(self.grads),
                                        P(self.loss), P(w), None))
        return self.loss, self.grads

    def fit(self, X, y, epochs=300, lr=2e-3, batch=512, seed=0):
        """Train on features X [N x nin] and targets y = log(time) (host arrays)."""
        import torch
        self.mu, self.sd = float(np.mean(y)), float(np.std(y) + 1e-6)
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(self.device)
        yd = torch.from_numpy(((np.asarray(y) - self.mu) / self.sd).astype(np.float32)).to(self.device)
        rng = np.random.default_rng(seed)
        n = len(y)
        P = lambda x: C.c_void_p(x.data_ptr())
        hist = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).to(self.device)
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb, yb = Xd[idx].contiguous(), yd[idx].contiguous()
                self.grad(xb, yb)
                self.step += 1
                check(lib.blasfeo_b200_mlp_adam(self.np, P(self.params), P(self.grads), P(self.m), P(self.v),
                                                self.step, lr, None))
            if ep % 50 == 0 or ep == epochs - 1:
                hist.append(float(self.loss.item()))
        return hist

    def predict(self, X):
        """Predicted log(time) for each row of X (host array)."""
        import torch
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(self.device)
        y = torch.empty(Xd.shape[0], dtype=torch.float32, device=self.device)
        P = lambda x: C.c_void_p(x.data_ptr())
        check(lib.blasfeo_b200_mlp_forward(self.nin, self.H, P(self.params), Xd.shape[0], P(Xd), P(y),
                                           P(self._ws(Xd.shape[0])), None))
        return y.cpu().numpy().astype(np.float64) * self.sd + self.mu

    def pick(self, feat_rows):
        """Variant with the smallest predicted time (feat_rows: one row per variant)."""
        return int(np.argmin(self.predict(feat_rows)))

    def install(self):
        """Make the library dispatch with this model: the *_vbatch routines called
        with variant -1 take its picks (blasfeo_b200_set_cost_model)."""
        p = np.ascontiguousarray(self.params.cpu().numpy(), dtype=np.float32)
        check(lib.blasfeo_b200_set_cost_model(self.nin, self.H, C.c_void_p(p.ctypes.data)))

    @staticmethod
    def uninstall():
        lib.blasfeo_b200_clear_cost_model()

    def save(self, path, key):
        """Persist the trained parameters, keyed like the autotune table (GPU,
        CUDA version, library build): load() refuses a file of another key."""
        np.savez(path, key=np.array(key), params=self.params.cpu().numpy(), nin=self.nin, hidden=self.H, mu=self.mu,
                 sd=self.sd)

    @classmethod
    def load(cls, path, key, device="cuda"):
        import torch
        d = np.load(path)
        if str(d["key"]) != key:
            return None
        cm = cls(int(d["nin"]), int(d["hidden"]), device=device)
        cm.params = torch.from_numpy(d["params"].astype(np.float32)).to(device)
        cm.mu, cm.sd = float(d["mu"]), float(d["sd"])
        return cm
