"""GPU checks of the learned dispatch: the CUDA MLP forward, gradient and Adam
kernels against the numpy oracle, training progress, and the regret of the
trained model's picks against the exhaustive sweep and the built-in rule."""
import ctypes as C

import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bf():
    import blasfeo_b200
    return blasfeo_b200


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


P = lambda x: C.c_void_p(x.data_ptr())


@pytest.mark.parametrize("nin,H,B", [(20, 128, 256), (7, 33, 50), (20, 128, 1)])
def test_forward_and_gradient_vs_oracle(bf, nin, H, B):
    import torch
    rng = np.random.default_rng(nin + H + B)
    npar = bf.lib.blasfeo_b200_mlp_param_count(nin, H)
    p = (rng.standard_normal(npar) / np.sqrt(H)).astype(np.float32)
    X = rng.standard_normal((B, nin)).astype(np.float32)
    t = rng.standard_normal(B).astype(np.float32)
    dp, dX, dt = _dev(p), _dev(X), _dev(t)
    work = torch.empty(bf.lib.blasfeo_b200_mlp_work_bytes(H, B) // 4 + 16, dtype=torch.float32, device="cuda")
    y = torch.empty(B, dtype=torch.float32, device="cuda")
    assert bf.lib.blasfeo_b200_mlp_forward(nin, H, P(dp), B, P(dX), P(y), P(work), None) == 0
    g = torch.empty(npar, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    assert bf.lib.blasfeo_b200_mlp_grad(nin, H, P(dp), B, P(dX), P(dt), P(g), P(loss), P(work), None) == 0
    torch.cuda.synchronize()
    yr, _ = mo.forward(p, X, nin, H)
    lr, gr = mo.loss_and_grad(p, X, t, nin, H)
    # FP32 kernels against the FP64 oracle on the same FP32 inputs
    assert np.linalg.norm(y.cpu().numpy() - yr) <= 1e-5 * max(1.0, np.linalg.norm(yr))
    assert abs(loss.item() - lr) <= 1e-5 * max(1.0, lr)
    gd = g.cpu().numpy()
    assert np.linalg.norm(gd - gr) <= 1e-4 * np.linalg.norm(gr)
    # per-block check: every parameter group gets its own gradient right
    for a, b in zip(mo.unpack(gd, nin, H), mo.unpack(gr, nin, H)):
        assert np.linalg.norm(a - b) <= 1e-4 * max(np.linalg.norm(b), 1e-6 * np.linalg.norm(gr))


def test_adam_step_vs_numpy(bf):
    import torch
    rng = np.random.default_rng(5)
    n = 3000
    p, g = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m, v = (rng.standard_normal(n) * 0.1).astype(np.float32), (rng.random(n) * 0.1).astype(np.float32)
    dp, dg, dm, dv = _dev(p), _dev(g), _dev(m), _dev(v)
    step, lr = 7, 1e-3
    assert bf.lib.blasfeo_b200_mlp_adam(n, P(dp), P(dg), P(dm), P(dv), step, lr, None) == 0
    torch.cuda.synchronize()
    m2 = 0.9 * m.astype(np.float64) + 0.1 * g
    v2 = 0.999 * v.astype(np.float64) + 0.001 * g.astype(np.float64) ** 2
    p2 = p - lr * (m2 / (1 - 0.9 ** step)) / (np.sqrt(v2 / (1 - 0.999 ** step)) + 1e-8)
    assert np.allclose(dm.cpu().numpy(), m2, rtol=1e-5, atol=1e-7)
    assert np.allclose(dv.cpu().numpy(), v2, rtol=1e-5, atol=1e-7)
    assert np.allclose(dp.cpu().numpy(), p2, rtol=1e-5, atol=1e-6)


def test_training_fits_a_smooth_function(bf):
    from blasfeo_b200.costmodel import CostModel
    rng = np.random.default_rng(11)
    X = rng.uniform(-1, 1, (2048, 6)).astype(np.float32)
    y = np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * np.abs(X[:, 3])
    cm = CostModel(6, hidden=64, seed=1)
    hist = cm.fit(X, y, epochs=60, lr=3e-3, batch=256)
    assert hist[-1] < 0.05 * hist[0]
    Xt = rng.uniform(-1, 1, (512, 6)).astype(np.float32)
    yt = np.sin(2 * Xt[:, 0]) + Xt[:, 1] * Xt[:, 2] + 0.5 * np.abs(Xt[:, 3])
    assert np.sqrt(np.mean((cm.predict(Xt) - yt) ** 2)) < 0.15 * np.std(yt) + 0.05


def test_learned_dispatch_regret(bf):
    """Sweep sampled launches of the mixed-op stream, train on 70% of them and
    score the held-out picks by regret against the exhaustive best."""
    from blasfeo_b200 import autotune as at
    from blasfeo_b200.costmodel import CostModel
    recs = at.sweep(48, seed=7, bmin=256, bmax=2048, nmax=256, reps=3)
    ntr = 34
    X, y = at.training_set(recs[:ntr])
    cm = CostModel(at.NFEAT, seed=0)
    cm.fit(X, y, epochs=300, lr=2e-3, batch=128)
    test = recs[ntr:]
    picks = [cm.pick(r["feat"]) for r in test]
    mlp_mean, mlp_tot = at.regret(test, picks)
    fixed_mean, fixed_tot = at.regret(test, [0] * len(test))
    print("regret mlp %.3f/%.3f  variant-0 %.3f/%.3f  rule %s" % (mlp_mean, mlp_tot, fixed_mean, fixed_tot,
                                                                  at.regret(test, [-1] * len(test))))
    rule_mean, rule_tot = at.regret(test, [-1] * len(test))
    assert mlp_tot < 0.25
    assert mlp_tot < fixed_tot
    # what the trained network gains over the method without it (the built-in
    # rule the library uses when no model is installed), on the held-out launches
    assert mlp_tot < rule_tot, (mlp_tot, rule_tot)


def test_library_dispatch_uses_the_installed_model(bf):
    """With the cost model installed, a *_vbatch call with variant -1 takes the
    model's pick (the same variant the Python-side argmin chooses), computed on
    the device from the launch's size arrays; without a model it takes the
    built-in rule (-1).  Results equal those of the picked variant."""
    import torch
    from blasfeo_b200 import autotune as at
    from blasfeo_b200.costmodel import CostModel
    recs = at.sweep(16, seed=3, bmin=256, bmax=1024, nmax=160, reps=2)
    X, y = at.training_set(recs)
    cm = CostModel(at.NFEAT, seed=1)
    cm.fit(X, y, epochs=120, lr=2e-3, batch=64)
    assert bf.lib.blasfeo_b200_cost_model_nfeat() == at.NFEAT
    rng = np.random.default_rng(9)
    P = lambda t: C.c_void_p(t.data_ptr())
    try:
        cm.install()
        for i in range(8):
            op, batch, m, n, k = at.sample_launch(rng, at.OPS[i % 4], 256, 1024, 160)
            L = at.Launch(op, batch, m, n, k, seed=i)
            want = cm.pick(L.feature_rows())
            got = bf.lib.blasfeo_b200_dispatch_pick(at.OPS.index(op), batch, P(L.mv), P(L.nv), P(L.kv), L.maxm, L.maxn,
                                                    L.maxk, None)
            assert got == want, (op, got, want)
            assert L.run(-1) == 0  # the call itself dispatches through the model (cached pick)
            torch.cuda.synchronize()
    finally:
        CostModel.uninstall()
    assert bf.lib.blasfeo_b200_dispatch_pick(0, 4, P(L.mv), P(L.nv), P(L.kv), 4, 4, 4, None) == -1
    assert bf.lib.blasfeo_b200_set_cost_model(at.NFEAT + 1, 128, None) == 1
