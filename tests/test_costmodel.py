"""CPU checks of the cost-model side: the numpy MLP oracle against finite
differences, the launch sampler and features, and the regret arithmetic."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def _params(nin, H, rng):
    n = nin * H + H + 2 * (H * H + H) + H + 1
    return rng.standard_normal(n) * 0.3


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, H, B = 5, 7, 9
    p = _params(nin, H, rng)
    X = rng.standard_normal((B, nin))
    t = rng.standard_normal(B)
    loss, g = mo.loss_and_grad(p, X, t, nin, H)
    y, _ = mo.forward(p, X, nin, H)
    assert abs(loss - np.mean((y - t) ** 2)) <= 1e-14 * max(1.0, loss)
    eps = 1e-6
    idx = rng.choice(len(p), 60, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mo.loss_and_grad(pp, X, t, nin, H)[0] - mo.loss_and_grad(pm, X, t, nin, H)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), i


def test_oracle_parameter_layout():
    nin, H = 3, 4
    p = np.arange(nin * H + H + 2 * (H * H + H) + H + 1, dtype=np.float64)
    W1, b1, W2, b2, W3, b3, W4, b4 = mo.unpack(p, nin, H)
    assert W1.shape == (nin, H) and W1[0, 1] == 1 and b1[0] == nin * H
    assert W4.shape == (H, 1) and b4[0] == p[-1]


def test_param_count_matches_library():
    import blasfeo_b200 as bf
    for nin, H in ((20, 128), (5, 7)):
        assert bf.lib.blasfeo_b200_mlp_param_count(nin, H) == nin * H + H + 2 * (H * H + H) + H + 1
    assert bf.lib.blasfeo_b200_mlp_param_count(0, 128) == -1


def test_sampler_and_features():
    from blasfeo_b200 import autotune as at
    rng = np.random.default_rng(3)
    ops = [at.sample_launch(rng)[0] for _ in range(2000)]
    frac = {op: ops.count(op) / len(ops) for op in at.OPS}
    for op, want in zip(at.OPS, (0.40, 0.25, 0.20, 0.15)):
        assert abs(frac[op] - want) < 0.04
    for _ in range(20):
        op, b, m, n, k = at.sample_launch(rng)
        assert 256 <= b <= 8192 and len(m) == b
        assert m.min() >= 4 and m.max() <= 384 and n.max() <= 384
        if op == "geqrf":
            assert (m == 2 * n).all()
        f = at.features(op, b, m, n, k, at.NVAR[op] - 1)
        assert f.shape == (at.NFEAT,) and f[at.OPS.index(op)] == 1 and f[-at.MAXVAR:].sum() == 1
    assert at.NVAR == {"gemm_nt": 6, "potrf_l": 6, "getrf_rp": 6, "geqrf": 6}


def test_flop_counts():
    from blasfeo_b200 import autotune as at
    assert at.flops("gemm_nt", [2], [3], [4]) == 48
    assert at.flops("potrf_l", [3], [3], [3]) == pytest.approx(9 + 4.5 + 0.5)
    assert at.flops("getrf_rp", [3], [3], [3]) == pytest.approx(18 - 4.5 + 2.5)
    assert at.flops("geqrf", [6], [3], [3]) == pytest.approx(108 - 18 + 18 + 9 + 14)


def test_regret_arithmetic():
    from blasfeo_b200 import autotune as at
    recs = [{"times": np.array([2.0, 1.0, 4.0]), "heur": 2.0}, {"times": np.array([3.0, 6.0]), "heur": 3.0}]
    assert at.regret(recs, [1, 0]) == (0.0, 0.0)
    mean, tot = at.regret(recs, [0, -1])
    assert mean == pytest.approx(0.5) and tot == pytest.approx(1 / 4)
