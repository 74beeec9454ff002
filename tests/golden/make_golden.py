"""Generate the golden fixtures from the COMPILED REFERENCE (BLASFEO 0.1.4.2).

Run in a container where the reference sources are present:
    make -C oracle generic haswell        # builds oracle/_ref/*.so from the reference tree
    python tests/golden/make_golden.py    # all fixtures; or name files: ... make_golden.py adjacent.npz

Every output stored here comes from the reference library itself (its
LA=HIGH_PERFORMANCE panel-major routines ``blasfeo_*``, TARGET=GENERIC so the
single-precision layout is the ps=4 one used on the device), called on the
seeded inputs that are stored next to them.  The oracle restatement and the GPU
kernels are both checked against these files (the oracle in
tests/test_oracle.py; the GPU kernels in tests/test_gpu_chain.py,
tests/test_gpu_riccati.py and tests/test_gpu_adjacent.py);
tests/golden/manifest.json records their SHA-256.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Api, HostMat, HostVec  # noqa: E402

NP = {"d": np.float64, "s": np.float32}


def ref_api(target="generic"):
    return Api("hp", target)


def testx_inputs(n=60):
    """tests/test_x.c:144-169 fixtures: A[i]=i+1 (column-major), A_ii += 1,
    B[i]=2(i+1), C[i]=0.5(i+1), A_po = A A^T + (1e6+i) I."""
    idx = np.arange(n * n, dtype=np.float64)
    A = (idx + 1).reshape(n, n, order="F")
    A[np.arange(n), np.arange(n)] += 1
    B = (2 * (idx + 1)).reshape(n, n, order="F")
    C = (0.5 * (idx + 1)).reshape(n, n, order="F")
    Apo = A @ A.T
    Apo[np.arange(n), np.arange(n)] += 1e6 + np.arange(n)
    return A, B, C, Apo


def run_testx(api, prec, n=60):
    A, B, C, Apo = testx_inputs(n)
    out = {}
    h = lambda X: HostMat(n, n, NP[prec]).set(X)
    hA, hB, hC, hD = h(A), h(B), h(C), HostMat(n, n, NP[prec])
    api.gemm_nt(prec, n, n, n, 1.0, hA, 0, 0, hB, 0, 0, 1.0, hC, 0, 0, hD, 0, 0)
    out["gemm_nt"] = hD.get()
    hD = h(np.zeros((n, n)))
    api.syrk_ln(prec, n, n, 1.0, hA, 0, 0, hA, 0, 0, 1.0, hC, 0, 0, hD, 0, 0)
    out["syrk_ln"] = np.tril(hD.get())
    hP, hL = h(Apo), HostMat(n, n, NP[prec])
    api.potrf_l(prec, n, hP, 0, 0, hL, 0, 0)
    out["potrf_l"] = np.tril(hL.get())
    out["potrf_l_dA"] = hL.diag(n)
    hX = HostMat(n, n, NP[prec])
    api.trsm_rltn(prec, n, n, 1.0, hL, 0, 0, hB, 0, 0, hX, 0, 0)
    out["trsm_rltn"] = hX.get()
    hLU = HostMat(n, n, NP[prec])
    out["getrf_rp_ipiv"] = api.getrf_rp(prec, n, n, hA, 0, 0, hLU, 0, 0)
    out["getrf_rp"] = hLU.get()
    hQ = HostMat(n, n, NP[prec])
    api.geqrf(prec, n, n, hP, 0, 0, hQ, 0, 0)
    out["geqrf"] = hQ.get()
    out["geqrf_tau"] = hQ.diag(n)
    return out


def cfg1(api):
    """64x64 single-instance chain, seed 0: gemm_nt (U[-1,1], C=0, alpha=1,
    beta=0), potrf_l of G G^T/64 + I, trsm_rltn of an N(0,1) RHS."""
    rng = np.random.default_rng(0)
    n = 64
    A = rng.uniform(-1, 1, (n, n))
    B = rng.uniform(-1, 1, (n, n))
    G = rng.standard_normal((n, n))
    S = G @ G.T / n + np.eye(n)
    R = rng.standard_normal((n, n))
    h = lambda X: HostMat(n, n).set(X)
    hA, hB, hC, hD = h(A), h(B), h(np.zeros((n, n))), HostMat(n, n)
    api.gemm_nt("d", n, n, n, 1.0, hA, 0, 0, hB, 0, 0, 0.0, hC, 0, 0, hD, 0, 0)
    hS, hL = h(S), HostMat(n, n)
    api.potrf_l("d", n, hS, 0, 0, hL, 0, 0)
    hR, hX = h(R), HostMat(n, n)
    api.trsm_rltn("d", n, n, 1.0, hL, 0, 0, hR, 0, 0, hX, 0, 0)
    return {"A": A, "B": B, "S": S, "R": R, "D": hD.get(), "L": np.tril(hL.get()), "L_dA": hL.diag(n),
            "X": hX.get()}


def cfg2(api, num=16):
    """Uniform n=16 chain per instance: S = A A^T + 16 I (syrk 16x32, ddiare),
    L = chol(S), X = R L^{-T}, D = C - X G^T (dgemm_nt 16x16x16)."""
    rng = np.random.default_rng(2)
    m, k = 16, 32
    A = rng.standard_normal((num, m, k))
    R = rng.standard_normal((num, m, m))
    C = rng.standard_normal((num, m, m))
    G = rng.standard_normal((num, m, m))
    L, X, D = np.zeros((num, m, m)), np.zeros((num, m, m)), np.zeros((num, m, m))
    for b in range(num):
        hA, hS = HostMat(m, k).set(A[b]), HostMat(m, m)
        api.syrk_ln("d", m, k, 1.0, hA, 0, 0, hA, 0, 0, 0.0, hS, 0, 0, hS, 0, 0)
        api.lib.blasfeo_ddiare.argtypes = None
        import ctypes as Ct
        api.lib.blasfeo_ddiare(m, Ct.c_double(16.0), hS.ref, 0, 0)
        hL = HostMat(m, m)
        api.potrf_l("d", m, hS, 0, 0, hL, 0, 0)
        hR, hX = HostMat(m, m).set(R[b]), HostMat(m, m)
        api.trsm_rltn("d", m, m, 1.0, hL, 0, 0, hR, 0, 0, hX, 0, 0)
        hC, hG, hD = HostMat(m, m).set(C[b]), HostMat(m, m).set(G[b]), HostMat(m, m)
        api.gemm_nt("d", m, m, m, -1.0, hX, 0, 0, hG, 0, 0, 1.0, hC, 0, 0, hD, 0, 0)
        L[b], X[b], D[b] = np.tril(hL.get()), hX.get(), hD.get()
    return {"A": A, "R": R, "C": C, "G": G, "L": L, "X": X, "D": D}


def spd_systems(rng, ns, logcond=6.0):
    mats, rhs = [], []
    for n in ns:
        q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        lam = 10.0 ** rng.uniform(0, logcond, n)
        a = (q * lam) @ q.T
        mats.append(0.5 * (a + a.T))
        rhs.append(rng.standard_normal(n))
    return mats, rhs


def cfg3(api):
    """Uneven SPD systems (cond up to 1e6), x by dpotrf_l + dtrsv_lnn + dtrsv_ltn."""
    rng = np.random.default_rng(3)
    ns = [4, 5, 7, 9, 13, 16, 17, 23, 31, 33, 40, 48]
    mats, rhs = spd_systems(rng, ns)
    out = {"ns": np.array(ns)}
    for i, (n, a, b) in enumerate(zip(ns, mats, rhs)):
        hA, hL = HostMat(n, n).set(a), HostMat(n, n)
        api.potrf_l("d", n, hA, 0, 0, hL, 0, 0)
        hb, hy, hx = HostVec(n).set(b), HostVec(n), HostVec(n)
        api.trsv_lnn("d", n, hL, 0, 0, hb, 0, hy, 0)
        api.trsv_ltn("d", n, hL, 0, 0, hy, 0, hx, 0)
        out["A%d" % i], out["b%d" % i], out["L%d" % i], out["x%d" % i] = a, b, np.tril(hL.get()), hx.get()
    return out


def riccati_problem(rng, nx=12, nu=4):
    """A = I + 0.1 N(0,1) scaled to spectral radius 0.95, B ~ N(0,1)/sqrt(nx)."""
    A = np.eye(nx) + 0.1 * rng.standard_normal((nx, nx))
    A *= 0.95 / np.max(np.abs(np.linalg.eigvals(A)))
    B = rng.standard_normal((nx, nu)) / np.sqrt(nx)
    return A, B


def riccati_ref(api, A, B, N=30):
    """examples/example_d_riccati_recursion.c:115-143 (d_back_ric_trf_libstr):
    L_N = chol(P_N); per stage work = BAbt * Lxx_{k+1} (dtrmm_rlnn), then
    L_k = chol(RSQ + work work^T) (dsyrk_dpotrf_ln).  Q = I, R = I, S = 0, P_N = I."""
    nx, nu = A.shape[0], B.shape[1]
    m = nu + nx
    BAbt = np.vstack([B.T, A.T])
    RSQ = np.eye(m)
    hBA = HostMat(m, nx).set(BAbt)
    hRSQ = HostMat(m, m).set(RSQ)
    Ls = [None] * (N + 1)
    hLN = HostMat(nx, nx)
    api.potrf_l("d", nx, HostMat(nx, nx).set(np.eye(nx)), 0, 0, hLN, 0, 0)
    Lprev, off = hLN, 0
    Ls[N] = np.tril(hLN.get())
    for k in range(N - 1, -1, -1):
        hW, hL = HostMat(m, nx), HostMat(m, m)
        api.trmm_rlnn("d", m, nx, 1.0, Lprev, off, off, hBA, 0, 0, hW, 0, 0)
        api.syrk_potrf_ln("d", m, nx, hW, 0, 0, hW, 0, 0, hRSQ, 0, 0, hL, 0, 0)
        Ls[k] = np.tril(hL.get())
        Lprev, off = hL, nu
    return Ls


def cfg4(api, num=2):
    rng = np.random.default_rng(4)
    out = {}
    for p in range(num):
        A, B = riccati_problem(rng)
        Ls = riccati_ref(api, A, B)
        out["A%d" % p], out["B%d" % p] = A, B
        out["L%d" % p] = np.stack([np.pad(L, ((0, 16 - L.shape[0]), (0, 16 - L.shape[1]))) for L in Ls])
    return out


def cfg4_trs(api, num=2):
    """The LQ solve of examples/example_d_riccati_recursion.c:203-270
    (d_back_ric_trs_libstr) on the factors of :115-143, through the compiled
    reference's level-2 routines (dtrmv_ltn/lnn, dgemv_n/t, dtrsv_lnn/ltn and
    their _mn forms): config-4 dynamics (as cfg4), Q = R = I, S = 0, P_N = I,
    linear terms rq_k ~ N(0,1) and b_k ~ N(0,1), N = 30, nx = 12, nu = 4."""
    from tests.ric_oracle import ric_trf, ric_trs
    rng = np.random.default_rng(44)
    N, nx, nu = 30, 12, 4
    m = nx + nu
    out = {}
    for p in range(num):
        A, B = riccati_problem(rng)
        BA = np.zeros((N, 16, nx))
        BA[:, :m] = np.vstack([B.T, A.T])
        RSQ = np.broadcast_to(np.eye(16), (N + 1, 16, 16)).copy()
        b = np.zeros((N, 16))
        b[:, :nx] = rng.standard_normal((N, nx))
        rq = np.zeros((N + 1, 16))
        rq[:N, :m] = rng.standard_normal((N, m))
        rq[N, :nx] = rng.standard_normal(nx)
        L = ric_trf(api, BA, RSQ, N, nx, nu)
        ux, pi = ric_trs(api, L, BA, b, rq, N, nx, nu)
        out["BA%d" % p], out["b%d" % p], out["rq%d" % p] = BA, b, rq
        out["ux%d" % p] = np.stack([np.pad(u, (0, 16 - len(u))) for u in ux])
        out["pi%d" % p] = np.stack(pi)
    return out


def cfg5(api):
    """A few ops of the mixed stream (log-uniform sizes 4..384): getrf_rp on
    N(0,1) square matrices (pivots), geqrf on tall m = 2n."""
    rng = np.random.default_rng(5)
    out = {}
    for i, n in enumerate([5, 11, 27, 64]):
        M = rng.standard_normal((n, n))
        hM, hD = HostMat(n, n).set(M), HostMat(n, n)
        out["lu_ipiv%d" % i] = api.getrf_rp("d", n, n, hM, 0, 0, hD, 0, 0)
        out["lu_in%d" % i], out["lu%d" % i], out["lu_dA%d" % i] = M, hD.get(), hD.diag(n)
    for i, n in enumerate([3, 8, 21, 40]):
        M = rng.standard_normal((2 * n, n))
        hM, hD = HostMat(2 * n, n).set(M), HostMat(2 * n, n)
        api.geqrf("d", 2 * n, n, hM, 0, 0, hD, 0, 0)
        out["qr_in%d" % i], out["qr%d" % i], out["qr_tau%d" % i] = M, hD.get(), hD.diag(n)
    return out


def adjacent(api):
    """The adjacent variants (zero offsets, which the HP routines take directly):
    syrk_ln_mn on a 23 x 13 trapezoid (k = 9), trsm_rltu with a unit lower
    factor, potrf_l_mn of a 23 x 13 trapezoid of an SPD matrix, getrf_np of a
    diagonally dominant matrix (square and 17 x 11), both precisions."""
    rng = np.random.default_rng(8)
    out = {}
    for prec in ("d", "s"):
        m, n, k = 23, 13, 9
        A, B, Cm = rng.standard_normal((m, k)), rng.standard_normal((n, k)), rng.standard_normal((m, n))
        hA, hB, hC, hD = (HostMat(m, k, NP[prec]).set(A), HostMat(n, k, NP[prec]).set(B),
                          HostMat(m, n, NP[prec]).set(Cm), HostMat(m, n, NP[prec]))
        api.syrk_ln_mn(prec, m, n, k, 0.5, hA, 0, 0, hB, 0, 0, -1.5, hC, 0, 0, hD, 0, 0)
        out[prec + "_syrkmn_A"], out[prec + "_syrkmn_B"], out[prec + "_syrkmn_C"] = A, B, Cm
        out[prec + "_syrkmn_D"] = hD.get()
        Lu = np.tril(rng.standard_normal((n, n)), -1) * 0.3 + np.eye(n) * 7.0   # diagonal must not be read
        X = rng.standard_normal((m, n))
        hL, hX, hY = HostMat(n, n, NP[prec]).set(Lu), HostMat(m, n, NP[prec]).set(X), HostMat(m, n, NP[prec])
        api.trsm_rltu(prec, m, n, 1.25, hL, 0, 0, hX, 0, 0, hY, 0, 0)
        out[prec + "_trsmu_L"], out[prec + "_trsmu_X"], out[prec + "_trsmu_Y"] = Lu, X, hY.get()
        g = rng.standard_normal((m, m))
        S = g @ g.T + m * np.eye(m)
        hS, hP = HostMat(m, m, NP[prec]).set(S), HostMat(m, m, NP[prec])
        api.potrf_l_mn(prec, m, n, hS, 0, 0, hP, 0, 0)
        out[prec + "_potrfmn_S"], out[prec + "_potrfmn_L"], out[prec + "_potrfmn_dA"] = S, hP.get(), hP.diag(n)
        for tag, (r, c) in (("sq", (15, 15)), ("rect", (17, 11))):
            M = rng.standard_normal((r, c)) + 4.0 * np.eye(r, c) * max(r, c) ** 0.5
            hM, hLU = HostMat(r, c, NP[prec]).set(M), HostMat(r, c, NP[prec])
            api.getrf_np(prec, r, c, hM, 0, 0, hLU, 0, 0)
            out[prec + "_lunp_%s_in" % tag], out[prec + "_lunp_%s" % tag] = M, hLU.get()
            out[prec + "_lunp_%s_dA" % tag] = hLU.diag(min(r, c))
    return out


def main(only=None):
    api = ref_api("generic")
    gens = {"cfg1.npz": cfg1, "cfg2.npz": cfg2, "cfg3.npz": cfg3, "cfg4.npz": cfg4, "cfg5.npz": cfg5,
            "adjacent.npz": adjacent, "cfg4_trs.npz": cfg4_trs}
    files = {}
    if only is None:
        for prec in ("d", "s"):
            files["testx_%s.npz" % prec] = run_testx(api, prec)
    for name, fn in gens.items():
        if only is None or name in only:
            files[name] = fn(api)
    mpath = os.path.join(HERE, "manifest.json")
    if only is None or not os.path.exists(mpath):
        manifest = {"generator": "tests/golden/make_golden.py", "reference": "BLASFEO 0.1.4.2 HP panel-major, "
                    "TARGET=GENERIC (oracle/Makefile)", "files": {}}
    else:
        manifest = json.load(open(mpath))
    for name, d in files.items():
        path = os.path.join(HERE, name)
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        manifest["files"][name] = hashlib.sha256(open(path, "rb").read()).hexdigest()
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote", ", ".join(sorted(files)))


if __name__ == "__main__":
    # optional arguments: only these fixture files (the others and their hashes stay as they are)
    main(sys.argv[1:] or None)
