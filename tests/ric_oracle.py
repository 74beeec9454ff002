"""Riccati recursion of examples/example_d_riccati_recursion.c restated on
host panel-major storage through a CPU API (the oracle restatement, or the
compiled reference itself): the factorization d_back_ric_trf_libstr (:115-143)
and the solve d_back_ric_trs_libstr (:203-270), plus the KKT residual of the
LQ problem they solve.  TEST INFRASTRUCTURE ONLY (the checker of the GPU
Riccati kernels).

Problem (one of the batch), stages k = 0..N-1 with nu inputs and nx states,
stage N with nx states only:
  min  sum_k 1/2 [u;x]_k^T RSQ_k [u;x]_k + rq_k^T [u;x]_k + 1/2 x_N^T Q_N x_N + q_N^T x_N
  s.t. x_{k+1} = BAbt_k^T [u;x]_k + b_k,
BAbt_k = [B_k^T; A_k^T] ((nu+nx) x nx), RSQ_k = [[R, S^T], [S, Q]]; x_0 is free.
"""
import numpy as np

from oracle.pyoracle import HostMat, HostVec


def ric_trf(api, BA, RSQ, N, nx, nu):
    """Factors L_k (list of HostMat, L_N nx x nx, the others (nu+nx) x (nu+nx))."""
    m = nu + nx
    L = [None] * (N + 1)
    hQ, hL = HostMat(nx, nx).set(RSQ[N][:nx, :nx]), HostMat(nx, nx)
    api.potrf_l("d", nx, hQ, 0, 0, hL, 0, 0)
    L[N] = hL
    for k in range(N - 1, -1, -1):
        off = 0 if k + 1 == N else nu
        hBA, hW = HostMat(m, nx).set(BA[k][:m]), HostMat(m, nx)
        hR, hLk = HostMat(m, m).set(RSQ[k][:m, :m]), HostMat(m, m)
        api.trmm_rlnn("d", m, nx, 1.0, L[k + 1], off, off, hBA, 0, 0, hW, 0, 0)
        api.syrk_potrf_ln("d", m, nx, hW, 0, 0, hW, 0, 0, hR, 0, 0, hLk, 0, 0)
        L[k] = hLk
    return L


def ric_trs(api, L, BA, b, rq, N, nx, nu):
    """d_back_ric_trs_libstr: ux_k = [u_k; x_k] (k < N, length nu+nx), ux_N = x_N,
    pi_k (k < N, length nx); returns (list of ux arrays, list of pi arrays)."""
    m = nu + nx
    nuv = [nu] * N + [0]
    nxv = [nx] * (N + 1)
    hBA = [HostMat(m, nx).set(BA[k][:m]) for k in range(N)]
    hb = [HostVec(nx).set(b[k][:nx]) for k in range(N)]
    ux = [HostVec(nuv[k] + nxv[k]).set(rq[k][:nuv[k] + nxv[k]]) for k in range(N + 1)]
    pi = [HostVec(nx) for _ in range(N)]
    Pb = [HostVec(nx) for _ in range(N)]
    w = HostVec(nx)
    # backward substitution
    for k in range(N - 1, -1, -1):
        o = nuv[k + 1]
        api.trmv_ltn("d", nx, L[k + 1], o, o, hb[k], 0, Pb[k], 0)
        api.trmv_lnn("d", nx, L[k + 1], o, o, Pb[k], 0, Pb[k], 0)
        w.set(Pb[k].get() + ux[k + 1].get()[o:o + nx])
        api.gemv_n("d", m, nx, 1.0, hBA[k], 0, 0, w, 0, 1.0, ux[k], 0, ux[k], 0)
        if k > 0:
            api.trsv_lnn_mn("d", m, nu, L[k], 0, 0, ux[k], 0, ux[k], 0)
        else:
            api.trsv_lnn("d", m, L[k], 0, 0, ux[k], 0, ux[k], 0)
    # forward substitution
    for k in range(N):
        o = nuv[k + 1]
        pi[k].set(ux[k + 1].get()[o:o + nx])
        v = ux[k].get()
        if k == 0:
            ux[k].set(-v)
            api.trsv_ltn("d", m, L[k], 0, 0, ux[k], 0, ux[k], 0)
        else:
            v[:nu] = -v[:nu]
            ux[k].set(v)
            api.trsv_ltn_mn("d", m, nu, L[k], 0, 0, ux[k], 0, ux[k], 0)
        nxt = HostVec(nx)
        api.gemv_t("d", m, nx, 1.0, hBA[k], 0, 0, ux[k], 0, 1.0, hb[k], 0, nxt, 0)
        full = ux[k + 1].get()
        full[o:o + nx] = nxt.get()
        ux[k + 1].set(full)
        w.set(nxt.get())
        api.trmv_ltn("d", nx, L[k + 1], o, o, w, 0, w, 0)
        api.trmv_lnn("d", nx, L[k + 1], o, o, w, 0, w, 0)
        pi[k].set(pi[k].get() + w.get())
    return [u.get() for u in ux], [p.get() for p in pi]


def kkt_residual(BA, RSQ, b, rq, ux, pi, N, nx, nu):
    """Stationarity and dynamics residuals of the LQ problem (numpy, FP64):
    RSQ_k ux_k + rq_k + BAbt_k pi_k - [0; pi_{k-1}] (k < N), Q_N x_N + q_N - pi_{N-1},
    BAbt_k^T ux_k + b_k - x_{k+1}."""
    m = nu + nx
    rs, rd = [], []
    for k in range(N + 1):
        if k < N:
            R = np.tril(RSQ[k][:m, :m]) + np.tril(RSQ[k][:m, :m], -1).T
            r = R @ ux[k][:m] + rq[k][:m] + BA[k][:m] @ pi[k]
            if k > 0:
                r[nu:] -= pi[k - 1]
        else:
            Q = np.tril(RSQ[N][:nx, :nx]) + np.tril(RSQ[N][:nx, :nx], -1).T
            r = Q @ ux[N][:nx] + rq[N][:nx] - pi[N - 1]
        rs.append(r)
        if k < N:
            xn = ux[k + 1][nu:nu + nx] if k + 1 < N else ux[k + 1][:nx]
            rd.append(BA[k][:m].T @ ux[k][:m] + b[k][:nx] - xn)
    return rs, rd
