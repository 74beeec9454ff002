"""Shared test helpers: the oracle (CPU checker), seeded inputs, error norms."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")


def ensure_oracle():
    so = os.path.join(ORACLE_DIR, "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)
    return so


def oracle_api():
    ensure_oracle()
    from oracle.pyoracle import Api
    return Api("oracle")


def relfro(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def spd(rng, n, shift=1.0):
    g = rng.standard_normal((n, n))
    return g @ g.T / max(n, 1) + shift * np.eye(n)


def tol(prec, s_factor=1):
    """Parity tolerance (relative Frobenius error against the oracle): 1e-13 for
    every FP64 result, the bar of the plain FP64 path; 2e-5 times a per-routine
    factor for FP32 results.  The compiled reference's own HP and REF builds
    differ by at most 1.2e-14 on the FP64 cases these tests use (getrf_rp at
    n = 384 is the largest spread; potrf_l and geqrf stay below 1e-15)."""
    return 1e-13 if prec == "d" else 2e-5 * s_factor
