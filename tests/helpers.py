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
