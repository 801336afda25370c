"""Shared helpers for the test-suite: seeded inputs and golden-fixture access."""
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden():
    z = np.load(GOLDEN / "shtns37_hotpath.npz")
    meta = json.loads((GOLDEN / "shtns37_hotpath.json").read_text())
    return z, meta


def rand_alm(lmax, mmax, nf=None, seed=0, power=1.0, mres=1, lmin=0):
    """Complex coefficients ~ N(0,1)/(l+1)^power, imag = 0 at m = 0, zero for l < m."""
    rng = np.random.default_rng(seed)
    shape = (lmax + 1, mmax + 1) + (() if nf is None else (nf,))
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    l = np.arange(lmax + 1).reshape((-1, 1) + (() if nf is None else (1,)))
    a = a / (l + 1.0) ** power
    a[:, 0, ...] = a[:, 0, ...].real
    for m in range(mmax + 1):
        a[:m, m, ...] = 0
        if m % mres:
            a[:, m, ...] = 0
    a[:lmin] = 0
    return a


def isapprox(a, b, atol, rtol):
    """Julia's isapprox on arrays: norm(a-b) <= max(atol, rtol*max(norm(a), norm(b)))."""
    a, b = np.asarray(a), np.asarray(b)
    d = np.linalg.norm((a - b).ravel())
    return d <= max(atol, rtol * max(np.linalg.norm(a.ravel()), np.linalg.norm(b.ravel())))


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    n = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0))
