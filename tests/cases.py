"""Seeded instances shared by the parity tests (no I/O, no reference access)."""
import numpy as np

from gpugst_b200 import gen


def tiny_cases(n, seed0=0, vmax=10, emax=16, kmax=4, dmax=4):
    """Tiny random graphs for brute-force checks."""
    out = []
    for seed in range(seed0, seed0 + n):
        rng = np.random.default_rng(seed)
        V = int(rng.integers(4, vmax + 1))
        E = int(rng.integers(V - 1, min(emax, V * (V - 1) // 2) + 1))
        g, gr = gen.small_instance(V, E, n_groups=6, smax=3, seed=seed)
        k = int(rng.integers(1, kmax + 1))
        q = rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32)
        D = int(rng.integers(0, dmax + 1))
        out.append((g, gr, q, D))
    return out


def small_cases(n, seed0=100, V=300, E=1500, n_groups=60, smax=8, kmax=5):
    out = []
    for seed in range(seed0, seed0 + n):
        rng = np.random.default_rng(seed)
        g, gr = gen.small_instance(V, E, n_groups=n_groups, smax=smax, seed=seed)
        k = int(rng.integers(2, kmax + 1))
        q = rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32)
        out.append((g, gr, q))
    return out
