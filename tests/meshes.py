"""Seeded synthetic meshes and fields shared by the tests (host only)."""
import numpy as np


def vertices(dim, n, lo=(0, 0, 0), hi=(1, 1, 1), distort=0.0, seed=20261203):
    """Lexicographic vertex coordinates; interior vertices moved by a uniform
    offset of +-distort*h per axis."""
    n = list(n)[:dim]
    axes = [np.linspace(lo[d], hi[d], n[d] + 1) for d in range(dim)]
    grid = np.meshgrid(*axes[::-1], indexing="ij")[::-1]
    X = np.stack([g.reshape(-1) for g in grid], axis=1)
    if distort:
        rng = np.random.default_rng(seed)
        h = np.array([(hi[d] - lo[d]) / n[d] for d in range(dim)])
        idx = np.stack(np.meshgrid(*[np.arange(k + 1) for k in n[::-1]], indexing="ij")[::-1], axis=-1).reshape(-1, dim)
        interior = np.all((idx > 0) & (idx < np.array(n)), axis=1)
        off = rng.uniform(-distort, distort, size=X.shape) * h
        X[interior] += off[interior]
    return X


def log_uniform(n, lo, hi, seed=7):
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), size=n)


def random_block_vector(nt, mesh_nodes, boundary_mask, seed=11):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((nt, mesh_nodes))
    v[:, boundary_mask] = 0.0
    return v.reshape(-1)


def boundary_mask(dim, n, p):
    nn = [k * p + 1 for k in list(n)[:dim]]
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in nn[::-1]], indexing="ij")[::-1], axis=-1).reshape(-1, dim)
    return np.any((idx == 0) | (idx == np.array(nn) - 1), axis=1)
