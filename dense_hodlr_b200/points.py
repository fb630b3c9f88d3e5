"""Seeded synthetic point clouds and the k-d median ordering.

The HODLR tree splits index ranges in half (src/HODLR_Tree.cpp:33-132), so the
points must be ordered so that every index half is a spatial cluster.  The
reference's precedent is rigidBody/MobFunctions.h:335-363 (get_KDTree_Sorted):
recursively sort by coordinate `depth % dim` and split with the left count
floor(N/2).  Its merge step takes the right element on equal keys; ties have
probability zero for continuous random clouds, so a stable sort gives the
same order.
"""
import numpy as np


def kd_order(pts):
    """Return the permutation that k-d median-orders `pts` (dim x n)."""
    pts = np.asarray(pts, dtype=np.float64)
    dim, n = pts.shape
    perm = np.arange(n)
    # iterative version of the recursion: (start, count, depth)
    stack = [(0, n, 0)]
    while stack:
        s, c, d = stack.pop()
        if c <= 1:
            continue
        seg = perm[s:s + c]
        key = pts[d % dim, seg]
        perm[s:s + c] = seg[np.argsort(key, kind="stable")]
        nl = c // 2
        stack.append((s + nl, c - nl, d + 1))
        stack.append((s, nl, d + 1))
    return perm


def uniform_1d_sorted(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(lo, hi, n))[None, :]


def uniform_cube(n, dim, seed):
    """Uniform in [0,1]^dim, k-d ordered, returned SoA (dim x n)."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, (dim, n))
    return np.ascontiguousarray(p[:, kd_order(p)])


def unit_sphere(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((3, n))
    p /= np.linalg.norm(p, axis=0, keepdims=True)
    return np.ascontiguousarray(p[:, kd_order(p)])


def gaussian_mixture(n, seed, components=8, sigma=0.05):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, (3, components))
    lab = rng.integers(0, components, n)
    p = centres[:, lab] + sigma * rng.standard_normal((3, n))
    return np.ascontiguousarray(p[:, kd_order(p)])
