"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

The reference (amiraa127/Dense_HODLR) ships no golden vectors and cannot be
built here (it needs Eigen and CppUnit), so the fixtures are produced by the
oracle restatement after it has passed the reference's own test assertions
(tests/test_oracle.py).

c1_aca.npz  pivots, ranks and iteration counts of the 1D workload: N=4096
            sorted uniform points on [-1,1] (numpy default_rng seed 1),
            K = exp(-(dx)^2/0.1^2) + 1.0*delta, leaf 64, ACA tol 1e-10;
            and per block a hash of the exact FP64 bytes of its W and V.
c2_blocks.npz  per block: level, size, rank, iterations, stopping margin and
            a hash of the pivot sequence, for the FP64-at-scale workload:
            N=262144 uniform [0,1]^2 (dense_hodlr_b200.points.uniform_cube,
            seed 2024), k-d ordered, Matern-3/2 l=0.2 + 1e-2*delta, leaf 128,
            ACA tol 1e-8.  (--c2; several minutes on 8 cores.)
Run from the repository root: python tests/golden/make_golden.py [--c2]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import OracleHODLR  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def pivot_hash(rows, cols):
    """64-bit polynomial hash of a pivot sequence (rows then columns)."""
    h = np.uint64(1469598103934665603)
    mul = np.uint64(1099511628211)
    with np.errstate(over="ignore"):
        for v in np.concatenate([rows, cols, [len(rows)]]).astype(np.int64):
            h = np.uint64((h ^ np.uint64(v & 0xFFFFFFFF)) * mul)
    return np.int64(h.astype(np.int64))


def factor_hash(W, V):
    """First 8 bytes of the SHA-256 of the FP64 bytes of W then V (column-major),
    as a signed 64-bit integer: pins the low-rank factors bit for bit."""
    import hashlib
    d = hashlib.sha256(np.asfortranarray(W).tobytes(order="F")
                       + np.asfortranarray(V).tobytes(order="F")).digest()
    return np.frombuffer(d[:8], dtype=np.int64)[0]


def block_shape(inner, b):
    """(m, n) of block b: 2p is node p's top block, 2p+1 its bottom block."""
    lv, mn, sp, mx = inner[b // 2]
    return (sp - mn + 1, mx - sp) if b % 2 == 0 else (mx - sp, sp - mn + 1)


def c1():
    rng = np.random.default_rng(1)
    pts = np.sort(rng.uniform(-1.0, 1.0, 4096))[None, :]
    o = OracleHODLR.from_kernel(pts, 0, 0.1, shift=1.0, leaf=64)
    o.set_lr(1e-10)
    o.compress()
    nb = o.num_blocks()
    prow = np.concatenate([o.pivots(b)[0] for b in range(nb)])
    pcol = np.concatenate([o.pivots(b)[1] for b in range(nb)])
    inner = o.inner_nodes()
    wv = np.array([factor_hash(*o.lowrank(b, *block_shape(inner, b))) for b in range(nb)],
                  dtype=np.int64)
    out = os.path.join(HERE, "c1_aca.npz")
    np.savez_compressed(out, points=pts[0], ranks=o.ranks(), iters=o.iters(), prow=prow,
                        pcol=pcol, wv_hash=wv)
    print(out, "blocks", nb, "pivots", len(prow))


def c2():
    from dense_hodlr_b200.points import uniform_cube
    pts = uniform_cube(262144, 2, 2024)
    o = OracleHODLR.from_kernel(pts, 1, 0.2, shift=1e-2, leaf=128)
    o.set_lr(1e-8)
    o.compress()
    inner = o.inner_nodes()
    nb = o.num_blocks()
    level, m, n, hashes = [], [], [], []
    for b in range(nb):
        lv, mn, sp, mx = inner[b // 2]
        level.append(lv)
        if b % 2 == 0:
            m.append(sp - mn + 1)
            n.append(mx - sp)
        else:
            m.append(mx - sp)
            n.append(sp - mn + 1)
        r, c = o.pivots(b)
        hashes.append(pivot_hash(r, c))
    out = os.path.join(HERE, "c2_blocks.npz")
    np.savez_compressed(out, level=np.array(level, np.int32), m=np.array(m, np.int32),
                        n=np.array(n, np.int32), rank=o.ranks(), iters=o.iters(),
                        margin=o.margins(), pivot_hash=np.array(hashes, np.int64),
                        points_sum=np.array([pts.sum(), (pts * pts).sum()]))
    print(out, "blocks", nb, "max rank", o.ranks().max())


if __name__ == "__main__":
    if "--c2" in sys.argv:
        c2()
    else:
        c1()
