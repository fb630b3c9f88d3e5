"""Generate tests/golden/c1_aca.npz from the CPU oracle.

The reference (amiraa127/Dense_HODLR) ships no golden vectors and cannot be
built here (it needs Eigen and CppUnit), so the C1 fixture is produced by the
oracle restatement after it has passed the reference's own test assertions
(tests/test_oracle.py).  It pins the pivots, ranks and iteration counts of
the C1 workload: N=4096 sorted uniform points on [-1,1] (numpy default_rng
seed 1), K = exp(-(dx)^2/0.1^2) + 1.0*delta, leaf 64, ACA tol 1e-10.
Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import OracleHODLR  # noqa: E402


def main():
    rng = np.random.default_rng(1)
    pts = np.sort(rng.uniform(-1.0, 1.0, 4096))[None, :]
    o = OracleHODLR.from_kernel(pts, 0, 0.1, shift=1.0, leaf=64)
    o.set_lr(1e-10)
    o.compress()
    nb = o.num_blocks()
    prow = np.concatenate([o.pivots(b)[0] for b in range(nb)])
    pcol = np.concatenate([o.pivots(b)[1] for b in range(nb)])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c1_aca.npz")
    np.savez_compressed(out, points=pts[0], ranks=o.ranks(), iters=o.iters(), prow=prow,
                        pcol=pcol)
    print(out, "blocks", nb, "pivots", len(prow))


if __name__ == "__main__":
    main()
