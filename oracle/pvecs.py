"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

The p-vector box used by the reference's dataset and GPU tests
(tests/test_dataset.py:59-63, tests/test_gpu.py:37-41, via the third-party
`latticepts.box_enum(B, H, 1, N, primitive=True)`, latticepts >= 0.1.2, not
installed here): every primitive integer p with |p|_inf <= B and H p >= 1
(row-wise).  Restated as a depth-first search over the coordinates that
prunes a prefix once some row can no longer reach 1 with the remaining
coordinates in [-B, B].  Returned in lexicographic order.
"""
import math

import numpy as np


def box_enum(B, H):
    H = np.asarray(H, dtype=np.int64)
    r, n = H.shape
    # suffix bound: max over the remaining coordinates of sum_j H_rj p_j
    absH = np.abs(H)
    tail = np.zeros((n + 1, r), dtype=np.int64)
    for j in range(n - 1, -1, -1):
        tail[j] = tail[j + 1] + absH[:, j] * B
    out = []
    p = [0] * n

    def rec(j, acc):
        if np.any(acc + tail[j] < 1):
            return
        if j == n:
            if math.gcd(*p) == 1:
                out.append(list(p))
            return
        for v in range(-B, B + 1):
            p[j] = v
            rec(j + 1, acc + H[:, j] * v)
        p[j] = 0

    rec(0, np.zeros(r, dtype=np.int64))
    return np.array(out, dtype=np.int64).reshape(-1, n)
