"""
Generate tests/golden/zpk.npz: golden vectors for coniZpK above D0.

For the 30 dataset geometries of tests/golden/dataset_pfvs.npz (kappa, Mbasis,
Q, M0min and their PFV directions), the first 8 directions each, and D0 in
(20, 150): the reference's own C kernel's lattice points and statuses
(oracle/_ref: czk_batch, pfvs/fp_kernel/coni_zpk.h:714) and the PFVs the
reference's coniZpK makes of them (pfvs/coni.py:612-631: the post-processing
restated in oracle/postproc.py, then dilation > D0, once each, sorted).  The
reference tree is not present where the GPU tests run; this file carries the
cases there.

    make -C oracle ref && python tests/golden/make_zpk_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import postproc, ref  # noqa: E402

D0S = (20, 150)
PER_GEO = 8


def _sorted_rows(*cols):
    n = len(cols[0])
    if n == 0:
        return np.zeros((0, sum(1 if np.ndim(c) == 1 else np.shape(c)[1] for c in cols)), dtype=np.int64)
    A = np.hstack([np.asarray(c, dtype=np.int64).reshape(n, -1) for c in cols])
    return A[np.lexsort(A.T[::-1])] if len(A) else A


def _dilation_above(kappa, p, K, M, D0):
    Z = np.tensordot(np.asarray(kappa).astype(object), np.asarray(p).astype(object), axes=([2], [0]))
    ZM = Z @ np.asarray(M).astype(object)
    num = math.gcd(*[int(x) for x in ZM[1:]])
    den = math.gcd(*[int(x) for x in np.asarray(K)[1:]])
    return num > D0 * den


def main():
    D = np.load(os.path.join(HERE, "dataset_pfvs.npz"))
    n_geo = len([k for k in D.files if k.endswith("_kappa")])
    out = {"d0s": np.array(D0S, dtype=np.int64)}
    for g in range(n_geo):
        kappa, Mb, scal = D[f"g{g}_kappa"], D[f"g{g}_Mbasis"], D[f"g{g}_scal"]
        h, Q, M0min = (int(x) for x in scal)
        ps = D[f"g{g}_ps"][:PER_GEO]
        out[f"g{g}_ps"] = ps
        for D0 in D0S:
            M, Kn, q, pidx, st = ref.coni_zpk_batch(kappa, Mb, ps, Q, M0min, D0)
            assert np.all(st == 0), (g, D0, st)
            out[f"g{g}_d{D0}_points"] = _sorted_rows(pidx, M, Kn, q)
            out[f"g{g}_d{D0}_status"] = st.astype(np.int32)
            Ks, Ms, keys = postproc.pfvs_from_points(M, Kn, q, pidx, kappa, h, Q, M0min)
            keep = [_dilation_above(kappa, ps[k], K, Mm, D0) for K, Mm, k in zip(Ks, Ms, keys)]
            keep = np.array(keep, dtype=bool)
            rows = _sorted_rows(np.asarray(keys)[keep], np.asarray(Ms).reshape(-1, h)[keep],
                                np.asarray(Ks).reshape(-1, h)[keep])
            out[f"g{g}_d{D0}_pfvs"] = np.unique(rows, axis=0) if len(rows) else np.zeros((0, 1 + 2 * h), np.int64)
        print(g, h, len(ps), [len(out[f"g{g}_d{D0}_points"]) for D0 in D0S],
              [len(out[f"g{g}_d{D0}_pfvs"]) for D0 in D0S])
    np.savez_compressed(os.path.join(HERE, "zpk.npz"), **out)


if __name__ == "__main__":
    main()
