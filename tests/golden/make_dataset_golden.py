"""
Generate tests/golden/dataset_pfvs.npz: a subset of the reference's coni
dataset geometries (tests/data/fixtures.json.gz of the reference, the
geometries whose published PFV set is non-empty, h11 <= 9) as inputs of the
batched pipeline -- kappa, the M-lattice basis, the p-vectors of the coni
cone's box (as the reference's coniZpM enumerates them), Q and the dilation --
with the published primitive PFVs (K, M).  The reference tree is not present
where the GPU tests run; this file carries the dataset there.

    python tests/golden/make_dataset_golden.py
"""
import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pvecs  # noqa: E402
from pfvs_b200 import intlat  # noqa: E402

FIXTURES = os.path.join(os.environ.get("PFVS_REFERENCE", "/root/reference"), "tests", "data", "fixtures.json.gz")


def geometry(g):
    h = g["h11"]
    kappa = np.zeros((h,) * 3, dtype=np.int64)
    for i, j, k, v in g["kappa_coo"]:
        for a, b, c in {(i, j, k), (i, k, j), (j, i, k), (j, k, i), (k, i, j), (k, j, i)}:
            kappa[a, b, c] = v
    Hc = np.array(g["H"], dtype=np.int64)
    Hc = Hc[np.any(Hc != 0, axis=1)]
    Mb = intlat.m_lattice(kappa, np.array(g["c2"]))
    ps = pvecs.box_enum(g["B"], Hc)
    ps = np.hstack([np.zeros((len(ps), 1), np.int64), ps]) if len(ps) else np.zeros((0, h), np.int64)
    return kappa, Mb, ps


def main():
    with gzip.open(FIXTURES) as f:
        F = json.load(f)
    out = {}
    k = 0
    for g in F["geometries"]:
        if not g["K"] or g["h11"] > 9:
            continue
        kappa, Mb, ps = geometry(g)
        h = g["h11"]
        out[f"g{k}_kappa"] = kappa
        out[f"g{k}_Mbasis"] = Mb
        out[f"g{k}_ps"] = ps
        out[f"g{k}_scal"] = np.array([h, h + g["h21"] + 4, 13], dtype=np.int64)    # h11, Q, M0min
        out[f"g{k}_D"] = np.array([float(g["D"])])
        out[f"g{k}_K"] = np.array(g["K"], dtype=np.int64).reshape(-1, h)
        out[f"g{k}_M"] = np.array(g["M"], dtype=np.int64).reshape(-1, h)
        print(k, "h11", h, "p-vectors", len(ps), "published PFVs", len(g["K"]))
        k += 1
    out["n_geometries"] = np.array([k])
    np.savez_compressed(os.path.join(HERE, "dataset_pfvs.npz"), **out)


if __name__ == "__main__":
    main()
