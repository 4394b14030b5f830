"""
Generate tests/golden/*.npz: points of the reference's own CPU kernel
(oracle/_ref, compiled from the reference sources by oracle/Makefile) on
seeded subsets of the synthetic workloads, in the canonical order
(pidx, M, Kn).  The reference tree is not present where the GPU tests run;
these files carry its answers there.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from pfvs_b200 import workloads  # noqa: E402
from parity import expected, layout  # noqa: E402

CASES = {
    "small_dil150": ("small", 128, (150.0,)),
    "small_dil5000": ("small", 64, (5000.0,)),
    "plain_dil150": ("plain", 96, (150.0,)),
    "plain_dil800": ("plain", 32, (800.0,)),
    "mixed": ("mixed", 96, None),
    "precision": ("precision", 8, None),
}


def main():
    for key, (name, n, dils) in CASES.items():
        w = workloads.build(name, n_p=n, dilations=dils)
        geoms, ps, pgeo, hs = layout(w)
        M, Kn, q, pidx, status = expected(geoms, ps, pgeo, "ref")
        hmax = max(hs)
        np.savez_compressed(os.path.join(HERE, f"{key}.npz"), M=M[:, :hmax], Kn=Kn[:, :hmax], q=q,
                            pidx=pidx, status=status, workload=name, n=n,
                            dilations=np.array(dils if dils else [], dtype=float))
        print(key, len(q), "points", int(np.sum(status == 0)), "/", len(status), "directions done")


if __name__ == "__main__":
    main()
