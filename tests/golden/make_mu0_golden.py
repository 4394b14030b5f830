"""
Generate tests/golden/mu0.npz: golden vectors for the coni dilation bound mu0.

From the reference's fixtures (tests/data/fixtures.json.gz of the reference:
the coni dataset geometries with their published PFVs), every PFV's direction
p_hat and dilation delta, recovered from its fluxes alone (K_r = N_rr p_r
with N = kappa . M, p = p_hat / delta, p_hat primitive), as the reference's
tests/test_dilation_bound.py:58-72 does; and for each direction mu0 from the
reference's own C code (oracle/_ref, coni_bound.h:255).  The reference tree
is not present where the GPU tests run; this file carries the cases there.

    python tests/golden/make_mu0_golden.py
"""
import gzip
import json
import math
import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from oracle.mu0 import _solve_exact  # noqa: E402

FIXTURES = os.path.join(os.environ.get("PFVS_REFERENCE", "/root/reference"), "tests", "data", "fixtures.json.gz")


def dense(coo, h):
    kappa = np.zeros((h,) * 3, dtype=np.int64)
    for i, j, k, v in coo:
        for a, b, c in {(i, j, k), (i, k, j), (j, i, k), (j, k, i), (k, i, j), (k, j, i)}:
            kappa[a, b, c] = v
    return kappa


def direction(kappa, K, M):
    """(p_hat, delta numerator, delta denominator) of the PFV (K, M)."""
    h = kappa.shape[0]
    N = [[sum(int(kappa[a, b, c]) * int(M[c]) for c in range(h)) for b in range(h)] for a in range(h)]
    pr = _solve_exact([row[1:] for row in N[1:]], [[int(x) for x in K[1:]]])[0]
    den = 1
    for x in pr:
        den = den * x.denominator // math.gcd(den, x.denominator)
    ints = [int(x * den) for x in pr]
    g = 0
    for x in ints:
        g = math.gcd(g, abs(x))
    p_hat = [0] + [x // g for x in ints]
    return p_hat, den, g


def main():
    with gzip.open(FIXTURES) as f:
        F = json.load(f)
    rows = {"h": [], "Q": [], "gidx": [], "p": [], "delta": [], "mu0": [], "status": []}
    kappas = []
    for gi, g in enumerate(F["geometries"]):
        h = g["h11"]
        if not g["K"]:
            continue
        kappa = dense(g["kappa_coo"], h)
        kappas.append(kappa)
        Q = h + g["h21"] + 4
        for K, M in zip(g["K"], g["M"]):
            p_hat, dn, dd = direction(kappa, K, M)
            st, mu, _ = ref.coni_mu0(kappa, np.array(p_hat[1:], dtype=np.int64))
            rows["h"].append(h)
            rows["Q"].append(Q)
            rows["gidx"].append(len(kappas) - 1)
            rows["p"].append(p_hat + [0] * (64 - h))
            rows["delta"].append((dn, dd))
            rows["mu0"].append((mu.numerator, mu.denominator) if st == 0 else (0, 0))
            rows["status"].append(st)
    out = {k: np.array(v, dtype=np.int64) for k, v in rows.items()}
    for k, kap in enumerate(kappas):
        out[f"kappa{k}"] = kap
    # directions that are not PFV directions (seeded, small entries), so that
    # "no bound" (status 1) and undecided cases of the C code are covered too
    rng = np.random.default_rng(7)
    rnd = {"r_gidx": [], "r_p": [], "r_mu0": [], "r_status": []}
    for k, kap in enumerate(kappas):
        h = kap.shape[0]
        for _ in range(12):
            p_r = rng.integers(-3, 7, size=h - 1)
            if not p_r.any():
                continue
            st, mu, _ = ref.coni_mu0(kap, p_r.astype(np.int64))
            rnd["r_gidx"].append(k)
            rnd["r_p"].append(list(p_r) + [0] * (64 - h))
            rnd["r_mu0"].append((mu.numerator, mu.denominator) if st == 0 else (0, 0))
            rnd["r_status"].append(st)
    out.update({k: np.array(v, dtype=np.int64) for k, v in rnd.items()})
    np.savez_compressed(os.path.join(HERE, "mu0.npz"), **out)
    st = out["status"]
    print(f"{len(st)} PFVs over {len(kappas)} geometries; reference C decided {int(np.sum(st == 0))}, "
          f"no bound {int(np.sum(st == 1))}, undecided {int(np.sum(st < 0))}")
    rs = out["r_status"]
    print(f"{len(rs)} other directions; decided {int(np.sum(rs == 0))}, no bound {int(np.sum(rs == 1))}, "
          f"undecided {int(np.sum(rs < 0))}")


if __name__ == "__main__":
    main()
