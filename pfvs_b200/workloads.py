"""
Seeded synthetic Calabi-Yau instances and p-hat directions for the batched
coniZpM search (the reference publishes no benchmark suite for this path;
these stand in for it).

Five named workloads follow the shapes of the benchmark configurations:

  name        h11           h21        #p      p entries  dilation      x_a rows
  small       5             60         256     [1, 6]     1             8, 1-3 ones
  plain       11            120        4096    [1, 8]     1             8, 1-4 ones
  mixed       8/16/24/32    2 h11+40   65536   [1, 10]    {1,2,3,4}     8, 1-4 ones
  precision   40            150        16384   [1, 12]    2             8, 1-4 ones
  large       60            200        4096    [1, 16]    1             70, 1-5 ones

Q = h11 + h21 + 2, M0min = 13, H = I (the orthant), coni curve e0 (so the
coni change of basis is the identity and p-hat = (0, p_1, ..., p_{h11-1})).

The triple intersection numbers.  A sum of positive rank-one cubes
sum_a w_a x_a^(x)3 (w_a > 0, x_a 0/1) makes kappa.p positive semidefinite
for p >= 0, so it can never have the signature (1, h11-1) that makes the
ellipsoid matrix -Binter^T (kappa.p) Binter positive definite.  The cubes are
therefore signed, Lorentzian like a Kahler cone's intersection form:

    kappa = w0 J  -  sum_{i>=1} s_i e_i^(x)3  -  sum_a w_a x_a^(x)3

with J the all-ones cube, w0 in {2, 4}, one negative singleton cube per
non-coni coordinate (s_i odd, from the workload's weight set; the singletons
give kappa.p full rank and, being odd against an even w0, make the parity
congruences a.M = 0 (mod 2) of the M-lattice independent), and the
workload's sparse rows x_a (support in coordinates 1..h11-1) with
w_a in {1..4}.  c2 is uniform even in [-20, 60].  Directions whose
kappa.p-hat lacks signature (1, h11-1) or has kappa(p,p,p) <= 0 are
rejected (counted in `rejected`).
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import intlat

M0MIN = 13


@dataclass
class Geometry:
    """One synthetic CY in the coni basis (the fields the search needs)."""
    h11: int
    h21: int
    kappa: np.ndarray          # (h, h, h) int64, totally symmetric
    c2: np.ndarray             # (h,) int64
    Mbasis: np.ndarray         # (h, h) int64, basis vectors as columns
    seed: int

    @property
    def Q(self):
        return self.h11 + self.h21 + 2


@dataclass
class Workload:
    """Geometries plus directions: p-vector i (with its leading 0) belongs to
    geometry pgeo[i] and is searched at dilation dil[i]."""
    name: str
    geoms: list
    ps: list                   # per direction: int64 array of length h11 of its geometry
    pgeo: np.ndarray           # (n,) int32
    dil: np.ndarray            # (n,) float64
    rejected: int = 0
    info: dict = field(default_factory=dict)

    def __len__(self):
        return len(self.ps)

    def groups(self):
        """(geometry index, dilation) -> direction indices, as the reference's
        mixed-dilation caller builds one geometry entry per distinct dilation
        (pfvs/coni.py:701-738)."""
        out = {}
        for i, (g, d) in enumerate(zip(self.pgeo.tolist(), self.dil.tolist())):
            out.setdefault((g, d), []).append(i)
        return out


def make_kappa(h, n_rows, ones, sing_weights, rng):
    """The signed cube sum of the module docstring."""
    kappa = np.zeros((h, h, h), dtype=np.int64)
    kappa += int(rng.choice([2, 4]))
    for i in range(1, h):
        kappa[i, i, i] -= int(rng.choice(sing_weights))
    for _ in range(n_rows):
        x = np.zeros(h, dtype=np.int64)
        k = int(rng.integers(ones[0], ones[1] + 1))
        x[1 + rng.choice(h - 1, k, replace=False)] = 1
        w = int(rng.integers(1, 5))
        kappa -= w * np.einsum("i,j,k->ijk", x, x, x)
    return kappa


def make_geometry(h, h21, n_rows, ones, sing_weights, seed):
    rng = np.random.default_rng(seed)
    kappa = make_kappa(h, n_rows, ones, sing_weights, rng)
    c2 = 2 * rng.integers(-10, 31, h).astype(np.int64)
    Mb = intlat.m_lattice(kappa, c2)
    return Geometry(h, h21, kappa, c2, Mb, seed)


def lorentzian_ok(kappa, p):
    """kappa.p has signature (1, h-1) and kappa(p, p, p) > 0 (then the
    ellipsoid matrix on the K.p = 0 lattice is positive definite).  Decided
    in floating point with a relative margin; the search itself re-decides
    positive definiteness exactly (fraction-free pivots)."""
    Z = np.tensordot(kappa, p, axes=([2], [0]))        # int64; |entries| << 2^63 here
    vol = int(p @ Z @ p)
    ev = np.linalg.eigvalsh(Z.astype(np.float64))
    tol = 1e-9 * max(1.0, float(np.max(np.abs(ev))))
    return (int(np.sum(ev > tol)) == 1 and int(np.sum(ev < -tol)) == len(p) - 1
            and vol > 0)


def sample_directions(geom, n, emax, rng, max_tries=None):
    """n distinct primitive p-hat = (0, p_1..p_{h-1}), entries in [1, emax],
    passing `lorentzian_ok`.  Returns (ps (n, h) int64, rejected)."""
    h = geom.h11
    seen, out, rej, tries = set(), [], 0, 0
    max_tries = max_tries or 50 * n + 1000
    while len(out) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could not sample {n} directions for h11={h}")
        p = np.concatenate([[0], rng.integers(1, emax + 1, h - 1)]).astype(np.int64)
        if math.gcd(*[int(x) for x in p]) != 1:
            continue
        t = tuple(p.tolist())
        if t in seen:
            continue
        seen.add(t)
        if not lorentzian_ok(geom.kappa, p):
            rej += 1
            continue
        out.append(p)
    return np.array(out, dtype=np.int64).reshape(-1, h), rej


# name -> (list of (h11, h21, n_rows, ones, singleton weights), n_p, emax, dilations)
SPECS = {
    "small":     ([(5, 60, 8, (1, 3), (1, 3))], 256, 6, (1,)),
    "plain":     ([(11, 120, 8, (1, 4), (1, 3))], 4096, 8, (1,)),
    "mixed":     ([(h, 2 * h + 40, 8, (1, 4), (1, 3, 5, 7, 9)) for h in (8, 16, 24, 32)],
                  65536, 10, (1, 2, 3, 4)),
    "precision": ([(40, 150, 8, (1, 4), (1, 3, 5, 7, 9, 11, 13, 15))], 16384, 12, (2,)),
    "large":     ([(60, 200, 70, (1, 5), (1,))], 4096, 16, (1,)),
}


def build(name, n_p=None, seed=0, dilations=None, geoms_only=False):
    """
    The named workload, deterministic in `seed`.  `n_p` (default: the
    workload's size) takes the first n_p directions of the full sampling
    order, so a smaller workload is a prefix of the larger one.
    `dilations` overrides the dilation set (used by deeper parity cases).
    Directions are split evenly over the geometries (round-robin), and each
    direction's dilation is drawn uniformly from the dilation set.
    """
    if name not in SPECS:
        raise ValueError(f"unknown workload {name!r} (one of {sorted(SPECS)})")
    gspecs, n_full, emax, dils = SPECS[name]
    dils = tuple(dilations) if dilations is not None else dils
    n = n_full if n_p is None else int(n_p)
    geoms = [make_geometry(h, h21, r, o, sw, seed * 1000 + 17 * k + h)
             for k, (h, h21, r, o, sw) in enumerate(gspecs)]
    if geoms_only:
        return Workload(name, geoms, [], np.zeros(0, np.int32), np.zeros(0))
    ng = len(geoms)
    per = [n // ng + (1 if k < n % ng else 0) for k in range(ng)]
    rng_dirs = [np.random.default_rng(seed * 7919 + 31 * k + 1) for k in range(ng)]
    samples, rej = [], 0
    for k, g in enumerate(geoms):
        ps, r = sample_directions(g, per[k], emax, rng_dirs[k])
        samples.append(ps)
        rej += r
    # round-robin interleave so that a prefix covers every geometry
    ps, pgeo = [], []
    idx = [0] * ng
    while len(ps) < n:
        for k in range(ng):
            if idx[k] < per[k] and len(ps) < n:
                ps.append(samples[k][idx[k]])
                pgeo.append(k)
                idx[k] += 1
    drng = np.random.default_rng(seed * 104729 + 5)
    dil = np.array([float(dils[int(drng.integers(len(dils)))]) for _ in range(n)])
    return Workload(name, geoms, ps, np.array(pgeo, dtype=np.int32), dil, rej,
                    info=dict(emax=emax, dilations=dils, seed=seed))
