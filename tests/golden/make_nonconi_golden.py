"""
Generate tests/golden/nonconi.npz: golden vectors for non-coni ZpM
(pfvs/nonconi.py:262), from the reference's own data and C code:

- the four non-coni vacua of the reference's paper examples
  (tests/data/paper_examples.json of the reference: kappa, c2, the Kahler
  cone H, the paper's p, (K, M) and dilation), searched as its
  tests/test_paper_examples.py:54-63 does (Qmin = 0, Qmax = -K.M, the
  paper's dilation);
- the non-coni Manwe geometry of its tests/test_manwe.py (KAPPA, C2, H, read
  from that file as text) with the primitive p-vectors of the smallest box
  holding at least 150 of them, at dilations 1 and 3 with the default Qmax
  h11 + h21 + 2 (its test_ZpM_routes_agree, tests/test_manwe.py:362-382).

For each case the lattice points of every p-vector from the reference's C
setup and kernel (oracle/_ref, composed as nonconi.ZpM composes them;
oracle/nonconi.py:ref_points) and the PFV set of the oracle's restated
post-processing.  The reference tree is not present where the GPU tests run;
this file carries the cases there.

    python tests/golden/make_nonconi_golden.py
"""
import ast
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import nonconi, pvecs  # noqa: E402
from pfvs_b200 import intlat  # noqa: E402

REF = os.environ.get("PFVS_REFERENCE", "/root/reference")


def manwe():
    """KAPPA, C2, H and H21 of the reference's tests/test_manwe.py, read as text."""
    src = open(os.path.join(REF, "tests", "test_manwe.py")).read()
    vals = {}
    for node in ast.parse(src).body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            t = node.targets[0]
            names = [t.id] if isinstance(t, ast.Name) else \
                [e.id for e in t.elts] if isinstance(t, ast.Tuple) else []
            v = node.value
            if isinstance(v, ast.Call) and v.args:           # np.array([...])
                v = v.args[0]
            try:
                lit = ast.literal_eval(v)
            except ValueError:
                continue
            if len(names) == 1:
                vals[names[0]] = lit
            elif isinstance(lit, tuple):
                vals.update(zip(names, lit))
    return vals["KAPPA"], vals["C2"], vals["H"], vals["H21"]


def case_points(kappa, Mb, ps, Qmax, D):
    """The reference's points of every p (rows in canonical order) and per-p statuses."""
    qmax = nonconi.qmax_of(Qmax, D)
    Ms, Ks, qs, pid, sts, Cs = [], [], [], [], [], []
    for i, p in enumerate(ps):
        st, C, M, Kn, q = nonconi.ref_points(kappa, Mb, p, Qmax, qmax)
        sts.append(st)
        if st == 0 and len(q):
            Ms.append(M); Ks.append(Kn); qs.append(q); pid.append(np.full(len(q), i)); Cs.append(C)
    h = kappa.shape[0]
    M = np.vstack(Ms) if Ms else np.zeros((0, h), np.int64)
    Kn = np.vstack(Ks) if Ks else np.zeros((0, h), np.int64)
    q = np.concatenate(qs) if qs else np.zeros(0, np.int64)
    pidx = np.concatenate(pid).astype(np.int64) if pid else np.zeros(0, np.int64)
    C = np.vstack(Cs) if Cs else np.zeros((0, h - 1), np.int32)
    keys = tuple(Kn[:, j] for j in range(h - 1, -1, -1)) + tuple(M[:, j] for j in range(h - 1, -1, -1)) + (pidx,)
    o = np.lexsort(keys) if len(q) else np.zeros(0, np.int64)
    return M[o], Kn[o], q[o], pidx[o], C[o], np.array(sts, np.int32)


def main():
    cases = []
    ex = json.load(open(os.path.join(REF, "tests", "data", "paper_examples.json")))["examples"]
    for e in ex:
        if e["kind"] != "non-coni":
            continue
        kappa = np.array(e["kappa"], dtype=np.int64)
        Q = -int(np.dot(e["K"], e["M"]))
        cases.append(dict(name="paper-" + e["section"], kappa=kappa, c2=np.array(e["c2"]), H=np.array(e["H"]),
                          ps=np.array([e["p"]], dtype=np.int64), Qmin=0, Qmax=Q, D=float(e["min_dilation"]),
                          known=(np.array(e["K"]), np.array(e["M"]))))
    KAPPA, C2, H, H21 = manwe()
    kappa = np.array(KAPPA, dtype=np.int64)
    h = kappa.shape[0]
    H = np.array(H, dtype=np.int64)
    for B in range(1, 6):
        ps = np.array(pvecs.box_enum(B, H), dtype=np.int64)
        if len(ps) >= 150:
            break
    for D in (1.0, 3.0):
        cases.append(dict(name=f"manwe-dil{D:g}", kappa=kappa, c2=np.array(C2), H=H, ps=ps, Qmin=0,
                          Qmax=h + H21 + 2, D=D, known=None))
    out = {"n_cases": np.array([len(cases)])}
    for k, c in enumerate(cases):
        Mb = intlat.m_lattice(c["kappa"], c["c2"], coni=False)
        M, Kn, q, pidx, C, sts = case_points(c["kappa"], Mb, c["ps"], c["Qmax"], c["D"])
        pf, _ = nonconi.zpm(c["kappa"], Mb, c["ps"], c["Qmin"], c["Qmax"], c["D"], source="ref")
        pf = sorted(pf)
        hh = c["kappa"].shape[0]
        out.update({f"c{k}_kappa": c["kappa"], f"c{k}_c2": c["c2"], f"c{k}_H": c["H"], f"c{k}_Mbasis": Mb,
                    f"c{k}_ps": c["ps"], f"c{k}_scal": np.array([c["Qmin"], c["Qmax"]], dtype=np.int64),
                    f"c{k}_D": np.array([c["D"]]), f"c{k}_M": M, f"c{k}_Kn": Kn, f"c{k}_q": q,
                    f"c{k}_pidx": pidx, f"c{k}_C": C, f"c{k}_status": sts,
                    f"c{k}_pfvK": np.array([a for a, _ in pf], dtype=np.int64).reshape(-1, hh),
                    f"c{k}_pfvM": np.array([b for _, b in pf], dtype=np.int64).reshape(-1, hh)})
        if c["known"] is not None:
            out[f"c{k}_knownK"], out[f"c{k}_knownM"] = c["known"]
            assert (tuple(int(x) for x in c["known"][0]), tuple(int(x) for x in c["known"][1])) in set(pf)
        print(k, c["name"], "h11", hh, "p-vectors", len(c["ps"]), "points", len(q), "PFVs", len(pf),
              "statuses", dict(zip(*np.unique(sts, return_counts=True))))
    np.savez_compressed(os.path.join(HERE, "nonconi.npz"), **out)


if __name__ == "__main__":
    main()
