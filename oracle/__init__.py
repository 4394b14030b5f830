"""
ORACLE / TEST INFRASTRUCTURE for the batched coniZpM path -- never part of
the product.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs import it, and only as the checker (or the timed CPU baseline).

- lattice.py, pfo.c/pfo.py: this repository's CPU restatement of the
  reference algorithm (setup, exact Fincke-Pohst search, emission).
- postproc.py: restatement of the lattice-points -> PFVs post-processing.
- ref_harness.c/ref.py: the reference's own CPU kernel compiled in place
  (oracle/Makefile -> oracle/_ref/), to pin the restatement and to time the
  reference CPU path.
"""
