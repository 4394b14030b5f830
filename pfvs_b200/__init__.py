"""
pfvs_b200: a B200-native (sm_100a) implementation of natemacfadden/pfvs's
batched lattice searches for perturbatively flat vacua, behind the
reference's own Python API and C ABI:

- the batched coniZpM search (lattice setup, exact Fincke-Pohst enumeration,
  exact acceptance, the post-processing to PFVs): pfvs_b200.gpu, the C ABI
  of include/pfvs_gpu.h;
- the coni dilation bound mu0 and the exhaustive coniZp driver:
  pfvs_b200.dilation, pfvs_b200.coni;
- coniZpK, the coni PFVs above a dilation D0: pfvs_b200.zpk;
- non-coni ZpM: pfvs_b200.nonconi;
- several GPUs through a shared chunk queue: pfvs_b200.multi;
- the search grid and GCD-row policy tuned per batch class: pfvs_b200.tune.
"""
__version__ = "0.3.0"
