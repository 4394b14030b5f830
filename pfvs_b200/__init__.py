"""
pfvs_b200: a B200-native (sm_100a) implementation of the batched coniZpM
search of natemacfadden/pfvs (lattice setup, exact Fincke-Pohst enumeration
and exact acceptance of conifold perturbatively flat vacua), behind the
reference's own Python API and C ABI.
"""
__version__ = "0.1.0"
