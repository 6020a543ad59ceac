"""chronusq_public_b200: a B200-native (sm_100a) direct-SCF two-electron engine.

Drop-in for ChronusQ's ``AOIntegrals::newTwoEContractDirect`` (density X in, G[X] = J - K
out) behind the C ABI in ``include/cqgpu.h``; this package holds the CUDA sources
(``csrc/``), the in-tree built library, and the host-side Python mirror of the
reference interface (:mod:`.aointegrals`), basis sets (:mod:`.basis`) and molecules
(:mod:`.molecule`).
"""
__version__ = "0.1.0"
