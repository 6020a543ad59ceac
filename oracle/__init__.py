"""CPU oracle for the direct-SCF two-electron contraction (test infrastructure only).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import this package.
"""
