"""CPU checkers for the PMG solve path.  TEST INFRASTRUCTURE ONLY.

Only the test suite, the smoke check and the CPU-baseline leg of the
benchmark load anything from this package.  The product library never does.
"""
