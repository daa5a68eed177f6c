"""CPU oracle for the HPL solve path (test infrastructure only).

Only the tests, the smoke check and the CPU-baseline leg of bench.py import
this package; the product library never does.
"""
