"""CPU oracles of the CoupLB hot path (test infrastructure only).

The product (couplb_b200) never imports this package; tests, smoke() and the
CPU-baseline leg of bench.py use it as the checker.
"""
