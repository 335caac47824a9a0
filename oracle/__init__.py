"""Test infrastructure: the CPU oracle for the neighbour-search path (see oracle.py).

Imported only by tests/, tests/golden/make_golden.py and bench.py's CPU-baseline leg.
"""
