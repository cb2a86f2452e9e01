"""Test infrastructure: the CPU oracle (checker) and CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this package; the library never does.
"""
