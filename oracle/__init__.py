"""Test infrastructure: the CPU oracle and the recipe that builds the reference.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package; the product path never does.
"""
