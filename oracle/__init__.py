"""CPU parity oracle for the ED/XAS/RIXS hot path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` (to check its results) and the CPU-baseline leg of
``bench.py`` import this package.  The product (``edrixs_b200``) never does.
"""
