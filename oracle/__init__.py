"""Test infrastructure: CPU restatement (oracle) of the GisSPA search path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  The product path (``gisspa_b200``) never does.
"""
