"""Test infrastructure: the CPU oracle (liboracle.so, a restatement of the
upstream algorithm) and the upstream reference harness (oracle/_ref, built
from the upstream sources where they lie).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may import this package -- it is the checker,
never the thing measured or shipped.
"""
