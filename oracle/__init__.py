"""TEST INFRASTRUCTURE: the oracle for slipcam framecor's correlate path (see oracle/oracle.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU leg import this package, as the checker.
"""
