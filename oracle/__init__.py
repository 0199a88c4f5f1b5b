"""CPU FP64 oracle for the SCMC Monte Carlo path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only as the checker.  The product never does.
"""
