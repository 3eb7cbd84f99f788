"""CPU oracle (test infrastructure): the checker for the CUDA path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The shipped library never links or calls it.
"""
