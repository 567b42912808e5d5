"""CPU restatement of gpu_tracking's locate-and-link path (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
