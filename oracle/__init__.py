"""CPU checker for the CUDA coloring path (test infrastructure only).

oracle.restatement -- scalar C restatement of the reference's hot path (oracle.c);
oracle.reference -- the reference's own C code compiled from its sources (oracle/_ref/libref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package.
"""
