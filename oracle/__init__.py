"""CPU oracle for the pcbroute search back end -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package, and only as the
checker or the timed CPU baseline. The C restatement lives in pcb_oracle.c (see its header for what it follows
in the reference and how it is pinned).
"""
