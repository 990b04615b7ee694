"""CPU oracle (test infrastructure only): FP64 restatement of the reference
reaction step, used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker.  Parity is unpinned (see oracle.cpp header)."""
