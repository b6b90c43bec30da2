"""Oracle package (test infrastructure only): CPU restatement of the reference's
BVE hot path, the shim-compiled reference itself, and their ctypes wrappers.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it."""
