"""Test infrastructure: the CPU oracle of the solve phase (restatement of the reference's algorithm)
and the recipe that builds the reference itself for pinning.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may use this package; the product path never does."""
