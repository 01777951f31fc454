"""CPU oracle package (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import this package;
the product package cudilithium_b200 never does.
"""
