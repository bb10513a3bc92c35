"""Test oracle for cufe_b200 (CPU restatement + reference CPU build).  Test infrastructure:
only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this package."""
