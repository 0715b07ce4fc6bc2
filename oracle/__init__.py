"""Test infrastructure: the CPU oracle (C restatement) and the reference's
own compiled counters. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this package, as the checker."""
