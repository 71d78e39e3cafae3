"""Test infrastructure: the CPU oracle of the SP step and the reference solver built from its
own sources.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it."""
