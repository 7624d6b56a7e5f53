"""Parity oracle for the graph search path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only to check GPU results against it (or, for the CPU
baseline, to time it).  The product package (scattersearch_b200) never
imports it.
"""
