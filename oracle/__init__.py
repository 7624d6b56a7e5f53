"""Parity oracle for the graph search path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only as the checker.  The product package
(scattersearch_b200) never imports it.
"""
