"""Test oracle for ns3d_wcns_b200 (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  See oracle/oracle.py.
"""
