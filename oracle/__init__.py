"""ORACLE — test infrastructure only (see oracle/trid_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs may import this package, and only as the checker or the timed
CPU baseline. The product package (tridsolver_b200) never imports it.
"""
