"""CPU oracle for the dose-calculation / fluence-optimization path.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product (fastdose_b200) never
imports it.  See fd_oracle.h for what is restated and where.
"""
from .oracle import *  # noqa: F401,F403
