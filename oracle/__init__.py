"""Checker package: the CPU oracle and the reference's own CPU code, via ctypes.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs; never by the product package.
"""
from .oracle import Oracle, RefLib, ORACLE_SO, ORACLE_LD_SO, REF_SO, build  # noqa: F401
