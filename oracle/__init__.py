"""Checker package: the CPU oracle, the reference's own CPU code and the reference's own
GPU kernels (built from its sources), via ctypes.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs; never by the product package.
"""
from .oracle import (Oracle, RefLib, RefGpuLib, ORACLE_SO, ORACLE_LD_SO, REF_SO, REF_GPU_SO, build,  # noqa: F401
                     reference_tree)
