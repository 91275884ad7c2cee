"""B200-native restarted-Halpern PDHG engine for PRAMANA LPs.

The compute path is libb2p_pdhg.so (hand-written CUDA for sm_100a behind the
C ABI of include/b2p_pdhg.h); this package is its Python mirror of the
reference's PDHG interface plus the seeded workload generators.
"""
from .model import LpCase, Model  # noqa: F401
from .pdhg import (Engine, PdhgOptions, PdhgResult, PdhgStats, csr_spmv, gpuAvailable,  # noqa: F401
                   gpuInfoJson, solvePdhg, solvePdhgBatch)
from . import generators  # noqa: F401

__all__ = ["Model", "LpCase", "PdhgOptions", "PdhgResult", "PdhgStats", "Engine", "solvePdhg", "solvePdhgBatch",
           "gpuAvailable", "gpuInfoJson", "csr_spmv", "generators"]
