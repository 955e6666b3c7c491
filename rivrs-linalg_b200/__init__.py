"""B200 numeric phase for sparse symmetric indefinite LDL^T with APTP.

A drop-in for the numeric half of rivrs-sparse (analyze -> factor -> solve):
the host computes the ordering and symbolic structure; factorization and
solve run as sm_100a CUDA kernels in librivrs_b200.so (include/rivrs_b200.h).
"""
from . import autotune, batch, ordering, problems, reference_io, replicas, selector
from ._native import LIB_PATH, RvgError
from .batch import BatchLDLT
from .selector import PrecisionSelector
from .solver import (AnalyzeOptions, DimensionMismatch, FactorOptions, InvalidInput, OrderingStrategy,
                     SolveBeforeFactor, SparseError, SparseLDLT, SymbolicStructure, solve_full, symbolic_analyze)

__all__ = ["AnalyzeOptions", "FactorOptions", "OrderingStrategy", "SparseLDLT", "SymbolicStructure", "SparseError",
           "DimensionMismatch", "InvalidInput", "SolveBeforeFactor", "RvgError", "solve_full", "symbolic_analyze",
           "ordering", "problems", "batch", "BatchLDLT", "replicas", "selector", "PrecisionSelector", "autotune", "reference_io", "LIB_PATH"]
