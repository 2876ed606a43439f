"""mycel_b200: B200 (sm_100a) implementation of Mycel.Core's FEM + SIMP inner loop behind a C ABI.

The product is libmycel_b200.so (include/mycel.h). This package holds its sources (csrc/), its build script,
and the Mycel.Core-shaped host interface used from Python (model.py, api.py).
"""
from .model import (ArgumentError, FeMaterial, FeModel, GridSpec, InvalidOperationError, IterationSnapshot, LoadCase,
                    MycelError, OptimizerOptions, PcgResult, StaticAnalysisOptions, StaticAnalysisResult,
                    SurfacePatch, TopologyOptimizationResult)

__all__ = ["ArgumentError", "FeMaterial", "FeModel", "GridSpec", "InvalidOperationError", "IterationSnapshot",
           "LoadCase", "MycelError", "OptimizerOptions", "PcgResult", "StaticAnalysisOptions", "StaticAnalysisResult",
           "SurfacePatch", "TopologyOptimizationResult"]


def __getattr__(name):
    # the GPU-facing API loads libmycel_b200.so on first use
    if name in ("Context", "Problem", "DensityFilter", "StaticAnalysis", "TopologyOptimizer", "IterationController",
                "SimpSession", "oc_update", "default_context"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
