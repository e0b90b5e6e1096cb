"""B200-native HDDM hot path of ADVENTURE_FullWave.

The batched CUDA solver lives in ``libfwgpu.so`` (C ABI in
``include/fwgpu.h``); ``hddm`` is its host API shaped after the reference's
``hddm_solver_CS`` plug-in table, and ``meshgen`` builds the synthetic
full-wave models the solver runs on.
"""
from . import meshgen  # noqa: F401

__all__ = ["meshgen", "hddm", "build"]
