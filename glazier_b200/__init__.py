"""glazier_b200: a B200-native device engine for glazier's Cellular Potts model.

A drop-in for glazier's ``--engine gpu`` path: the Blueprint reader
(``blueprint``), the ``GpuSimulation`` backend (``engine``, over the C ABI in
include/glazier_gpu.h) and the ``glazier._native`` entry points (``native``).
The kernels are ahead-of-time CUDA for sm_100a in ``csrc/``.
"""

from .blueprint import Blueprint, BlueprintError, CellType, Model, Species, Start

__all__ = ["Blueprint", "BlueprintError", "CellType", "Model", "Species", "Start"]
