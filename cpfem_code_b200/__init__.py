"""B200-native (sm_100a) implementation of FASOLT3's per-increment hot path.

The crystal-plasticity Gauss-point update, element assembly, penalty boundary
conditions and multicolour SOR of gabortimar/CPFEM_code's ``fasolt3``
(src/fasolt), behind the C ABI of ``include/fasolt_gpu.h``.
"""
from . import abi, generator  # noqa: F401
from .problem import Control, Problem  # noqa: F401
from .solver import GpuSolver, NewtonStepper, ReplayHistory, load_library, LIB_PATH  # noqa: F401

__all__ = ["abi", "generator", "Control", "Problem", "GpuSolver", "NewtonStepper", "load_library", "LIB_PATH"]
