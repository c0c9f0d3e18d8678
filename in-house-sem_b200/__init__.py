"""insem_b200: B200 (sm_100a) backend of insem's per-time-step path.

The package directory is ``in-house-sem_b200``; it is imported under the
module name ``insem_b200`` (see ``__graft_entry__.load_package``).

Layout:
  csrc/        CUDA kernels and the C ABI implementation (libinsem_cuda.so)
  native.py    ctypes binding of include/insem_cuda.h
  problem.py   host description of one solve (what Solver(Problem) builds)
  solver.py    device solver with the reference Solver's Python API
  batch.py     many solves advanced by shared launches
  kernels.py   per-block and DofMap seams
  build.py     in-tree nvcc build for sm_100a
"""

from .native import InsemError, lib  # noqa: F401
from .problem import BlockData, DomainData, ProblemData, ReceiverData, SourceData  # noqa: F401
from .solver import Solver  # noqa: F401
from .batch import Batch, BatchMember  # noqa: F401

__version__ = "0.1.0"
