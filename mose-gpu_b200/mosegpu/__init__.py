"""mose-gpu B200 engine: the explicit residual evaluation and Runge-Kutta stage update of MOSE-GPU's
multi-block structured compressible Euler / Navier-Stokes solver, as hand-written CUDA for sm_100a
behind a C ABI (include/mose_b200.h).

  abi     ctypes mirror of the C ABI
  case    host-side case construction (meshes, metrics, boundary records, tables, initial states)
  engine  the binding of libmose_b200.so (device memory and streams through torch)
  serving continuous batching of independent cases (request loop, HBM budget, per-case clocks)
  native_io   the reference's native field file (backup / restart)
  tecplot     the reference's Tecplot ASCII solution file
"""
from . import abi  # noqa: F401

__all__ = ["abi", "case", "engine", "serving", "native_io", "tecplot"]
