"""ip_cu_lbm_b200 -- B200-native (sm_100a) implementation of the IP_CU_LBM
per-step lattice Boltzmann path.

* ``legacy()``: the reference's kernel-entry API (function/*.cu) as C-ABI
  launchers in libipcu.so, same names and argument order.
* ``Sim``: the structured-grid solver, one fused collide-and-stream launch
  per step.
* ``my_module``: the pybind-style ``GPUMemory`` / ``LockExchange`` front end
  of the reference's pybind_LockExchange prototype.
"""
from ._lib import IpcuError, lib, legacy, LIB_PATH  # noqa: F401
from .sim import Sim  # noqa: F401

__all__ = ["IpcuError", "lib", "legacy", "Sim", "LIB_PATH"]
