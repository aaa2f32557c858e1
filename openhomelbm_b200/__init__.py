"""openhomelbm_b200: the HOME-LBM moment-encoded stream-collide step of kuiwuchn/OpenHOMELBM,
re-built for NVIDIA B200 (sm_100a).

* ``openhomelbm_b200.lbm``   - ``HomeFlow`` / ``LBM_Solver`` (D2Q9, polygon solids)
* ``openhomelbm_b200.lbm3d`` - ``HomeFlow3D`` / ``LBM_Solver3D`` (D3Q27, mesh solids)

All computation runs in libhomelbm.so (hand-written CUDA, C ABI in include/homelbm.h).
"""
from . import _lib
from ._lib import HomeLBMError

__version__ = "0.1.0"
__all__ = ["HomeLBMError", "_lib", "__version__"]
