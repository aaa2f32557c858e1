"""Three-dimensional HOME-LBM (D3Q27): drop-in for the reference's envs/lbm3d solver layer."""
from .lbm_core_3d import HomeFlow3D
from .lbm_solver_3d import LBM_Solver3D

__all__ = ["HomeFlow3D", "LBM_Solver3D"]
