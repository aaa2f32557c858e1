"""Two-dimensional HOME-LBM (D2Q9): drop-in for the reference's envs/lbm solver layer."""
from .lbm_core import HomeFlow
from .lbm_solver import LBM_Solver

__all__ = ["HomeFlow", "LBM_Solver"]
