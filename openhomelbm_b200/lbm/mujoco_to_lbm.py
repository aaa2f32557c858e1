"""The reference's envs/lbm/mujoco_to_lbm.py names: xy outlines of MuJoCo geoms and bodies for
the 2D solver, implemented in openhomelbm_b200.geometry."""
from ..geometry import (compute_convex_hull_2d, extract_lbm_polygon_from_mujoco, extract_mesh_projection_2d,
                        get_body_vertices_2d, get_geom_vertices_2d, resample_polygon)

__all__ = ["compute_convex_hull_2d", "extract_lbm_polygon_from_mujoco", "extract_mesh_projection_2d",
           "get_body_vertices_2d", "get_geom_vertices_2d", "resample_polygon"]
