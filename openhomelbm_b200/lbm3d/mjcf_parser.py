"""The reference's envs/lbm3d/mjcf_parser.py names: MJCF bodies as closed triangle meshes for
the 3D solver, implemented in openhomelbm_b200.geometry (no trimesh)."""
from ..geometry import (TriMesh, get_body_world_positions, parse_mjcf, parse_mjcf_as_urdf_format,
                        parse_mjcf_to_meshes)

__all__ = ["TriMesh", "get_body_world_positions", "parse_mjcf", "parse_mjcf_as_urdf_format", "parse_mjcf_to_meshes"]
