"""Tetrahedral mesh containers and structured box meshers."""
from .tet_mesh import TetMesh, box_mesh  # noqa: F401
from .tet10_mesh import EDGES, Tet10Mesh, box_mesh_tet10, tet4_to_tet10  # noqa: F401
