"""Tet10 3D linear elasticity on the GPU.

Drop-in for cloudfem/physics/elastic_tet10.py (``__all__`` :34-37):
``assemble_elasticity_tet10`` (:135-211) builds the 30 x 30 Keast-5
element matrices (one warp per element, gradients staged in shared
memory) and reduces their 3 x 3 nodal blocks into the pattern; traction
on 6-node faces uses the 3-point rule; ``solve_elasticity_tet10``
(:214-229) solves with 3 x 3 block-Jacobi PCG on the device;
``element_stress_tet10`` (:232-279) recovers centroid strain and stress.
"""

import numpy as np

from .. import _native as N
from .._faces import FACE_EDGES as _FACE_EDGES  # noqa: F401
from .._faces import TRI_L3 as _TRI_L, TRI_W3 as _TRI_W  # noqa: F401
from .._faces import face_shape6 as _face_shape  # noqa: F401
from ..device import DeviceMesh, evaluate
from ..fem.tet10 import element_operators, shape_functions  # noqa: F401
from ..mesh.tet10_mesh import EDGES  # noqa: F401
from .elastic3d import (_EYE3, _as_vector, _assemble, _bmat, _element_stress, _solve,
                        apply_dirichlet_vec3, constitutive_3d)  # noqa: F401

__all__ = [
    "boundary_faces10", "assemble_elasticity_tet10",
    "solve_elasticity_tet10", "element_stress_tet10",
]

FACES10 = (((0, 1, 2), (4, 5, 6)), ((0, 3, 1), (7, 8, 4)),
           ((0, 2, 3), (6, 9, 7)), ((1, 3, 2), (8, 9, 5)))


def boundary_faces10(mesh, name):
    """(F, 6) exterior 6-node faces [c0, c1, c2, m01, m12, m20]."""
    return DeviceMesh(mesh).boundary_faces(name, tet10=True)


def _strain_displacement10(G):
    from .elastic3d import _strain_displacement
    return _strain_displacement(G)


def _dof_map10(el):
    el = np.asarray(el, dtype=int)
    return (3 * el[:, None] + np.arange(3)).ravel()


def assemble_elasticity_tet10(mesh, E, nu, body=None, traction=None, T=None,
                              alpha=0.0, T_ref=0.0):
    """(A csr (3N, 3N), rhs (3N,)) of Tet10 elasticity with loads."""
    dm = DeviceMesh(mesh)
    vals, rhs = _assemble(dm, mesh, N.OP_T10_ELAST, E, nu, body, traction, T,
                          alpha, T_ref, tet10=True)
    return dm.pattern.to_scipy(3, vals), rhs.cpu().numpy()


def solve_elasticity_tet10(mesh, E, nu, bc=None, body=None, traction=None,
                           T=None, alpha=0.0, T_ref=0.0, *, precision="fp64",
                           rtol=None, max_iter=None):
    """Solve Tet10 elasticity; returns (ux, uy, uz) over all nodes."""
    return _solve(mesh, N.OP_T10_ELAST, True, E, nu, bc, body, traction, T,
                  alpha, T_ref, precision, rtol, max_iter,
                  "solve_elasticity_tet10")


def element_stress_tet10(mesh, u, E, nu, T=None, alpha=0.0, T_ref=0.0):
    """Centroid strain and stress per element, each (M, 6)
    (elastic_tet10.py:232-262), on the device."""
    return _element_stress(mesh, u, E, nu, T, alpha, T_ref)
