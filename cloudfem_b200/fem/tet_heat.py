"""Transient P1 heat conduction (theta method) on the GPU.

Drop-in for cloudfem/fem/tet_heat.py:

* ``assemble_mass_tet`` (:72-94): consistent capacity rho_cp V/20 (1+d_ij),
  built by the device element kernel and CSR reduction.
* ``_boundary_faces`` (:97-120): exterior faces on a named set; candidate
  faces are selected on the device, the once-only count runs on the
  candidates (first-occurrence order kept).
* ``assemble_boundary_terms`` (:136-172): Neumann q A / 3 and Robin face
  mass h A/12 (1 + d_ij) plus h T_inf A / 3.
* ``transient_heat_tet`` (:197-274): K, F and C assembled on the device;
  A_sys = C + theta h K and R_sys = C - (1-theta) h K formed there; every
  step is an SpMV plus one device PCG solve warm-started from the previous
  field (the reference factorises A_sys once with SuperLU).
"""

import numpy as np

from .. import _native as N
from .. import _faces
from .._driver import THETA, n_steps_of, theta_march
from ..device import DeviceMesh, fixed_scalar
from .tet_poisson import apply_dirichlet, assemble  # noqa: F401


def assemble_mass_tet(mesh, rho_cp=1.0):
    """Consistent P1 capacity matrix int rho_cp phi_i phi_j dV (csr)."""
    dm = DeviceMesh(mesh)
    vals, _ = dm.assemble(N.OP_P1_MASS, coef=rho_cp)
    return dm.pattern.to_scipy(1, vals)


def _boundary_faces(mesh, name):
    """(F, 3) exterior faces on mesh.boundaries[name]."""
    return DeviceMesh(mesh).boundary_faces(name)


def _face_geometry(mesh, tri):
    """Centroid and area of one triangular face (3 node indices)."""
    p = mesh.nodes[np.asarray(tri)]
    cen = p.mean(axis=0)
    cr = np.cross(p[1] - p[0], p[2] - p[0])
    return cen, 0.5 * float(np.linalg.norm(cr))


def _scalar_fn(v):
    """Normalise a float-or-callable(x, y, z) spec to a callable."""
    return v if callable(v) else (lambda x, y, z, v=v: v)


def _terms(dm, mesh, neumann, robin):
    n = mesh.n_nodes
    F = np.zeros(n)
    rows, cols, data = [], [], []
    for name, q in (neumann or {}).items():
        _faces.p1_neumann(mesh.nodes, dm.boundary_faces(name), q, F)
    for name, (h, tinf) in (robin or {}).items():
        _faces.p1_robin(mesh.nodes, dm.boundary_faces(name), h, tinf, F,
                        rows, cols, data)
    return _faces.coo_csr(rows, cols, data, n), F


def assemble_boundary_terms(mesh, neumann=None, robin=None):
    """(K_add csr, F_add) of Neumann fluxes and Robin convection."""
    return _terms(DeviceMesh(mesh), mesh, neumann, robin)


def _dirichlet_values(mesh, bc):
    """Resolve a tet_poisson-style bc dict to {node_index: value}."""
    idx, vals = fixed_scalar(mesh, bc)
    return dict(zip(idx.tolist(), vals.tolist()))


def add_csr_into(dm, vals, K_add):
    """vals += K_add on the mesh pattern (K + K_add, tet_heat.py:227-230)."""
    import torch
    if K_add.nnz == 0:
        return
    K_add = K_add.tocsr()
    K_add.sum_duplicates()
    K_add.sort_indices()
    rt = dm.rt
    dev = rt.device
    ap = torch.from_numpy(K_add.indptr.astype(np.int32)).to(dev)
    ai = torch.from_numpy(K_add.indices.astype(np.int32)).to(dev)
    av = torch.from_numpy(K_add.data.astype(np.float64)).to(dev)
    N.check(rt.lib.cfem_csr_add_subset(rt.ctx, dm.pattern.handle, N.ptr(ap),
                                       N.ptr(ai), N.ptr(av), dm.n_nodes,
                                       N.ptr(vals), rt.stream()))


def transient_heat_tet(mesh, k=1.0, rho_cp=1.0, f=0.0, bc=None,
                       neumann=None, robin=None, t_end=1.0, dt=0.1,
                       T0=0.0, method="cn", *, precision="fp64", rtol=None,
                       max_iter=None):
    """Transient heat conduction on a TetMesh; returns (times, T_history)."""
    import torch
    if method not in THETA:
        raise ValueError(f"unknown method {method!r}; "
                         f"use one of {sorted(THETA)}")
    theta = THETA[method]
    dm = DeviceMesh(mesh)
    K, F = dm.assemble(N.OP_P1_STIFF, coef=k, load=f)
    K_add, F_add = _terms(dm, mesh, neumann, robin)
    add_csr_into(dm, K, K_add)
    F = F + torch.from_numpy(F_add).to(dm.rt.device)
    C, _ = dm.assemble(N.OP_P1_MASS, coef=rho_cp)
    n_steps = n_steps_of(t_end, dt)
    idx, vals = fixed_scalar(mesh, bc)
    return theta_march(dm, K, C, F, idx, vals, t_end, n_steps, T0, theta,
                       precision, rtol, max_iter)
