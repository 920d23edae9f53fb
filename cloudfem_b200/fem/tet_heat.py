"""Transient P1 heat conduction (theta method) on the GPU.

Drop-in for cloudfem/fem/tet_heat.py:

* ``assemble_mass_tet`` (:72-94): consistent capacity rho_cp V/20 (1+d_ij),
  built by the device element kernel and CSR reduction.
* ``_boundary_faces`` (:97-120): exterior faces on a named set; candidate
  faces are selected on the device, the once-only count runs on the
  candidates (first-occurrence order kept).
* ``assemble_boundary_terms`` (:136-172): Neumann q A / 3 and Robin face
  mass h A/12 (1 + d_ij) plus h T_inf A / 3, integrated on the device over
  the device face lists (``_faces``: cfem_face_geometry,
  cfem_face_integrate); the returned CSR has the reference's face-pair
  structure.
* ``transient_heat_tet`` (:197-274): K, F and C assembled on the device;
  A_sys = C + theta h K and R_sys = C - (1-theta) h K formed there; every
  step is an SpMV plus one device PCG solve warm-started from the previous
  field (the reference factorises A_sys once with SuperLU).
"""

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


def _scalar_fn(v):
    """Normalise a float-or-callable(x, y, z) spec to a callable."""
    return v if callable(v) else (lambda x, y, z, v=v: v)


def _terms(dm, mesh, neumann, robin, rule=None, tet10=False):
    """Device Neumann and Robin terms: (K_add node-pattern values or None,
    F_add, the Robin face lists) (tet_heat.py:136-172; Tet10:
    tet10.py:362-435 with rule _faces.T10)."""
    import torch
    rule = rule or _faces.P1
    dev = dm.rt.device
    F = torch.zeros(mesh.n_nodes, dtype=torch.float64, device=dev)
    K, faces = None, []
    for name, q in (neumann or {}).items():
        _faces.add_load(dm, dm.boundary_faces_device(name, tet10), rule, [q], F)
    for name, (h, tinf) in (robin or {}).items():
        fd = dm.boundary_faces_device(name, tet10)
        if K is None:
            K = torch.zeros(dm.pattern.nnz, dtype=torch.float64, device=dev)
        _faces.add_robin(dm, fd, rule, h, tinf, F, K)
        faces.append(fd)
    return K, F, faces


def boundary_csr(dm, K, faces):
    """Host CSR of device face terms with the reference's structure."""
    import scipy.sparse as sp
    if K is None:
        return sp.csr_matrix((dm.n_nodes, dm.n_nodes))
    return _faces.face_csr(dm, [f.cpu().numpy() for f in faces], K)


def add_into(dm, K, K_add):
    """K + K_add (device node-pattern values) as a new array."""
    import torch
    if K_add is None:
        return K
    out = torch.empty_like(K)
    rt = dm.rt
    N.check(rt.lib.cfem_axpby(rt.ctx, K.numel(), 1.0, N.ptr(K), 1.0, N.ptr(K_add),
                              N.ptr(out), rt.stream()))
    return out


def assemble_boundary_terms(mesh, neumann=None, robin=None):
    """(K_add csr, F_add) of Neumann fluxes and Robin convection."""
    dm = DeviceMesh(mesh)
    K, F, faces = _terms(dm, mesh, neumann, robin)
    return boundary_csr(dm, K, faces), F.cpu().numpy()


def _dirichlet_values(mesh, bc):
    """Resolve a tet_poisson-style bc dict to {node_index: value}."""
    idx, vals = fixed_scalar(mesh, bc)
    return dict(zip(idx.tolist(), vals.tolist()))


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
    K_add, F_add, _ = _terms(dm, mesh, neumann, robin)
    K = add_into(dm, K, K_add)
    F = F + F_add
    C, _ = dm.assemble(N.OP_P1_MASS, coef=rho_cp)
    n_steps = n_steps_of(t_end, dt)
    idx, vals = fixed_scalar(mesh, bc)
    return theta_march(dm, K, C, F, idx, vals, t_end, n_steps, T0, theta,
                       precision, rtol, max_iter)
