"""P1 tetrahedral assembly, Dirichlet elimination and steady solve.

Drop-in for cloudfem/fem/tet_poisson.py. Same signatures and results:

* ``assemble`` (:35-69) -> (scipy csr (N, N), rhs (N,)); the element
  matrices k V G G^T and loads f V / 4 are built on the GPU and reduced
  into the CSR pattern in element order.
* ``apply_dirichlet`` (:72-110) -> (csr, rhs). Rows of fixed nodes become
  identity rows and fixed columns are removed from the free rows. The
  reference stores those removed entries as explicit zeros; the returned
  matrix equals the reference's after ``eliminate_zeros()`` on them.
* ``solve_tet_poisson`` (:113-122) -> u (N,): assembly, elimination and a
  Jacobi-PCG solve all on the device (the reference calls SuperLU).
"""

import ctypes

import numpy as np
import scipy.sparse as sp

from .. import _native as N
from .._driver import solve_block
from ..device import DeviceMesh, csr_to_device, fixed_scalar

_G_REF = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0],
                   [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def _tet_gradients(p):
    """Gradients of the four P1 basis functions on one tetrahedron.

    p : (4, 3) node coordinates. Returns (G (4, 3), volume).
    """
    p = np.asarray(p, dtype=float)
    m = np.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]], axis=1)
    vol = abs(np.linalg.det(m)) / 6.0
    return np.linalg.solve(m.T, _G_REF.T).T, vol


def assemble(mesh, k=1.0, f=0.0):
    """Stiffness matrix A (csr) and load vector rhs of -div(k grad u) = f.

    k, f : float or callable(x, y, z), sampled at element centroids.
    """
    dm = DeviceMesh(mesh)
    vals, rhs = dm.assemble(N.OP_P1_STIFF, coef=k, load=f)
    return dm.pattern.to_scipy(1, vals), rhs.cpu().numpy()


def apply_dirichlet(A, rhs, mesh, bc):
    """Identity rows for fixed nodes, fixed columns lifted into rhs.

    bc : dict boundary name (or 'all') -> value or callable(x, y, z).
    """
    import torch
    rhs = np.asarray(rhs, dtype=float)
    n = mesh.n_nodes
    idx, vals = fixed_scalar(mesh, bc)
    A = sp.csr_matrix(A)
    if len(idx) == 0:
        return A.copy(), rhs.copy()
    rt = N.runtime()
    d_ptr, d_idx, d_val, Ac = csr_to_device(rt, A)
    dev = rt.device
    mask = np.zeros(n, dtype=np.uint8)
    mask[idx] = 1
    fval = np.zeros(n)
    fval[idx] = vals
    d_mask = torch.from_numpy(mask).to(dev)
    d_fval = torch.from_numpy(fval).to(dev)
    d_rhs = torch.from_numpy(np.ascontiguousarray(rhs)).to(dev)
    o_ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    cap = max(Ac.nnz + len(idx), 1)
    o_idx = torch.empty(cap, dtype=torch.int32, device=dev)
    o_val = torch.empty(cap, dtype=torch.float64, device=dev)
    o_rhs = torch.empty(n, dtype=torch.float64, device=dev)
    nnz = N._i64()
    N.check(rt.lib.cfem_dirichlet_csr(
        rt.ctx, n, N.ptr(d_ptr), N.ptr(d_idx), N.ptr(d_val), N.ptr(d_rhs),
        N.ptr(d_mask), N.ptr(d_fval), N.ptr(o_ptr), N.ptr(o_idx),
        N.ptr(o_val), N.ptr(o_rhs), ctypes.byref(nnz), rt.stream()))
    m = nnz.value
    out = sp.csr_matrix((o_val[:m].cpu().numpy(), o_idx[:m].cpu().numpy(),
                         o_ptr.cpu().numpy()), shape=A.shape)
    return out, o_rhs.cpu().numpy()


def solve_tet_poisson(mesh, k=1.0, f=0.0, bc=None, *, precision="fp64",
                      rtol=None, max_iter=None):
    """Solve -div(k grad u) = f with Dirichlet BCs; returns nodal u."""
    dm = DeviceMesh(mesh)
    vals, rhs = dm.assemble(N.OP_P1_STIFF, coef=k, load=f)
    idx, v = fixed_scalar(mesh, bc)
    x = solve_block(dm, 1, vals, rhs, idx, v, precision, rtol, max_iter,
                    what="solve_tet_poisson")
    return x.cpu().numpy()
