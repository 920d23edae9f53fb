"""P1 3D linear elasticity on the GPU.

Drop-in for cloudfem/physics/elastic3d.py: Voigt order [xx, yy, zz, yz,
xz, xy], DOF 3 i + c. ``assemble_elasticity_3d`` (:105-189) builds the
12 x 12 element blocks V B^T D B on the device (nodal 3 x 3 blocks of the
pattern); ``apply_dirichlet_vec3`` (:192-233) is the free-DOF reduction,
solved by the device PCG; ``solve_elasticity_3d`` (:236-249) keeps the
whole chain on the device with 3 x 3 block-Jacobi PCG on the nodal block
matrix. Stress recovery (:252-302) is vectorised on the host.
"""

import ctypes

import numpy as np
import scipy.sparse as sp

from .. import _native as N
from .. import _faces
from .._driver import solve_block, solve_csr
from ..device import DeviceMesh, csr_to_device, evaluate, fixed_vector, ptr
from ..fem.tet_poisson import _tet_gradients


def constitutive_3d(E, nu):
    """6 x 6 isotropic D, Voigt [xx, yy, zz, yz, xz, xy]."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2.0 * mu
    D[0, 1] = D[0, 2] = D[1, 0] = D[1, 2] = D[2, 0] = D[2, 1] = lam
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    return D


def boundary_faces(mesh, name):
    """(F, 3) exterior faces whose nodes all lie in mesh.boundaries[name]."""
    return DeviceMesh(mesh).boundary_faces(name)


def _strain_displacement(G):
    """B (6, 3n) from basis gradients G (n, 3)."""
    G = np.asarray(G, dtype=float)
    n = G.shape[0]
    B = np.zeros((6, 3 * n))
    gx, gy, gz = G[:, 0], G[:, 1], G[:, 2]
    B[0, 0::3] = gx
    B[1, 1::3] = gy
    B[2, 2::3] = gz
    B[3, 1::3] = gz
    B[3, 2::3] = gy
    B[4, 0::3] = gz
    B[4, 2::3] = gx
    B[5, 0::3] = gy
    B[5, 1::3] = gx
    return B


def _dof_map(el):
    el = np.asarray(el, dtype=int)
    return (3 * el[:, None] + np.arange(3)).ravel()


def _assemble(dm, mesh, op, E, nu, body, traction, T, alpha, T_ref, tet10):
    import torch
    vals, rhs = dm.assemble_elastic(op, E, nu, body=body, T=T, alpha=alpha,
                                    T_ref=T_ref)
    if traction:
        # face loads on the device into a separate vector, then added once
        # (the reference sums the traction vector before adding it)
        extra = torch.zeros(3 * mesh.n_nodes, dtype=torch.float64, device=dm.rt.device)
        rule = _faces.T10_TRACTION if tet10 else _faces.P1
        for name, comps in traction.items():
            _faces.add_load(dm, dm.boundary_faces_device(name, tet10), rule, list(comps), extra)
        rhs += extra
    return vals, rhs


def assemble_elasticity_3d(mesh, E, nu, body=None, traction=None, T=None,
                           alpha=0.0, T_ref=0.0):
    """(A csr (3N, 3N), rhs (3N,)) of P1 elasticity with loads."""
    dm = DeviceMesh(mesh)
    vals, rhs = _assemble(dm, mesh, N.OP_P1_ELAST, E, nu, body, traction, T,
                          alpha, T_ref, tet10=False)
    return dm.pattern.to_scipy(3, vals), rhs.cpu().numpy()


def apply_dirichlet_vec3(A, rhs, mesh, bc, *, precision="fp64", rtol=None,
                         max_iter=None):
    """Solve A u = rhs with vector Dirichlet data; returns u (3N,).

    bc : name (or 'all') -> (ux, uy, uz), components float, callable or None.
    The free-DOF reduction A_ff u_f = rhs_f - A_fD u_D is solved in place by
    masking the fixed DOFs in the device PCG.
    """
    import torch
    rt = N.runtime()
    n3 = 3 * mesh.n_nodes
    idx, v = fixed_vector(mesh, bc or {})
    d_ptr, d_idx, d_val, _ = csr_to_device(rt, A)
    d_rhs = torch.from_numpy(np.ascontiguousarray(rhs, dtype=float)).to(
        rt.device)
    x = solve_csr(rt, d_ptr, d_idx, d_val, d_rhs, idx, v, n3, precision, rtol,
                  max_iter, what="apply_dirichlet_vec3")
    return x.cpu().numpy()


def _solve(mesh, op, tet10, E, nu, bc, body, traction, T, alpha, T_ref,
           precision, rtol, max_iter, what):
    dm = DeviceMesh(mesh)
    vals, rhs = _assemble(dm, mesh, op, E, nu, body, traction, T, alpha,
                          T_ref, tet10)
    idx, v = fixed_vector(mesh, bc or {})
    x = solve_block(dm, 3, vals, rhs, idx, v, precision, rtol, max_iter,
                    what=what)
    u = x.cpu().numpy()
    return u[0::3].copy(), u[1::3].copy(), u[2::3].copy()


def solve_elasticity_3d(mesh, E, nu, bc=None, body=None, traction=None,
                        T=None, alpha=0.0, T_ref=0.0, *, precision="fp64",
                        rtol=None, max_iter=None):
    """Solve P1 elasticity; returns (ux, uy, uz)."""
    return _solve(mesh, N.OP_P1_ELAST, False, E, nu, bc, body, traction, T,
                  alpha, T_ref, precision, rtol, max_iter,
                  "solve_elasticity_3d")


def _as_vector(mesh, u):
    if isinstance(u, tuple):
        uv = np.empty(3 * mesh.n_nodes)
        uv[0::3], uv[1::3], uv[2::3] = u
        return uv
    return np.asarray(u, dtype=float).ravel()


_EYE3 = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])


def _bmat(G):
    """Batched B (M, 6, 3n) from gradients (M, n, 3)."""
    M, n, _ = G.shape
    B = np.zeros((M, 6, 3 * n))
    gx, gy, gz = G[..., 0], G[..., 1], G[..., 2]
    B[:, 0, 0::3] = gx
    B[:, 1, 1::3] = gy
    B[:, 2, 2::3] = gz
    B[:, 3, 1::3] = gz
    B[:, 3, 2::3] = gy
    B[:, 4, 0::3] = gz
    B[:, 4, 2::3] = gx
    B[:, 5, 0::3] = gy
    B[:, 5, 1::3] = gx
    return B


def _element_stress(mesh, u, E, nu, T, alpha, T_ref):
    """Centroid (sig, eps) per element on the device (cfem_element_stress)."""
    import torch
    dm = DeviceMesh(mesh)
    dev = dm.rt.device
    uv = torch.from_numpy(np.ascontiguousarray(_as_vector(mesh, u), dtype=float)).to(dev)
    if uv.numel() != 3 * dm.n_nodes:
        raise ValueError(f"displacement has {uv.numel()} values, mesh needs "
                         f"{3 * dm.n_nodes}")
    tcoef, keep = None, None
    if T is not None and alpha != 0.0:
        if callable(T):
            vals = np.asarray(evaluate(T, dm.sample_points("centroid")), dtype=float)
            vals = np.array(np.broadcast_to(vals, (dm.n_elems,)), dtype=float)
            keep = torch.from_numpy(vals).to(dev)
            tcoef = N.Coef(ptr(keep), 0.0, N.COEF_ELEM, 0)
        else:
            tcoef, keep = dm.nodal_coef(np.asarray(T, dtype=float))
    sig = torch.empty(dm.n_elems * 6, dtype=torch.float64, device=dev)
    eps = torch.empty_like(sig)
    N.check(dm.rt.lib.cfem_element_stress(
        dm.rt.ctx, ptr(dm.nodes), ptr(dm.elems), dm.n_elems, dm.npe, ptr(uv),
        float(E), float(nu), ctypes.byref(tcoef) if tcoef is not None else None,
        float(alpha), float(T_ref), ptr(sig), ptr(eps), dm.rt.stream()))
    del keep
    return (sig.cpu().numpy().reshape(-1, 6), eps.cpu().numpy().reshape(-1, 6))


def element_stress_strain_3d(mesh, u, E, nu, T=None, alpha=0.0, T_ref=0.0):
    """Per-element (sig, eps), each (M, 6), Voigt order (elastic3d.py:171-185)."""
    return _element_stress(mesh, u, E, nu, T, alpha, T_ref)


def von_mises_3d(sig):
    """Von Mises stress of Voigt stresses (M, 6) or (6,)."""
    s = np.asarray(sig, dtype=float)
    sxx, syy, szz = s[..., 0], s[..., 1], s[..., 2]
    tyz, txz, txy = s[..., 3], s[..., 4], s[..., 5]
    return np.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2
                          + (szz - sxx) ** 2)
                   + 3.0 * (tyz ** 2 + txz ** 2 + txy ** 2))


__all__ = ["constitutive_3d", "boundary_faces", "assemble_elasticity_3d",
           "apply_dirichlet_vec3", "solve_elasticity_3d",
           "element_stress_strain_3d", "von_mises_3d", "_tet_gradients",
           "sp"]
