"""Second-order (Tet10) scalar problems on the GPU.

Drop-in for cloudfem/fem/tet10.py (``__all__`` at :52-56):

* ``shape_functions`` (:63-81), ``quadrature`` (:84-100) and
  ``element_operators`` (:103-126) are the small host helpers other modules
  import; the device kernels use the same tables from constant memory.
* ``assemble_tet10`` (:138-165): V sum_q w_q k(x_q) G_q G_q^T and
  V sum_q w_q f(x_q) N_q, one warp per element with the Keast-5 physical
  gradients staged in shared memory.
* ``assemble_mass_tet10`` (:229-249): rho_cp(centroid) V MASS_REF.
* ``_boundary_faces10`` (:329-352), ``assemble_boundary_terms_tet10``
  (:438-464) on 6-node faces with the 6-point Dunavant rule, integrated on
  the device (``_faces``).
* ``solve_tet10_poisson`` (:168-178) and ``transient_heat_tet10``
  (:467-548) solve on the device.
"""

from math import factorial

import numpy as np
import scipy.sparse as sp

from .. import _native as N
from .. import _faces
from .._driver import THETA, n_steps_of, solve_block, theta_march
from ..device import DeviceMesh, fixed_scalar
from ..mesh.tet10_mesh import EDGES
from .tet_heat import _terms, add_into, boundary_csr
from .tet_poisson import apply_dirichlet  # noqa: F401

__all__ = [
    "shape_functions", "quadrature", "element_operators",
    "assemble_tet10", "assemble_mass_tet10", "solve_tet10_poisson",
    "assemble_boundary_terms_tet10", "transient_heat_tet10",
]


def shape_functions(L):
    """Tet10 shape functions N (..., 10) and dN/dL (..., 10, 4)."""
    L = np.asarray(L, dtype=float)
    Nv = np.empty(L.shape[:-1] + (10,))
    dN = np.zeros(L.shape[:-1] + (10, 4))
    for i in range(4):
        Nv[..., i] = L[..., i] * (2.0 * L[..., i] - 1.0)
        dN[..., i, i] = 4.0 * L[..., i] - 1.0
    for k, (i, j) in enumerate(EDGES):
        Nv[..., 4 + k] = 4.0 * L[..., i] * L[..., j]
        dN[..., 4 + k, i] = 4.0 * L[..., j]
        dN[..., 4 + k, j] = 4.0 * L[..., i]
    return Nv, dN


def quadrature():
    """5-point Keast rule: (Lq (5, 4), wq (5,)), sum(wq) = 1."""
    a, b = 0.5, 1.0 / 6.0
    Lq = np.array([[0.25, 0.25, 0.25, 0.25], [a, b, b, b], [b, a, b, b],
                   [b, b, a, b], [b, b, b, a]])
    wq = np.array([-4.0 / 5.0] + [9.0 / 20.0] * 4)
    return Lq, wq


def element_operators(mesh, el):
    """(G (5, 10, 3), N (5, 10), xq (5, 3), vol) of one element."""
    el = np.asarray(el, dtype=int)
    p = mesh.nodes[el[:4]]
    J = np.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]], axis=1)
    vol = abs(float(np.linalg.det(J))) / 6.0
    Lq, _ = quadrature()
    Nq, dN = shape_functions(Lq)
    dxi = np.stack([dN[..., 1] - dN[..., 0], dN[..., 2] - dN[..., 0],
                    dN[..., 3] - dN[..., 0]], axis=-1)
    return dxi @ np.linalg.inv(J), Nq, Lq @ p, vol


def _scalar_fn(v):
    return v if callable(v) else (lambda x, y, z, v=v: v)


def _mass_reference():
    """Unit-volume Tet10 mass int N_a N_b dV / V from the barycentric
    moments 6 a! / (|a| + 3)! (tet10.py:185-223)."""
    polys = []
    for i in range(4):
        e2 = [0] * 4
        e2[i] = 2
        e1 = [0] * 4
        e1[i] = 1
        polys.append([(2.0, e2), (-1.0, e1)])
    for i, j in EDGES:
        e = [0] * 4
        e[i] += 1
        e[j] += 1
        polys.append([(4.0, e)])
    M = np.zeros((10, 10))
    for a in range(10):
        for b in range(10):
            s = 0.0
            for c1, a1 in polys[a]:
                for c2, a2 in polys[b]:
                    al = [x + y for x, y in zip(a1, a2)]
                    num = 1
                    for v in al:
                        num *= factorial(v)
                    s += c1 * c2 * 6.0 * num / factorial(sum(al) + 3)
            M[a, b] = s
    return M


_MASS_REF = _mass_reference()


def assemble_tet10(mesh, k=1.0, f=0.0):
    """Tet10 stiffness (csr) and load; k, f sampled at the Keast points."""
    dm = DeviceMesh(mesh)
    vals, rhs = dm.assemble(N.OP_T10_STIFF, coef=k, load=f)
    return dm.pattern.to_scipy(1, vals), rhs.cpu().numpy()


def solve_tet10_poisson(mesh, k=1.0, f=0.0, bc=None, *, precision="fp64",
                        rtol=None, max_iter=None):
    """Solve -div(k grad u) = f on a Tet10Mesh; returns nodal u."""
    dm = DeviceMesh(mesh)
    vals, rhs = dm.assemble(N.OP_T10_STIFF, coef=k, load=f)
    idx, v = fixed_scalar(mesh, bc)
    x = solve_block(dm, 1, vals, rhs, idx, v, precision, rtol, max_iter,
                    what="solve_tet10_poisson")
    return x.cpu().numpy()


def assemble_mass_tet10(mesh, rho_cp=1.0):
    """Consistent Tet10 capacity matrix, exact element integrals (csr)."""
    dm = DeviceMesh(mesh)
    vals, _ = dm.assemble(N.OP_T10_MASS, coef=rho_cp)
    return dm.pattern.to_scipy(1, vals)


_THETA = THETA


def _dirichlet_values(mesh, bc):
    idx, vals = fixed_scalar(mesh, bc)
    return dict(zip(idx.tolist(), vals.tolist()))


_FACES10 = (((0, 1, 2), (4, 5, 6)), ((0, 3, 1), (7, 8, 4)),
            ((0, 2, 3), (6, 9, 7)), ((1, 3, 2), (8, 9, 5)))
_FACE_EDGES = _faces.FACE_EDGES
_TRI_L6 = _faces.TRI_L6
_TRI_W6 = _faces.TRI_W6
_face_shape6 = _faces.face_shape6
_FACE_N6 = _faces.FACE_N6


def _boundary_faces10(mesh, name):
    """(F, 6) exterior 6-node faces [c0, c1, c2, m01, m12, m20]."""
    return DeviceMesh(mesh).boundary_faces(name, tet10=True)


def _flux_at(q, t):
    """A Neumann flux spec at time t: a float, or f(x, y, z) (tet10.py:366-381)."""
    if not callable(q):
        return float(q)
    fn, timedep = _faces.flux_fn(q)
    return (lambda x, y, z: fn(x, y, z, t)) if timedep else q


def _neumann_load(dm, mesh, neumann, t):
    """Device Neumann load of the named faces at time t."""
    _, F, _ = _terms(dm, mesh, {name: _flux_at(q, t) for name, q in neumann.items()},
                     None, _faces.T10, True)
    return F


def _robin_terms(dm, mesh, robin):
    """Device Robin terms: (K_add node-pattern values, F_add, face lists)."""
    return _terms(dm, mesh, None, robin, _faces.T10, True)


def assemble_boundary_terms_tet10(mesh, neumann=None, robin=None, t=0.0):
    """(K_add csr, F_add) of Neumann and Robin terms at time t."""
    dm = DeviceMesh(mesh)
    n = mesh.n_nodes
    neu = {name: _flux_at(q, t) for name, q in (neumann or {}).items()}
    K_add, F, faces = _terms(dm, mesh, neu, robin, _faces.T10, True)
    K = sp.csr_matrix((n, n))
    if robin:
        K = K + boundary_csr(dm, K_add, faces)
    return K, F.cpu().numpy()


def transient_heat_tet10(mesh, k=1.0, rho_cp=1.0, f=0.0, bc=None,
                         neumann=None, robin=None, t_end=1.0, dt=0.1, T0=0.0,
                         method="cn", *, precision="fp64", rtol=None,
                         max_iter=None):
    """Transient Tet10 heat conduction; returns (times, T_history)."""
    if method not in THETA:
        raise ValueError(f"unknown method {method!r}; "
                         f"use one of {sorted(THETA)}")
    theta = THETA[method]
    dm = DeviceMesh(mesh)
    dev = dm.rt.device
    K, F = dm.assemble(N.OP_T10_STIFF, coef=k, load=f)
    if robin:
        K_add, F_add, _ = _robin_terms(dm, mesh, robin)
        K = add_into(dm, K, K_add)
        F = F + F_add
    load_fn = None
    if neumann:
        timedep = any(_faces.flux_fn(q)[1] for q in neumann.values())
        if timedep:
            base = F

            def load_fn(step, h):
                Fs = ((1.0 - theta) * _neumann_load(dm, mesh, neumann, step * h)
                      + theta * _neumann_load(dm, mesh, neumann,
                                              (step + 1) * h))
                return base + Fs
        else:
            F = F + _neumann_load(dm, mesh, neumann, 0.0)
    C, _ = dm.assemble(N.OP_T10_MASS, coef=rho_cp)
    n_steps = n_steps_of(t_end, dt)
    idx, vals = fixed_scalar(mesh, bc)
    return theta_march(dm, K, C, F, idx, vals, t_end, n_steps, T0, theta,
                       precision, rtol, max_iter, load_fn)
