"""Boundary-face integrals (host side; O(surface) work).

Face lists come from the device candidate kernel (DeviceMesh.boundary_faces);
the per-face integrals below are the reference's rules evaluated over all
faces at once:

* P1 Neumann / Robin on 3-node faces with the centroid value
  (cloudfem/fem/tet_heat.py:136-172);
* Tet10 Neumann / Robin on 6-node faces with the 6-point degree-4 Dunavant
  rule (cloudfem/fem/tet10.py:295-435);
* P1 traction, centroid value, t A / 3 per node (physics/elastic3d.py:171-186);
* Tet10 traction with the 3-point degree-2 rule
  (physics/elastic_tet10.py:351-357, 494-508).
"""

import inspect

import numpy as np
import scipy.sparse as sp

from .device import evaluate

# 6-point Dunavant rule (barycentric points, weights summing to 1) as
# tabulated by the reference (tet10.py:300-308).
TRI_L6 = np.array([
    [0.445948490915965, 0.445948490915965, 0.108103018168070],
    [0.445948490915965, 0.108103018168070, 0.445948490915965],
    [0.108103018168070, 0.445948490915965, 0.445948490915965],
    [0.091576213509771, 0.091576213509771, 0.816847572980459],
    [0.091576213509771, 0.816847572980459, 0.091576213509771],
    [0.816847572980459, 0.091576213509771, 0.091576213509771],
])
TRI_W6 = np.array([0.223381589678011] * 3 + [0.109951743655322] * 3)
# 3-point degree-2 rule (elastic_tet10.py:352-355)
TRI_L3 = np.array([[2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0],
                   [1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0],
                   [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]])
TRI_W3 = np.full(3, 1.0 / 3.0)
FACE_EDGES = ((0, 1), (1, 2), (2, 0))


def face_shape6(l):
    """6-node triangle shape functions [c0, c1, c2, m01, m12, m20]."""
    l = np.asarray(l, dtype=float)
    out = np.empty(l.shape[:-1] + (6,))
    for i in range(3):
        out[..., i] = l[..., i] * (2.0 * l[..., i] - 1.0)
    for k, (i, j) in enumerate(FACE_EDGES):
        out[..., 3 + k] = 4.0 * l[..., i] * l[..., j]
    return out


FACE_N6 = face_shape6(TRI_L6)
FACE_N3 = face_shape6(TRI_L3)


def corner_geometry(nodes, faces):
    """Centroid (F, 3) and area (F,) of the corner triangles."""
    p = nodes[faces[:, :3]]
    cen = p.mean(axis=1)
    cr = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    return cen, 0.5 * np.linalg.norm(cr, axis=1), p


def add_at(F, idx, vals):
    """F[idx] += vals with repeated indices summed (np.add.at semantics),
    through np.bincount, which is much faster for large face sets."""
    idx = np.asarray(idx).ravel()
    vals = np.asarray(vals).ravel()
    if np.iscomplexobj(vals):
        F += (np.bincount(idx, weights=vals.real, minlength=len(F))
              + 1j * np.bincount(idx, weights=vals.imag, minlength=len(F)))
    else:
        F += np.bincount(idx, weights=vals, minlength=len(F))


def _as_array(v, n):
    return np.full(n, v) if np.isscalar(v) else v


def coo_csr(rows, cols, data, n):
    if len(data) == 0:
        return sp.csr_matrix((n, n))
    return sp.coo_matrix((np.concatenate(data),
                          (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n)).tocsr()


# ----------------------------------------------------------------- P1 faces

def p1_neumann(nodes, faces, q, F):
    cen, area, _ = corner_geometry(nodes, faces)
    qv = _as_array(evaluate(q, cen), len(faces))
    add_at(F, faces.ravel(), np.repeat(qv * area / 3.0, 3))


def p1_robin(nodes, faces, h, tinf, F, rows, cols, data):
    """Exact face mass h A/12 (1 + d_ij) and ambient load h T_inf A / 3."""
    cen, area, _ = corner_geometry(nodes, faces)
    hv = _as_array(evaluate(h, cen), len(faces))
    tv = _as_array(evaluate(tinf, cen), len(faces))
    fm = (np.ones((3, 3)) + np.eye(3)) / 12.0
    rows.append(np.repeat(faces[:, :, None], 3, axis=2).ravel())
    cols.append(np.repeat(faces[:, None, :], 3, axis=1).ravel())
    data.append(((hv * area)[:, None, None] * fm).ravel())
    add_at(F, faces.ravel(), np.repeat(hv * tv * area / 3.0, 3))


def p1_traction(nodes, faces, comps, rhs):
    cen, area, _ = corner_geometry(nodes, faces)
    for c, v in enumerate(comps):
        tv = _as_array(evaluate(0.0 if v is None else v, cen), len(faces))
        add_at(rhs, (3 * faces + c).ravel(),
                  np.repeat(tv * area / 3.0, 3))


# ----------------------------------------------------------------- Tet10 faces

def flux_fn(q):
    """float, f(x, y, z) or time-dependent f(x, y, z, t) (tet10.py:366-381)."""
    if not callable(q):
        v = float(q)
        return (lambda x, y, z, t: v), False
    try:
        n_par = len(inspect.signature(q).parameters)
    except (TypeError, ValueError):
        n_par = 3
    if n_par >= 4:
        return q, True
    return (lambda x, y, z, t: q(x, y, z)), False


def t10_points(nodes, faces, L):
    _, area, pc = corner_geometry(nodes, faces)
    return area, np.einsum("qc,fcd->fqd", L, pc)


def t10_neumann(nodes, faces, q, t, F):
    fn, _ = flux_fn(q)
    area, xq = t10_points(nodes, faces, TRI_L6)
    qv = evaluate(lambda x, y, z: fn(x, y, z, t), xq)
    qv = np.broadcast_to(qv, xq.shape[:-1])
    fe = area[:, None] * np.einsum("qa,fq->fa", FACE_N6, TRI_W6 * qv)
    add_at(F, faces.ravel(), fe.ravel())


def t10_robin(nodes, faces, h, tinf, F, rows, cols, data):
    area, xq = t10_points(nodes, faces, TRI_L6)
    hv = np.broadcast_to(evaluate(h, xq), xq.shape[:-1])
    tv = np.broadcast_to(evaluate(tinf, xq), xq.shape[:-1])
    Ke = area[:, None, None] * np.einsum("qa,fq,qb->fab", FACE_N6,
                                         TRI_W6 * hv, FACE_N6)
    fe = area[:, None] * np.einsum("qa,fq->fa", FACE_N6, TRI_W6 * hv * tv)
    add_at(F, faces.ravel(), fe.ravel())
    rows.append(np.repeat(faces[:, :, None], 6, axis=2).ravel())
    cols.append(np.repeat(faces[:, None, :], 6, axis=1).ravel())
    data.append(Ke.ravel())


def t10_traction(nodes, faces, comps, rhs):
    area, xq = t10_points(nodes, faces, TRI_L3)
    tv = np.stack([np.broadcast_to(evaluate(0.0 if v is None else v, xq),
                                   xq.shape[:-1]) for v in comps], axis=-1)
    fe = area[:, None, None] * np.einsum("q,qa,fqc->fac", TRI_W3, FACE_N3, tv)
    dofs = (3 * faces[:, :, None] + np.arange(3)).reshape(len(faces), -1)
    add_at(rhs, dofs.ravel(), fe.ravel())
