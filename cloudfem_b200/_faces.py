"""Boundary-face integrals on the device (O(surface) work).

Face lists come from the device face kernels (DeviceMesh.boundary_faces_device:
cfem_face_candidates, cfem_face_exterior); the integrals are the reference's
rules, evaluated by cfem_face_geometry (areas, quadrature points) and
cfem_face_integrate (per-face terms, then a stable sort by node or pattern
position and fixed-order sums into the device load vector and matrix):

* P1 Neumann / Robin on 3-node faces with the centroid value and the exact
  face mass h A / 12 (1 + d_ij) (cloudfem/fem/tet_heat.py:136-172);
* Tet10 Neumann / Robin on 6-node faces with the 6-point degree-4 Dunavant
  rule (cloudfem/fem/tet10.py:295-435);
* P1 traction, centroid value, t A / 3 per node (physics/elastic3d.py:171-186);
* Tet10 traction with the 3-point degree-2 rule
  (physics/elastic_tet10.py:50-66, 192-205).

Coefficients given as host functions are evaluated at the points the
device computed; constants never leave the host.
"""

import inspect

import numpy as np
import scipy.sparse as sp

from . import _native as N
from .device import evaluate, ptr

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
# 3-point degree-2 rule (elastic_tet10.py:50-53)
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


def add_at(F, idx, vals):
    """F[idx] += vals with repeated indices summed (np.add.at semantics),
    through np.bincount (host; used by host-side post-processing)."""
    idx = np.asarray(idx).ravel()
    vals = np.asarray(vals).ravel()
    if np.iscomplexobj(vals):
        F += (np.bincount(idx, weights=vals.real, minlength=len(F))
              + 1j * np.bincount(idx, weights=vals.imag, minlength=len(F)))
    else:
        F += np.bincount(idx, weights=vals, minlength=len(F))


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


class Rule:
    """A face quadrature rule as the device kernels take it: barycentric
    points on the corners, weights, shape values (nq, npf) and, for Robin,
    the mass tables mt[q] (npf, npf) with K_ab = A sum_q mt[q]_ab w_q h_q."""

    def __init__(self, npf, bary, w, shape, mt):
        self.npf = npf
        self.bary = np.ascontiguousarray(bary, dtype=float)
        self.w = np.ascontiguousarray(w, dtype=float)
        self.shape = np.ascontiguousarray(shape, dtype=float)
        self.mt = None if mt is None else np.ascontiguousarray(mt, dtype=float)
        self.nq = len(self.w)
        self._dev = {}

    def device(self, rt):
        """Device copies (bary, w, shape, mt), kept per device."""
        import torch
        key = str(rt.device)
        if key not in self._dev:
            def up(a):
                return None if a is None else torch.from_numpy(a).to(rt.device)
            self._dev[key] = (up(self.bary), up(self.w), up(self.shape), up(self.mt))
        return self._dev[key]


# P1: the centroid value; Robin with the exact face mass (1 + d_ij) / 12
P1 = Rule(3, [[1.0 / 3.0] * 3], [1.0], [[1.0 / 3.0] * 3],
          [(np.ones((3, 3)) + np.eye(3)) / 12.0])
# Tet10: Dunavant-6 for Neumann and Robin, the 3-point rule for traction
T10 = Rule(6, TRI_L6, TRI_W6, FACE_N6, np.einsum("qa,qb->qab", FACE_N6, FACE_N6))
T10_TRACTION = Rule(6, TRI_L3, TRI_W3, FACE_N3, None)


def _geometry(dm, faces_d, rule, need_pts):
    """Face areas (device) and, when asked, the quadrature points (host,
    (F, nq, 3)) for evaluating host functions."""
    import torch
    rt = dm.rt
    nf = int(faces_d.shape[0])
    area = torch.empty(max(nf, 1), dtype=torch.float64, device=rt.device)
    pts = (torch.empty((max(nf, 1), rule.nq, 3), dtype=torch.float64, device=rt.device)
           if need_pts else None)
    bary = rule.device(rt)[0]
    N.check(rt.lib.cfem_face_geometry(rt.ctx, rule.npf, nf, ptr(faces_d), ptr(dm.nodes),
                                      rule.nq, ptr(bary), ptr(pts), ptr(area), rt.stream()))
    return area, (pts[:nf].cpu().numpy() if need_pts else None)


def _host_values(spec, pts, nf, nq):
    """A float, or a host function's values at the points, as (nf, nq)."""
    v = evaluate(spec, pts) if callable(spec) else float(spec)
    return np.broadcast_to(np.asarray(v, dtype=float), (nf, nq))


def _to_device(rt, a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=float).ravel()).to(rt.device)


def add_load(dm, faces_d, rule, specs, F):
    """F (device, ncomp values per node) += A sum_q w_q N_a(x_q) load(x_q)
    over the faces, one spec per component (None: 0)."""
    rt = dm.rt
    nf = int(faces_d.shape[0])
    if nf == 0:
        return
    specs = [0.0 if v is None else v for v in specs]
    area, pts = _geometry(dm, faces_d, rule, any(callable(v) for v in specs))
    vals = np.stack([_host_values(v, pts, nf, rule.nq) for v in specs], axis=-1)
    d_vals = _to_device(rt, vals)
    _, w, shape, _ = rule.device(rt)
    N.check(rt.lib.cfem_face_integrate(
        rt.ctx, rule.npf, nf, ptr(faces_d), ptr(area), rule.nq, ptr(w), ptr(shape),
        len(specs), ptr(d_vals), ptr(F), None, None, None, None, dm.n_nodes, None,
        rt.stream()))


def add_robin(dm, faces_d, rule, h, tinf, F, K):
    """Robin convection over the faces: K (device node-pattern values) +=
    A sum_q mt_q w_q h(x_q), F += A sum_q w_q N_a h(x_q) T_inf(x_q)."""
    rt = dm.rt
    nf = int(faces_d.shape[0])
    if nf == 0:
        return
    area, pts = _geometry(dm, faces_d, rule, callable(h) or callable(tinf))
    hv = _host_values(h, pts, nf, rule.nq)
    load = hv * _host_values(tinf, pts, nf, rule.nq)
    d_h, d_load = _to_device(rt, hv), _to_device(rt, load)
    _, w, shape, mt = rule.device(rt)
    pat = dm.pattern
    N.check(rt.lib.cfem_face_integrate(
        rt.ctx, rule.npf, nf, ptr(faces_d), ptr(area), rule.nq, ptr(w), ptr(shape), 1,
        ptr(d_load), ptr(F), ptr(d_h), ptr(mt), pat.row_ptr, pat.col, dm.n_nodes, ptr(K),
        rt.stream()))


def face_csr(dm, face_lists, K):
    """The reference's CSR of face terms (tet_heat.py:160-172): one entry per
    pair of nodes of a common face (duplicates summed, indices sorted),
    its value read from the device pattern values K."""
    n = dm.n_nodes
    face_lists = [f for f in face_lists if len(f)]
    if not face_lists:
        return sp.csr_matrix((n, n))
    rows = np.concatenate([np.repeat(f[:, :, None], f.shape[1], axis=2).ravel()
                           for f in face_lists])
    cols = np.concatenate([np.repeat(f[:, None, :], f.shape[1], axis=1).ravel()
                           for f in face_lists])
    S = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    full = dm.pattern.to_scipy(1, K)
    r = np.repeat(np.arange(n), np.diff(S.indptr))
    S.data = np.asarray(full[r, S.indices]).ravel().astype(float)
    return S
