"""CPU oracle: a NumPy/SciPy restatement of CloudFEM's hot path.

TEST INFRASTRUCTURE ONLY. Only the test-suite, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import this module, and only
as the checker (or as the timed CPU baseline). The product path in
``cloudfem_b200`` never calls it.

Every function restates one reference function of zhangkalin627-svg/CloudFEM
(pure Python, NumPy + SciPy) with the per-element Python loop replaced by
array operations over all elements. The arithmetic per element and the
order of the COO triplets handed to ``scipy.sparse.coo_matrix(...).tocsr()``
are the reference's, so the CSR structure is identical and values agree to
round-off. Citations are ``file:line`` inside the reference project.

Third-party arithmetic used exactly as the reference uses it: SciPy's
COO->CSR duplicate summation and SuperLU (``spsolve`` / ``factorized``);
SciPy 1.18.1 and NumPy 2.3.5 in this image (``requirements.txt`` of the
reference pins only ``scipy>=1.10``, ``numpy>=1.24``).

Pinned against ``tests/golden/ref_fixtures.npz``, which
``tests/golden/make_golden.py`` produced by running the reference itself.
"""

import inspect
from math import factorial

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))   # tet10_mesh.py:33


class Mesh:
    """Minimal mesh record (``TetMesh`` / ``Tet10Mesh`` fields)."""

    def __init__(self, nodes, elements, boundaries, n_corners=None):
        self.nodes = np.asarray(nodes, dtype=float)
        self.elements = np.asarray(elements, dtype=np.int64)
        self.boundaries = dict(boundaries)
        self.n_corners = n_corners

    @property
    def n_nodes(self):
        return self.nodes.shape[0]

    @property
    def n_elements(self):
        return self.elements.shape[0]

    def element_volumes(self):
        """tet_mesh.py:36-44 / tet10_mesh.py:66-74."""
        p = self.nodes[self.elements[:, :4]]
        m = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                      p[:, 3] - p[:, 0]], axis=2)
        return np.abs(np.linalg.det(m)) / 6.0


# ------------------------------------------------------------------ helpers

def eval_points(spec, pts):
    """Evaluate float-or-callable(x, y, z) at points (..., 3).

    The reference calls the callable once per point with scalars
    (tet_poisson.py:54-56, tet10.py:152-153); here one array call is tried
    first and the scalar loop is the fallback when the callable does not
    broadcast.
    """
    shape = pts.shape[:-1]
    if not callable(spec):
        return np.full(shape, float(spec))
    flat = pts.reshape(-1, 3)
    try:
        with np.errstate(all="ignore"):
            v = np.asarray(spec(flat[:, 0], flat[:, 1], flat[:, 2]),
                           dtype=float)
        if v.shape == (flat.shape[0],):
            return v.reshape(shape)
        if v.ndim == 0:
            return np.full(shape, float(v))
    except Exception:  # noqa: BLE001 - non-vectorisable callable
        pass
    out = np.array([spec(x, y, z) for x, y, z in flat], dtype=float)
    return out.reshape(shape)


def coo_csr(rows, cols, data, shape):
    """``sp.coo_matrix((data, (rows, cols))).tocsr()`` as the reference."""
    return sp.coo_matrix((np.asarray(data).ravel(),
                          (np.asarray(rows).ravel(),
                           np.asarray(cols).ravel())),
                         shape=shape).tocsr()


# ------------------------------------------------------------------ meshes

def box_mesh(nx, ny, nz, xlim=(0.0, 1.0), ylim=(0.0, 1.0), zlim=(0.0, 1.0)):
    """tet_mesh.py:47-102: Kuhn 6-tet box mesh, cells in k, j, i order."""
    x = np.linspace(xlim[0], xlim[1], nx + 1)
    y = np.linspace(ylim[0], ylim[1], ny + 1)
    z = np.linspace(zlim[0], zlim[1], nz + 1)
    xx, yy, zz = np.meshgrid(x, y, z, indexing="ij")
    nodes = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])

    def idx(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx),
                          indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    c = [idx(i + di, j + dj, k + dk)
         for dk in (0, 1) for dj in (0, 1) for di in (0, 1)]
    n0, n1, n2, n3, n4, n5, n6, n7 = c
    tets = [(n0, n1, n3, n7), (n0, n1, n7, n5), (n0, n5, n7, n4),
            (n0, n3, n2, n7), (n0, n2, n6, n7), (n0, n6, n4, n7)]
    elements = np.stack([np.stack(t, axis=1) for t in tets],
                        axis=1).reshape(-1, 4).astype(np.int64)

    def face(fix_axis, val):
        if fix_axis == 0:
            kk, jj = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1),
                                 indexing="ij")
            return idx(val, jj.ravel(), kk.ravel())
        if fix_axis == 1:
            kk, ii = np.meshgrid(np.arange(nz + 1), np.arange(nx + 1),
                                 indexing="ij")
            return idx(ii.ravel(), val, kk.ravel())
        jj, ii = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1),
                             indexing="ij")
        return idx(ii.ravel(), jj.ravel(), val)

    bnd = {"xmin": face(0, 0), "xmax": face(0, nx), "ymin": face(1, 0),
           "ymax": face(1, ny), "zmin": face(2, 0), "zmax": face(2, nz)}
    bnd = {kk: np.asarray(v, dtype=np.int64) for kk, v in bnd.items()}
    return Mesh(nodes, elements, bnd)


def tet4_to_tet10(mesh):
    """tet10_mesh.py:77-112: midpoints in sorted-unique edge order."""
    els = mesh.elements
    n0 = mesh.n_nodes
    m = els.shape[0]
    pairs = np.stack([els[:, list(e)] for e in EDGES], axis=1)
    flat = np.sort(pairs.reshape(-1, 2), axis=1)
    uniq, inv = np.unique(flat, axis=0, return_inverse=True)
    inv = np.asarray(inv).ravel()
    mid = 0.5 * (mesh.nodes[uniq[:, 0]] + mesh.nodes[uniq[:, 1]])
    elements = np.column_stack([els, n0 + inv.reshape(m, 6)])
    nodes = np.vstack([mesh.nodes, mid])
    boundaries = {}
    for name, ids in mesh.boundaries.items():
        inset = np.zeros(n0, dtype=bool)
        inset[np.asarray(ids, dtype=np.int64)] = True
        keep = inset[uniq[:, 0]] & inset[uniq[:, 1]]
        extra = n0 + np.nonzero(keep)[0]
        boundaries[name] = np.sort(np.concatenate(
            [np.asarray(ids, dtype=np.int64), extra]))
    return Mesh(nodes, elements, boundaries, n_corners=n0)


def box_mesh_tet10(nx, ny, nz, xlim=(0.0, 1.0), ylim=(0.0, 1.0),
                   zlim=(0.0, 1.0)):
    """tet10_mesh.py:115-135: face sets re-selected by coordinate."""
    mesh = tet4_to_tet10(box_mesh(nx, ny, nz, xlim, ylim, zlim))
    tol = 1e-9 * max(1.0, float(np.ptp(mesh.nodes)))
    lims = {"xmin": (0, xlim[0]), "xmax": (0, xlim[1]),
            "ymin": (1, ylim[0]), "ymax": (1, ylim[1]),
            "zmin": (2, zlim[0]), "zmax": (2, zlim[1])}
    mesh.boundaries = {
        name: np.nonzero(np.abs(mesh.nodes[:, ax] - v) <= tol)[0]
        for name, (ax, v) in lims.items()}
    return mesh


# ------------------------------------------------------------------ P1 scalar

_G_REF = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0],
                   [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def tet_gradients(p):
    """tet_poisson.py:17-32 over a stack p (M, 4, 3) -> G (M, 4, 3), vol."""
    m = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                  p[:, 3] - p[:, 0]], axis=2)
    vol = np.abs(np.linalg.det(m)) / 6.0
    rhs = np.broadcast_to(_G_REF.T, m.shape[:-2] + (3, 4))
    g = np.linalg.solve(np.swapaxes(m, 1, 2), rhs)
    return np.swapaxes(g, 1, 2), vol


def assemble_p1(mesh, k=1.0, f=0.0):
    """tet_poisson.py:35-69."""
    n = mesh.n_nodes
    els = mesh.elements
    p = mesh.nodes[els]
    G, vol = tet_gradients(p)
    cen = p.mean(axis=1)
    kv = eval_points(k, cen)
    fv = eval_points(f, cen)
    ae = (kv * vol)[:, None, None] * np.einsum("eik,ejk->eij", G, G)
    rows = np.repeat(els[:, :, None], 4, axis=2)
    cols = np.repeat(els[:, None, :], 4, axis=1)
    A = coo_csr(rows, cols, ae, (n, n))
    rhs = np.zeros(n)
    np.add.at(rhs, els.ravel(), np.repeat(fv * vol / 4.0, 4))
    return A, rhs


def dirichlet_values(mesh, bc):
    """tet_heat.py:297-312: {node: value}; later names win."""
    fixed = {}
    if not bc:
        return fixed
    for name, value in bc.items():
        ids = (np.arange(mesh.n_nodes) if name == "all"
               else np.asarray(mesh.boundaries[name], dtype=np.int64))
        vals = eval_points(value, mesh.nodes[ids])
        fixed.update(zip(ids.tolist(), vals.tolist()))
    return fixed


def apply_dirichlet(A, rhs, mesh, bc):
    """tet_poisson.py:72-110, the same SciPy steps (explicit zeros kept)."""
    A = A.tolil()
    rhs = rhs.copy()
    fixed = dirichlet_values(mesh, bc)
    for i, v in fixed.items():
        A.rows[i] = [i]
        A.data[i] = [1.0]
        rhs[i] = v
    A = A.tocsr()
    fixed_idx = np.array(sorted(fixed), dtype=int)
    if len(fixed_idx):
        v = np.array([fixed[i] for i in fixed_idx])
        rhs = rhs - A[:, fixed_idx] @ v
        rhs[fixed_idx] = v
        A[:, fixed_idx] = 0
        A = A.tocsr()
        A[fixed_idx, fixed_idx] = 1.0
    return A, rhs


def solve_p1_poisson(mesh, k=1.0, f=0.0, bc=None):
    """tet_poisson.py:113-122."""
    A, rhs = assemble_p1(mesh, k, f)
    if bc:
        A, rhs = apply_dirichlet(A, rhs, mesh, bc)
    return np.asarray(spla.spsolve(A, rhs)).ravel()


# ------------------------------------------------------------------ P1 heat

def assemble_mass_p1(mesh, rho_cp=1.0):
    """tet_heat.py:72-94: rho_cp(centroid) * V/20 (1 + delta_ij)."""
    n = mesh.n_nodes
    els = mesh.elements
    base = (np.ones((4, 4)) + np.eye(4)) / 20.0
    vols = mesh.element_volumes()
    cen = mesh.nodes[els].mean(axis=1)
    me = (eval_points(rho_cp, cen) * vols)[:, None, None] * base
    rows = np.repeat(els[:, :, None], 4, axis=2)
    cols = np.repeat(els[:, None, :], 4, axis=1)
    return coo_csr(rows, cols, me, (n, n))


def _first_unique_faces(tris_local, keys, inset):
    """Faces (first occurrence order) whose key occurs once, all in set."""
    _, first, counts = np.unique(keys, axis=0, return_index=True,
                                 return_counts=True)
    sel = first[counts == 1]
    sel = sel[inset[keys[sel]].all(axis=1)]
    return tris_local[np.sort(sel)]


def boundary_faces_p1(mesh, name):
    """tet_heat.py:97-120 (= elastic3d.py:37-59): exterior faces on a set."""
    els = mesh.elements[:, :4]
    inset = np.zeros(mesh.n_nodes, dtype=bool)
    inset[np.asarray(mesh.boundaries[name], dtype=np.int64)] = True
    loc = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
    tris = np.stack([els[:, list(t)] for t in loc], axis=1).reshape(-1, 3)
    out = _first_unique_faces(tris, np.sort(tris, axis=1), inset)
    return out if len(out) else np.zeros((0, 3), dtype=np.int64)


def _face_geometry(nodes, tris):
    """tet_heat.py:123-128 over a stack of faces."""
    p = nodes[tris]
    cen = p.mean(axis=1)
    cr = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    return cen, 0.5 * np.linalg.norm(cr, axis=1)


def assemble_boundary_terms_p1(mesh, neumann=None, robin=None):
    """tet_heat.py:136-172: Neumann q A/3, Robin h A/12 (1 + delta_ij)."""
    n = mesh.n_nodes
    F = np.zeros(n)
    fm = (np.ones((3, 3)) + np.eye(3)) / 12.0
    rows, cols, data = [], [], []
    for name, q in (neumann or {}).items():
        tris = boundary_faces_p1(mesh, name)
        cen, area = _face_geometry(mesh.nodes, tris)
        np.add.at(F, tris.ravel(),
                  np.repeat(eval_points(q, cen) * area / 3.0, 3))
    for name, (h, tinf) in (robin or {}).items():
        tris = boundary_faces_p1(mesh, name)
        cen, area = _face_geometry(mesh.nodes, tris)
        hv = eval_points(h, cen)
        ke = (hv * area)[:, None, None] * fm
        rows.append(np.repeat(tris[:, :, None], 3, axis=2).ravel())
        cols.append(np.repeat(tris[:, None, :], 3, axis=1).ravel())
        data.append(ke.ravel())
        np.add.at(F, tris.ravel(),
                  np.repeat(hv * eval_points(tinf, cen) * area / 3.0, 3))
    if data:
        K = coo_csr(np.concatenate(rows), np.concatenate(cols),
                    np.concatenate(data), (n, n))
    else:
        K = coo_csr([], [], [], (n, n))
    return K, F


THETA = {"be": 1.0, "implicit_euler": 1.0, "cn": 0.5, "crank_nicolson": 0.5}


def _theta_march(A_sys, R_sys, F, mesh, bc, t_end, n_steps, T0,
                 load_fn=None):
    """tet_heat.py:239-274 / tet10.py:509-548: one LU, then the steps."""
    n = mesh.n_nodes
    h = t_end / n_steps
    fixed = dirichlet_values(mesh, bc)
    if fixed:
        A_bc, _ = apply_dirichlet(A_sys, np.zeros(n), mesh, bc)
        fixed_idx = np.array(sorted(fixed), dtype=int)
        fixed_val = np.array([fixed[i] for i in fixed_idx])
        cols = A_sys.tocsr()[:, fixed_idx]
    else:
        A_bc = A_sys
        fixed_idx = fixed_val = cols = None
    solve = spla.factorized(A_bc.tocsc())
    T = (np.full(n, T0, dtype=float) if np.isscalar(T0)
         else np.asarray(T0, dtype=float).copy())
    if fixed_idx is not None:
        T[fixed_idx] = fixed_val
    times = [0.0]
    hist = [T.copy()]
    for step in range(n_steps):
        F_step = F if load_fn is None else load_fn(step, h)
        rhs = R_sys @ T + h * F_step
        if fixed_idx is not None:
            rhs = rhs - cols @ fixed_val
            rhs[fixed_idx] = fixed_val
        T = np.asarray(solve(rhs)).ravel()
        if fixed_idx is not None:
            T[fixed_idx] = fixed_val
        times.append(times[-1] + h)
        hist.append(T.copy())
    times[-1] = t_end
    return np.array(times), np.array(hist)


def _n_steps(t_end, dt):
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    return n_steps


def transient_heat_p1(mesh, k=1.0, rho_cp=1.0, f=0.0, bc=None,
                      neumann=None, robin=None, t_end=1.0, dt=0.1, T0=0.0,
                      method="cn"):
    """tet_heat.py:197-274."""
    if method not in THETA:
        raise ValueError(f"unknown method {method!r}")
    theta = THETA[method]
    K, F = assemble_p1(mesh, k, f)
    K_add, F_add = assemble_boundary_terms_p1(mesh, neumann, robin)
    K = K + K_add
    F = F + F_add
    C = assemble_mass_p1(mesh, rho_cp)
    n_steps = _n_steps(t_end, dt)
    h = t_end / n_steps
    A_sys = C + theta * h * K
    R_sys = C - (1.0 - theta) * h * K
    return _theta_march(A_sys, R_sys, F, mesh, bc, t_end, n_steps, T0)


# ------------------------------------------------------------------ Tet10

def shape_functions(L):
    """tet10.py:63-81."""
    L = np.asarray(L, dtype=float)
    N = np.empty(L.shape[:-1] + (10,))
    dN = np.zeros(L.shape[:-1] + (10, 4))
    for i in range(4):
        N[..., i] = L[..., i] * (2.0 * L[..., i] - 1.0)
        dN[..., i, i] = 4.0 * L[..., i] - 1.0
    for kk, (i, j) in enumerate(EDGES):
        N[..., 4 + kk] = 4.0 * L[..., i] * L[..., j]
        dN[..., 4 + kk, i] = 4.0 * L[..., j]
        dN[..., 4 + kk, j] = 4.0 * L[..., i]
    return N, dN


def quadrature():
    """tet10.py:84-100: 5-point Keast rule, weights sum to 1."""
    a, b = 0.5, 1.0 / 6.0
    Lq = np.array([[0.25] * 4, [a, b, b, b], [b, a, b, b], [b, b, a, b],
                   [b, b, b, a]])
    wq = np.array([-4.0 / 5.0] + [9.0 / 20.0] * 4)
    return Lq, wq


def _dN_dxi(L):
    _, dN = shape_functions(L)
    return np.stack([dN[..., 1] - dN[..., 0], dN[..., 2] - dN[..., 0],
                     dN[..., 3] - dN[..., 0]], axis=-1)


def element_operators_all(mesh):
    """tet10.py:103-126 for every element: G (M,5,10,3), N, xq, vol."""
    p = mesh.nodes[mesh.elements[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                  p[:, 3] - p[:, 0]], axis=2)
    vol = np.abs(np.linalg.det(J)) / 6.0
    Lq, _ = quadrature()
    N, _ = shape_functions(Lq)
    Jinv = np.linalg.inv(J)
    G = np.einsum("qai,eij->eqaj", _dN_dxi(Lq), Jinv)
    xq = np.einsum("qc,ecd->eqd", Lq, p)
    return G, N, xq, vol


def assemble_tet10(mesh, k=1.0, f=0.0):
    """tet10.py:138-165."""
    n = mesh.n_nodes
    els = mesh.elements
    _, wq = quadrature()
    G, N, xq, vol = element_operators_all(mesh)
    kv = eval_points(k, xq)
    fv = eval_points(f, xq)
    Ke = vol[:, None, None] * np.einsum("eq,eqji,eqki->ejk", wq * kv, G, G)
    fe = vol[:, None] * np.einsum("qa,eq->ea", N, wq * fv)
    rows = np.repeat(els[:, :, None], 10, axis=2)
    cols = np.repeat(els[:, None, :], 10, axis=1)
    A = coo_csr(rows, cols, Ke, (n, n))
    rhs = np.zeros(n)
    np.add.at(rhs, els.ravel(), fe.ravel())
    return A, rhs


def solve_tet10_poisson(mesh, k=1.0, f=0.0, bc=None):
    """tet10.py:168-178."""
    A, rhs = assemble_tet10(mesh, k, f)
    if bc:
        A, rhs = apply_dirichlet(A, rhs, mesh, bc)
    return np.asarray(spla.spsolve(A, rhs)).ravel()


def _shape_polys():
    polys = []
    for i in range(4):
        e2 = [0, 0, 0, 0]
        e2[i] = 2
        e1 = [0, 0, 0, 0]
        e1[i] = 1
        polys.append([(2.0, tuple(e2)), (-1.0, tuple(e1))])
    for (i, j) in EDGES:
        e = [0, 0, 0, 0]
        e[i] += 1
        e[j] += 1
        polys.append([(4.0, tuple(e))])
    return polys


def mass_reference():
    """tet10.py:185-226: exact unit-volume Tet10 mass, 6 a!/(|a|+3)!."""
    polys = _shape_polys()
    M = np.zeros((10, 10))
    for a in range(10):
        for b in range(10):
            s = 0.0
            for c1, a1 in polys[a]:
                for c2, a2 in polys[b]:
                    al = tuple(x + y for x, y in zip(a1, a2))
                    num = 1
                    for v in al:
                        num *= factorial(v)
                    s += c1 * c2 * 6.0 * num / factorial(sum(al) + 3)
            M[a, b] = s
    return M


MASS_REF = mass_reference()


def assemble_mass_tet10(mesh, rho_cp=1.0):
    """tet10.py:229-249: rho_cp(centroid) * V * MASS_REF."""
    n = mesh.n_nodes
    els = mesh.elements
    vols = mesh.element_volumes()
    cen = mesh.nodes[els[:, :4]].mean(axis=1)
    me = (eval_points(rho_cp, cen) * vols)[:, None, None] * MASS_REF
    rows = np.repeat(els[:, :, None], 10, axis=2)
    cols = np.repeat(els[:, None, :], 10, axis=1)
    return coo_csr(rows, cols, me, (n, n))


FACES10 = (((0, 1, 2), (4, 5, 6)), ((0, 3, 1), (7, 8, 4)),
           ((0, 2, 3), (6, 9, 7)), ((1, 3, 2), (8, 9, 5)))   # tet10.py:287
TRI_L6 = np.array([
    [0.445948490915965, 0.445948490915965, 0.108103018168070],
    [0.445948490915965, 0.108103018168070, 0.445948490915965],
    [0.108103018168070, 0.445948490915965, 0.445948490915965],
    [0.091576213509771, 0.091576213509771, 0.816847572980459],
    [0.091576213509771, 0.816847572980459, 0.091576213509771],
    [0.816847572980459, 0.091576213509771, 0.091576213509771],
])                                                            # tet10.py:300
TRI_W6 = np.array([0.223381589678011] * 3 + [0.109951743655322] * 3)


def face_shape6(l):
    """tet10.py:311-323: 6-node triangle shape functions."""
    N = np.empty(l.shape[:-1] + (6,))
    for i in range(3):
        N[..., i] = l[..., i] * (2.0 * l[..., i] - 1.0)
    for kk, (i, j) in enumerate(((0, 1), (1, 2), (2, 0))):
        N[..., 3 + kk] = 4.0 * l[..., i] * l[..., j]
    return N


FACE_N6 = face_shape6(TRI_L6)


def boundary_faces10(mesh, name):
    """tet10.py:329-352 (= elastic_tet10.py:68-91): (F, 6) faces."""
    els = mesh.elements
    inset = np.zeros(mesh.n_nodes, dtype=bool)
    inset[np.asarray(mesh.boundaries[name], dtype=np.int64)] = True
    full = np.stack([els[:, list(c + m)] for c, m in FACES10],
                    axis=1).reshape(-1, 6)
    out = _first_unique_faces(full, np.sort(full[:, :3], axis=1), inset)
    return out if len(out) else np.zeros((0, 6), dtype=np.int64)


def _face10_geometry(nodes, faces, L):
    pc = nodes[faces[:, :3]]
    cr = np.cross(pc[:, 1] - pc[:, 0], pc[:, 2] - pc[:, 0])
    area = 0.5 * np.linalg.norm(cr, axis=1)
    xq = np.einsum("qc,fcd->fqd", L, pc)
    return area, xq


def _flux_fn(q):
    """tet10.py:366-381: float, f(x,y,z) or time-dependent f(x,y,z,t)."""
    if not callable(q):
        v = float(q)
        return (lambda x, y, z, t: v + 0.0 * x), False
    try:
        n_par = len(inspect.signature(q).parameters)
    except (TypeError, ValueError):
        n_par = 3
    if n_par >= 4:
        return q, True
    return (lambda x, y, z, t: q(x, y, z)), False


def _eval_t(fn, pts, t):
    return eval_points(lambda x, y, z: fn(x, y, z, t), pts)


def neumann_load_tet10(mesh, neumann, t):
    """tet10.py:384-401: F += area * sum_q w_q q(x_q, t) N6_q."""
    F = np.zeros(mesh.n_nodes)
    for name, q in neumann.items():
        fn, _ = _flux_fn(q)
        faces = boundary_faces10(mesh, name)
        area, xq = _face10_geometry(mesh.nodes, faces, TRI_L6)
        qv = _eval_t(fn, xq, t)
        fe = area[:, None] * np.einsum("qa,fq->fa", FACE_N6, TRI_W6 * qv)
        np.add.at(F, faces.ravel(), fe.ravel())
    return F


def robin_terms_tet10(mesh, robin):
    """tet10.py:404-435: face mass h int N N dA and h T_inf int N dA."""
    n = mesh.n_nodes
    F = np.zeros(n)
    rows, cols, data = [], [], []
    for name, (h, tinf) in robin.items():
        faces = boundary_faces10(mesh, name)
        area, xq = _face10_geometry(mesh.nodes, faces, TRI_L6)
        hv = eval_points(h, xq)
        tv = eval_points(tinf, xq)
        Ke = area[:, None, None] * np.einsum("qa,fq,qb->fab", FACE_N6,
                                             TRI_W6 * hv, FACE_N6)
        fe = area[:, None] * np.einsum("qa,fq->fa", FACE_N6,
                                       TRI_W6 * hv * tv)
        np.add.at(F, faces.ravel(), fe.ravel())
        rows.append(np.repeat(faces[:, :, None], 6, axis=2).ravel())
        cols.append(np.repeat(faces[:, None, :], 6, axis=1).ravel())
        data.append(Ke.ravel())
    if data:
        K = coo_csr(np.concatenate(rows), np.concatenate(cols),
                    np.concatenate(data), (n, n))
    else:
        K = sp.csr_matrix((n, n))
    return K, F


def assemble_boundary_terms_tet10(mesh, neumann=None, robin=None, t=0.0):
    """tet10.py:438-464."""
    n = mesh.n_nodes
    F = np.zeros(n)
    K = sp.csr_matrix((n, n))
    if neumann:
        F += neumann_load_tet10(mesh, neumann, t)
    if robin:
        Kr, Fr = robin_terms_tet10(mesh, robin)
        K = K + Kr
        F += Fr
    return K, F


def transient_heat_tet10(mesh, k=1.0, rho_cp=1.0, f=0.0, bc=None,
                         neumann=None, robin=None, t_end=1.0, dt=0.1,
                         T0=0.0, method="cn"):
    """tet10.py:467-548."""
    if method not in THETA:
        raise ValueError(f"unknown method {method!r}")
    theta = THETA[method]
    K, F = assemble_tet10(mesh, k, f)
    if robin:
        K_add, F_add = assemble_boundary_terms_tet10(mesh, robin=robin)
        K = K + K_add
        F = F + F_add
    load_fn = None
    if neumann:
        timedep = any(_flux_fn(q)[1] for q in neumann.values())
        if timedep:
            F_base = F

            def load_fn(step, h):
                return F_base + (
                    (1.0 - theta) * neumann_load_tet10(mesh, neumann, step * h)
                    + theta * neumann_load_tet10(mesh, neumann,
                                                 (step + 1) * h))
        else:
            F = F + neumann_load_tet10(mesh, neumann, 0.0)
    C = assemble_mass_tet10(mesh, rho_cp)
    n_steps = _n_steps(t_end, dt)
    h = t_end / n_steps
    A_sys = C + theta * h * K
    R_sys = C - (1.0 - theta) * h * K
    return _theta_march(A_sys, R_sys, F, mesh, bc, t_end, n_steps, T0,
                        load_fn)


# ------------------------------------------------------------------ elasticity

def constitutive_3d(E, nu):
    """elastic3d.py:26-34: Voigt [xx, yy, zz, yz, xz, xy]."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2.0 * mu
    D[0, 1] = D[0, 2] = D[1, 0] = D[1, 2] = D[2, 0] = D[2, 1] = lam
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    return D


def strain_displacement(G):
    """elastic3d.py:62-77 / elastic_tet10.py:94-109 over (..., n, 3)."""
    nn = G.shape[-2]
    B = np.zeros(G.shape[:-2] + (6, 3 * nn))
    gx, gy, gz = G[..., 0], G[..., 1], G[..., 2]
    B[..., 0, 0::3] = gx
    B[..., 1, 1::3] = gy
    B[..., 2, 2::3] = gz
    B[..., 3, 1::3] = gz
    B[..., 3, 2::3] = gy
    B[..., 4, 0::3] = gz
    B[..., 4, 2::3] = gx
    B[..., 5, 0::3] = gy
    B[..., 5, 1::3] = gx
    return B


def dof_map(els):
    """elastic3d.py:80-85: DOF 3 i + c, interleaved."""
    return (3 * els[..., :, None] + np.arange(3)).reshape(
        els.shape[:-1] + (3 * els.shape[-1],))


def _components(vals):
    """elastic3d.py:88-102: None -> 0."""
    return [0.0 if v is None else v for v in vals]


_EYE3 = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])


def _traction_p1(mesh, traction, rhs):
    for name, vals in (traction or {}).items():
        comps = _components(vals)
        tris = boundary_faces_p1(mesh, name)
        p = mesh.nodes[tris]
        cen = p.mean(axis=1)
        tv = np.stack([eval_points(c, cen) for c in comps], axis=1)
        cr = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        area = 0.5 * np.linalg.norm(cr, axis=1)
        contrib = np.repeat((tv * area[:, None] / 3.0)[:, None, :], 3, 1)
        np.add.at(rhs, dof_map(tris).ravel(), contrib.ravel())


def assemble_elasticity_p1(mesh, E, nu, body=None, traction=None, T=None,
                           alpha=0.0, T_ref=0.0):
    """elastic3d.py:105-189."""
    D = constitutive_3d(E, nu)
    n3 = 3 * mesh.n_nodes
    els = mesh.elements
    p = mesh.nodes[els]
    G, vol = tet_gradients(p)
    B = strain_displacement(G)
    ke = np.einsum("eai,ab,ebj->eij", B, D, B) * vol[:, None, None]
    dofs = dof_map(els)
    rows = np.repeat(dofs[:, :, None], 12, axis=2)
    cols = np.repeat(dofs[:, None, :], 12, axis=1)
    A = coo_csr(rows, cols, ke, (n3, n3))
    rhs = np.zeros(n3)
    cen = p.mean(axis=1)
    comps = _components(body) if body is not None else [0.0] * 3
    bv = np.stack([eval_points(c, cen) for c in comps], axis=1)
    contrib = np.repeat((bv * vol[:, None] / 4.0)[:, None, :], 4, axis=1)
    np.add.at(rhs, dofs.ravel(), contrib.ravel())
    if T is not None and alpha != 0.0:
        if callable(T):
            Tc = eval_points(T, cen)
        else:
            Tc = np.asarray(T, dtype=float)[els].mean(axis=1)
        eth = (alpha * (Tc - T_ref))[:, None] * _EYE3
        fth = np.einsum("eai,ab,eb->ei", B, D, eth) * vol[:, None]
        np.add.at(rhs, dofs.ravel(), fth.ravel())
    _traction_p1(mesh, traction, rhs)
    return A, rhs


def vector_dirichlet_values(mesh, bc):
    """elastic3d.py:204-218: {dof: value}, None components stay free."""
    fixed = {}
    for name, vals in bc.items():
        ids = (np.arange(mesh.n_nodes) if name == "all"
               else np.asarray(mesh.boundaries[name], dtype=np.int64))
        for comp, v in enumerate(vals):
            if v is None:
                continue
            vv = eval_points(v, mesh.nodes[ids])
            fixed.update(zip((3 * ids + comp).tolist(), vv.tolist()))
    return fixed


def apply_dirichlet_vec3(A, rhs, mesh, bc):
    """elastic3d.py:192-233: free-DOF reduction, then SuperLU."""
    rhs = np.asarray(rhs, dtype=float).copy()
    n3 = 3 * mesh.n_nodes
    fixed = vector_dirichlet_values(mesh, bc)
    u = np.zeros(n3)
    fixed_idx = np.array(sorted(fixed), dtype=int)
    if len(fixed_idx):
        v = np.array([fixed[i] for i in fixed_idx])
        u[fixed_idx] = v
        free = np.ones(n3, dtype=bool)
        free[fixed_idx] = False
        A = A.tocsr()
        rhs_free = rhs[free] - A[free][:, fixed_idx] @ v
        A_free = A[free][:, free].tocsr()
        u[free] = spla.spsolve(A_free, rhs_free)
    else:
        u = np.asarray(spla.spsolve(A.tocsr(), rhs)).ravel()
    return u


def solve_elasticity_p1(mesh, E, nu, bc=None, body=None, traction=None,
                        T=None, alpha=0.0, T_ref=0.0):
    """elastic3d.py:236-249."""
    A, rhs = assemble_elasticity_p1(mesh, E, nu, body, traction, T, alpha,
                                    T_ref)
    if bc:
        u = apply_dirichlet_vec3(A, rhs, mesh, bc)
    else:
        u = np.asarray(spla.spsolve(A.tocsr(), rhs)).ravel()
    return u[0::3].copy(), u[1::3].copy(), u[2::3].copy()


def _as_vector(mesh, u):
    if isinstance(u, tuple):
        uv = np.empty(3 * mesh.n_nodes)
        uv[0::3], uv[1::3], uv[2::3] = u
        return uv
    return np.asarray(u, dtype=float).ravel()


def element_stress_strain_p1(mesh, u, E, nu, T=None, alpha=0.0, T_ref=0.0):
    """elastic3d.py:252-289."""
    uv = _as_vector(mesh, u)
    D = constitutive_3d(E, nu)
    els = mesh.elements
    p = mesh.nodes[els]
    G, _ = tet_gradients(p)
    B = strain_displacement(G)
    eps = np.einsum("eai,ei->ea", B, uv[dof_map(els)])
    eth = np.zeros_like(eps)
    if T is not None and alpha != 0.0:
        cen = p.mean(axis=1)
        Tc = (eval_points(T, cen) if callable(T)
              else np.asarray(T, dtype=float)[els].mean(axis=1))
        eth = (alpha * (Tc - T_ref))[:, None] * _EYE3
    sig = np.einsum("ab,eb->ea", D, eps - eth)
    return sig, eps


def von_mises_3d(sig):
    """elastic3d.py:292-302."""
    s = np.asarray(sig, dtype=float)
    sxx, syy, szz = s[..., 0], s[..., 1], s[..., 2]
    tyz, txz, txy = s[..., 3], s[..., 4], s[..., 5]
    return np.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2
                          + (szz - sxx) ** 2)
                   + 3.0 * (tyz ** 2 + txz ** 2 + txy ** 2))


TRI_L3 = np.array([[2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0],
                   [1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0],
                   [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]])    # elastic_tet10.py:52
TRI_W3 = np.full(3, 1.0 / 3.0)


def assemble_elasticity_tet10(mesh, E, nu, body=None, traction=None, T=None,
                              alpha=0.0, T_ref=0.0):
    """elastic_tet10.py:135-211."""
    _, wq = quadrature()
    D = constitutive_3d(E, nu)
    n3 = 3 * mesh.n_nodes
    els = mesh.elements
    G, N, xq, vol = element_operators_all(mesh)
    dofs = dof_map(els)
    B = strain_displacement(G)                               # (M,5,6,30)
    DB = np.einsum("ab,eqbi->eqai", D, B)
    Ke = vol[:, None, None] * np.einsum("q,eqai,eqaj->eij", wq, B, DB)
    rows = np.repeat(dofs[:, :, None], 30, axis=2)
    cols = np.repeat(dofs[:, None, :], 30, axis=1)
    A = coo_csr(rows, cols, Ke, (n3, n3))
    rhs = np.zeros(n3)
    comps = _components(body) if body is not None else [0.0] * 3
    bv = np.stack([eval_points(c, xq) for c in comps], axis=-1)  # (M,5,3)
    fe = vol[:, None, None] * np.einsum("q,qa,eqc->eac", wq, N, bv)
    np.add.at(rhs, dofs.ravel(), fe.ravel())
    if T is not None and alpha != 0.0:
        if callable(T):
            Tq = eval_points(T, xq)
        else:
            Tq = np.einsum("qa,ea->eq", N, np.asarray(T, dtype=float)[els])
        eth = (alpha * (Tq - T_ref))[..., None] * _EYE3          # (M,5,6)
        Deth = eth @ D.T
        fth = vol[:, None] * np.einsum("q,eqai,eqa->ei", wq, B, Deth)
        np.add.at(rhs, dofs.ravel(), fth.ravel())
    if traction:
        Nf = face_shape6(TRI_L3)
        for name, vals in traction.items():
            comps = _components(vals)
            faces = boundary_faces10(mesh, name)
            area, xqf = _face10_geometry(mesh.nodes, faces, TRI_L3)
            tv = np.stack([eval_points(c, xqf) for c in comps], axis=-1)
            fe = area[:, None, None] * np.einsum("q,qa,fqc->fac", TRI_W3,
                                                 Nf, tv)
            np.add.at(rhs, dof_map(faces).ravel(), fe.ravel())
    return A, rhs


def solve_elasticity_tet10(mesh, E, nu, bc=None, body=None, traction=None,
                           T=None, alpha=0.0, T_ref=0.0):
    """elastic_tet10.py:214-229."""
    A, rhs = assemble_elasticity_tet10(mesh, E, nu, body, traction, T,
                                       alpha, T_ref)
    if bc:
        u = apply_dirichlet_vec3(A, rhs, mesh, bc)
    else:
        u = np.asarray(spla.spsolve(A.tocsr(), rhs)).ravel()
    return u[0::3].copy(), u[1::3].copy(), u[2::3].copy()


def element_stress_tet10(mesh, u, E, nu, T=None, alpha=0.0, T_ref=0.0):
    """elastic_tet10.py:232-279: centroid strain and stress."""
    uv = _as_vector(mesh, u)
    D = constitutive_3d(E, nu)
    els = mesh.elements
    Lc = np.array([[0.25, 0.25, 0.25, 0.25]])
    Nc, _ = shape_functions(Lc)
    dxi = _dN_dxi(Lc)[0]
    p = mesh.nodes[els[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                  p[:, 3] - p[:, 0]], axis=2)
    Gc = np.einsum("ai,eij->eaj", dxi, np.linalg.inv(J))
    B = strain_displacement(Gc)
    eps = np.einsum("eai,ei->ea", B, uv[dof_map(els)])
    eth = np.zeros_like(eps)
    if T is not None and alpha != 0.0:
        Tc = (eval_points(T, p.mean(axis=1)) if callable(T)
              else np.asarray(T, dtype=float)[els] @ Nc[0])
        eth = (alpha * (Tc - T_ref))[:, None] * _EYE3
    sig = np.einsum("ab,eb->ea", D, eps - eth)
    return sig, eps


# ------------------------------------------------------------------ A-V blocks

_EPS = np.zeros((3, 3, 3))
for _i, _j, _k in [(0, 1, 2), (1, 2, 0), (2, 0, 1)]:
    _EPS[_i, _j, _k] = 1.0
for _i, _j, _k in [(0, 2, 1), (2, 1, 0), (1, 0, 2)]:
    _EPS[_i, _j, _k] = -1.0


def conductor_components(mesh, conducting):
    """em3d_tet10.py:140-169: union-find, pin the smallest node per part."""
    cond_nodes = np.unique(mesh.elements[conducting])
    parent = {int(nd): int(nd) for nd in cond_nodes}

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for el in mesh.elements[conducting]:
        ids = [int(i) for i in el]
        for other in ids[1:]:
            ra, rb = find(ids[0]), find(other)
            if ra != rb:
                parent[rb] = ra
    comps = {}
    for nd in cond_nodes:
        comps.setdefault(find(int(nd)), []).append(int(nd))
    pinned = {min(mem) for mem in comps.values()}
    v_nodes = np.array([nd for nd in cond_nodes if nd not in pinned],
                       dtype=np.int64)
    return v_nodes


def assemble_tet10_av(mesh, nu, sigma=0.0, gauge_eps=1e-6):
    """em3d_tet10.py:172-264: real blocks K, M, G, S of the A-V system."""
    n = mesh.n_nodes
    els = mesh.elements
    cen = mesh.nodes[els[:, :4]].mean(axis=1)
    nu_e = eval_points(nu, cen)
    sig_e = eval_points(sigma, cen)
    conducting = sig_e > 0.0
    sig_max = sig_e.max() if conducting.any() else 0.0
    sig_reg = gauge_eps * sig_max
    v_nodes = conductor_components(mesh, conducting)
    v_col = np.full(n, -1, dtype=np.int64)
    v_col[v_nodes] = np.arange(len(v_nodes))
    n_v = len(v_nodes)
    _, wq = quadrature()
    G, N, _, vol = element_operators_all(mesh)
    dofs = dof_map(els)                                       # (M,30)

    Cc = np.einsum("klm,eqpl->eqpmk", _EPS, G)
    ke = (nu_e * vol)[:, None, None, None, None] * np.einsum(
        "q,eqpmk,eqrnk->epmrn", wq, Cc, Cc)
    ke = ke.reshape(-1, 30, 30)
    K = coo_csr(np.repeat(dofs[:, :, None], 30, axis=2),
                np.repeat(dofs[:, None, :], 30, axis=1), ke, (3 * n, 3 * n))

    seff = np.where(conducting, sig_e, sig_reg)
    mm = seff > 0.0
    me = (seff * vol)[mm][:, None, None] * MASS_REF
    rows, cols, data = [], [], []
    for e_idx, e in enumerate(np.nonzero(mm)[0]):
        for m in range(3):
            dm = dofs[e, m::3]
            rows.append(np.repeat(dm, 10))
            cols.append(np.tile(dm, 10))
            data.append(me[e_idx].ravel())

    def _coo(r, c, d, shape):
        if d:
            return coo_csr(np.concatenate(r), np.concatenate(c),
                           np.concatenate(d), shape)
        return sp.csr_matrix(shape)

    M = _coo(rows, cols, data, (3 * n, 3 * n))

    g_r, g_c, g_d, s_r, s_c, s_d = [], [], [], [], [], []
    for e in np.nonzero(conducting)[0]:
        el = els[e]
        se = float(sig_e[e])
        smask = v_col[el] >= 0
        scol = v_col[el][smask]
        if scol.size:
            ge = se * vol[e] * np.einsum("q,qp,qjm->pmj", wq, N, G[e])
            ge = ge[:, :, smask]
            g_r.append(np.repeat(dofs[e], scol.size))
            g_c.append(np.tile(scol, 30))
            g_d.append(ge.ravel())
            se_mat = se * vol[e] * np.einsum("q,qil,qjl->ij", wq, G[e], G[e])
            se_mat = se_mat[np.ix_(smask, smask)]
            s_r.append(np.repeat(scol, scol.size))
            s_c.append(np.tile(scol, scol.size))
            s_d.append(se_mat.ravel())
    Gs = _coo(g_r, g_c, g_d, (3 * n, n_v))
    S = _coo(s_r, s_c, s_d, (n_v, n_v))
    return K, M, Gs, S, v_nodes, sig_e, conducting


# ------------------------------------------------ Tet10 A-V phasor solve
def boundary_nodes_em(mesh, boundary):
    """em3d.py:85-105: None -> 'outer', 'boundary' or the union of all
    sets; a name, a list of names, or an index array."""
    if boundary is None:
        if "outer" in mesh.boundaries:
            return np.asarray(mesh.boundaries["outer"], dtype=int)
        if "boundary" in mesh.boundaries:
            return np.asarray(mesh.boundaries["boundary"], dtype=int)
        sets = [np.asarray(v, dtype=int) for v in mesh.boundaries.values()]
        return np.unique(np.concatenate(sets)) if sets else np.array([], int)
    if isinstance(boundary, str):
        return np.asarray(mesh.boundaries[boundary], dtype=int)
    if isinstance(boundary, (list, tuple)) and boundary and isinstance(boundary[0], str):
        return np.unique(np.concatenate(
            [np.asarray(mesh.boundaries[k], dtype=int) for k in boundary]))
    return np.asarray(boundary, dtype=int)


def js_load_tet10(mesh, J_s):
    """em3d_tet10.py:322-331: rhs[3p+m] += V sum_q w_q J_m(x_q) N_qp
    (complex J allowed), vectorised over elements."""
    n = mesh.n_nodes
    _, wq = quadrature()
    _, Nq, xq, vol = element_operators_all(mesh)
    pts = xq.reshape(-1, 3)
    Jq = np.array([np.asarray(J_s(x, y, z), dtype=complex).ravel() for x, y, z in pts])
    Jq = Jq.reshape(xq.shape[0], xq.shape[1], 3)
    fe = vol[:, None, None] * np.einsum("q,eqm,qp->epm", wq, Jq, Nq)
    rhs = np.zeros(3 * n, dtype=complex)
    np.add.at(rhs, (3 * mesh.elements[:, :, None] + np.arange(3)).ravel(), fe.ravel())
    return rhs


def solve_eddy_current_tet10(mesh, nu=1.0 / (4e-7 * np.pi), sigma=0.0, omega=0.0,
                             B_applied=None, J_s=None, boundary=None, a_bc=None,
                             gauge_eps=1e-6):
    """em3d_tet10.py:267-375 (SuperLU on the eliminated A-V system)."""
    if omega <= 0:
        raise ValueError("omega must be positive")
    if B_applied is None and J_s is None:
        raise ValueError("no excitation")
    K, M, Gs, S, v_nodes, sig_e, conducting = assemble_tet10_av(
        mesh, nu=nu, sigma=sigma, gauge_eps=gauge_eps)
    if not conducting.any():
        raise ValueError("no conducting elements (sigma > 0) in mesh")
    n = mesh.n_nodes
    n_v = len(v_nodes)
    A_sys = sp.bmat([[K + 1j * omega * M, Gs], [1j * omega * Gs.T, S]], format="csr")
    rhs = np.zeros(3 * n + n_v, dtype=complex)
    if J_s is not None:
        rhs[:3 * n] += js_load_tet10(mesh, J_s)
    fixed = {}
    for p in boundary_nodes_em(mesh, boundary):
        x = mesh.nodes[int(p)]
        val = 0.5 * np.cross(np.asarray(B_applied, dtype=float), x) \
            if B_applied is not None else np.zeros(3)
        for m in range(3):
            fixed[3 * int(p) + m] = complex(val[m])
    for name, vals in (a_bc or {}).items():
        fn = vals if callable(vals) else (lambda x, y, z, v=vals: np.asarray(v, dtype=complex))
        for p in np.asarray(mesh.boundaries[name], dtype=int):
            vv = np.asarray(fn(*mesh.nodes[int(p)]), dtype=complex).ravel()
            for m in range(3):
                fixed[3 * int(p) + m] = vv[m]
    idx = np.array(sorted(fixed), dtype=int)
    val = np.array([fixed[i] for i in idx], dtype=complex)
    keep = np.ones(A_sys.shape[0], dtype=bool)
    if len(idx):
        rhs = rhs - A_sys[:, idx] @ val
        keep[idx] = False
    A2 = A_sys[keep][:, keep]
    sol = spla.spsolve(A2.tocsc(), rhs[keep])
    full = np.zeros(3 * n + n_v, dtype=complex)
    full[keep] = np.asarray(sol).ravel()
    if len(idx):
        full[idx] = val
    v = np.zeros(n, dtype=complex)
    v[v_nodes] = full[3 * n:]
    return full[:3 * n], v


# ------------------------------------------ Tet10 A-V transient (theta)
THETA_EM = {"be": 1.0, "implicit_euler": 1.0, "cn": 0.5, "crank_nicolson": 0.5}


def _l_nodes():
    """Barycentric coordinates of the 10 Tet10 nodes (corners, then edge
    midpoints in EDGES order)."""
    L = np.zeros((10, 4))
    L[np.arange(4), np.arange(4)] = 1.0
    for k, (i, j) in enumerate(EDGES):
        L[4 + k, i] = L[4 + k, j] = 0.5
    return L


def nodal_gradients_all(mesh):
    """em3d_tet10.py:122-137 for every element: grad N_j at node p,
    (M, 10, 10, 3)."""
    p = mesh.nodes[mesh.elements[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    _, dN_dL = shape_functions(_l_nodes())
    dN_dxi = np.stack([dN_dL[..., 1] - dN_dL[..., 0], dN_dL[..., 2] - dN_dL[..., 0],
                       dN_dL[..., 3] - dN_dL[..., 0]], axis=-1)          # (10, 10, 3)
    return np.einsum("pjk,ekl->epjl", dN_dxi, np.linalg.inv(J))


def transient_joule_power_tet10(mesh, a_prev, a_new, v, sigma, h, grads=None):
    """em3d_tet10.py:665-692: sigma V sum_pq MASS_REF E_p.E_q over the
    conducting elements, E = -(a_new - a_prev)/h - grad V at the nodes."""
    a_prev = np.asarray(a_prev, dtype=float).reshape(-1, 3)
    a_new = np.asarray(a_new, dtype=float).reshape(-1, 3)
    v = np.asarray(v, dtype=float)
    cen = mesh.nodes[mesh.elements[:, :4]].mean(axis=1)
    sig_e = np.asarray(eval_points(sigma, cen), dtype=float) * np.ones(len(mesh.elements))
    p = mesh.nodes[mesh.elements[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    vols = np.abs(np.linalg.det(J)) / 6.0
    on = sig_e > 0.0
    els = mesh.elements[on]
    g = (nodal_gradients_all(mesh) if grads is None else grads)[on]
    Ep = -(a_new[els] - a_prev[els]) / h - np.einsum("epjx,ej->epx", g, v[els])
    re = np.einsum("epm,eqm->epq", Ep, Ep)
    Pe = sig_e[on] * vols[on] * np.einsum("pq,epq->e", mass_reference(), re)
    Q = np.zeros(len(mesh.elements))
    Q[on] = Pe / vols[on]
    return float(np.sum(Q * vols)), Q


def transient_eddy_current_tet10(mesh, nu=1.0 / (4e-7 * np.pi), sigma=0.0, t_end=1.0,
                                 dt=0.1, method="cn", J_s=None, time_scale=None,
                                 B_applied=None, boundary=None, a_bc=None,
                                 gauge_eps=1e-6):
    """em3d_tet10.py:479-662 (monolithic theta step, one LU), without the
    history option; returns {times, P, a_end, v_end}."""
    theta = THETA_EM[method]
    K, M, Gs, S, v_nodes, sig_e, conducting = assemble_tet10_av(
        mesh, nu=nu, sigma=sigma, gauge_eps=gauge_eps)
    n = mesh.n_nodes
    n_v = len(v_nodes)
    nx = 3 * n + n_v
    E = sp.bmat([[M, sp.csr_matrix((3 * n, n_v))], [Gs.T, sp.csr_matrix((n_v, n_v))]], format="csr")
    Km = sp.bmat([[K, Gs], [sp.csr_matrix((n_v, 3 * n)), S]], format="csr")
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    h = t_end / n_steps
    A_lhs = (E / h + theta * Km).tocsr()
    A_rhs = (E / h - (1.0 - theta) * Km).tocsr()
    fixed = {}
    Bv = np.asarray(B_applied, dtype=float) if B_applied is not None else None
    for p in boundary_nodes_em(mesh, boundary):
        x = mesh.nodes[int(p)]
        val = 0.5 * np.cross(Bv, x) if Bv is not None else np.zeros(3)
        for m in range(3):
            fixed[3 * int(p) + m] = float(val[m])
    for name, vals in (a_bc or {}).items():
        fn = vals if callable(vals) else (lambda x, y, z, v=vals: np.asarray(v, dtype=float))
        for p in np.asarray(mesh.boundaries[name], dtype=int):
            vv = np.asarray(fn(*mesh.nodes[int(p)]), dtype=float).ravel()
            for m in range(3):
                fixed[3 * int(p) + m] = vv[m]
    idx = np.array(sorted(fixed), dtype=int)
    val = np.array([fixed[i] for i in idx], dtype=float)
    keep = np.ones(nx, dtype=bool)
    keep[idx] = False
    solve = spla.factorized(A_lhs[keep][:, keep].tocsc())
    A_kf = A_lhs[keep][:, idx] if len(idx) else None
    solve_S = spla.factorized(S.tocsc())
    f_static = np.real(js_load_tet10(mesh, J_s)) if J_s is not None else None
    ts = (lambda t: 1.0) if time_scale is None else time_scale
    times = np.linspace(0.0, t_end, n_steps + 1)
    P = np.zeros(n_steps + 1)
    grads = nodal_gradients_all(mesh)
    x = np.zeros(nx)
    x[idx] = val
    a_prev = x[:3 * n].copy()
    v_end = np.zeros(n)
    for k in range(1, n_steps + 1):
        f = np.zeros(nx)
        if f_static is not None:
            f[:3 * n] = (theta * ts(times[k]) + (1.0 - theta) * ts(times[k - 1])) * f_static
        b = (A_rhs @ x + f)[keep]
        if A_kf is not None:
            b = b - A_kf @ val
        xk = np.zeros(nx)
        xk[keep] = solve(b)
        xk[idx] = val
        x = xk
        a_new = x[:3 * n]
        adot = (a_new - a_prev) / h
        v_new = np.zeros(n)
        v_new[v_nodes] = -solve_S(Gs.T @ adot)
        P[k] = transient_joule_power_tet10(mesh, a_prev, a_new, v_new, sigma, h, grads)[0]
        a_prev = a_new.copy()
        v_end = v_new
    return {"times": times, "P": P, "a_end": x[:3 * n].copy(), "v_end": v_end}
