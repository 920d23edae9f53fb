"""Tet10 nodal A-V eddy-current blocks on the GPU.

Drop-in for the assembly of cloudfem/physics/em3d_tet10.py:

* ``assemble_tet10_av`` (:172-264): real blocks K (curl-curl, nu), M (sigma
  vector mass with the gauge conductivity in air), G (A-V coupling) and
  S (sigma scalar stiffness on the conductor V nodes), plus v_nodes, the
  per-element conductivity and the conducting mask;
* ``_assemble_curl_curl_tet10_nu`` (:746-771): K alone for per-element nu
  (rebuilt at every Picard step of the nonlinear solver, :938);
* ``solve_eddy_current_tet10`` (:267-375): the phasor solve, by COCG on the
  device in place of SuperLU (see its docstring);
* ``transient_eddy_current_tet10`` (:479-662): theta stepping with a
  symmetric positive definite scaling of the step matrix and one device
  PCG solve (one graph launch) per step, the step's V by a second device
  PCG solve and its Joule power by a device kernel, so the fields stay on
  the GPU for the whole march; ``transient_joule_power_tet10`` (:665-692)
  by the same kernel.
* ``solve_eddy_current_nonlinear_tet10`` (:849-982): the secant B-H Picard
  loop, K rebuilt on the device from the updated per-element reluctivity
  each iteration and each linear phasor solve by device COCG warm-started
  from the previous iterate; ``bh_secant_mu_r`` (:716-743) is the model
  curve.
* Post-processing the reference's other modules import
  (``induction3d_tet10.py:101-104``, ``inductance.py:22-24``):
  ``element_flux_density_tet10`` (:378-390), ``total_joule_power_tet10``
  (:393-419), ``source_complex_power_tet10`` (:422-451) and
  ``magnetic_energy_tet10`` (:695-713), vectorised over elements on the host
  (``magnetic_energy_tet10`` assembles K on the device when not given).

Element matrices are computed by warp-per-element kernels (Keast-5
gradients staged in shared memory) and summed into the node pattern by the
deterministic segmented reduction: K is a 3x3-block curl-curl operator on
the mesh pattern, M and S reuse the scalar Tet10 mass and stiffness kernels
with per-element coefficients, G the N_p dN_j/dx_m coupling kernels (one per
component m), S and G on the pattern of the conducting elements. The
conductor components (one pinned node each, :140-169) are found with a
connected-components pass on the host. Returned matrices are SciPy CSR with
the reference's sorted, canonical structure.
"""

import ctypes
import types

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from .. import _native as N
from .._faces import add_at
from ..device import DeviceMesh, centroids, evaluate, ptr

MU0 = 4e-7 * np.pi

__all__ = ["assemble_tet10_av", "solve_eddy_current_tet10",
           "element_flux_density_tet10", "total_joule_power_tet10",
           "source_complex_power_tet10", "magnetic_energy_tet10",
           "bh_secant_mu_r", "solve_eddy_current_nonlinear_tet10",
           "transient_eddy_current_tet10", "transient_joule_power_tet10", "MU0"]


def _element_values(mesh, q):
    """Float or callable(x, y, z) at element centroids, or a per-element
    array as it is, (M,) float."""
    els = np.asarray(mesh.elements)
    if isinstance(q, np.ndarray) and q.shape == (len(els),):
        return np.asarray(q, dtype=float).copy()
    v = evaluate(q, centroids(np.asarray(mesh.nodes, dtype=float), els))
    return np.full(len(els), float(v)) if np.isscalar(v) else np.asarray(v, dtype=float)


def _conductor_components(mesh, conducting):
    """V-node ids: the nodes of conducting elements minus the smallest node
    of each connected conductor part (em3d_tet10.py:140-169)."""
    els = np.asarray(mesh.elements)[conducting]
    if els.size == 0:
        return np.zeros(0, dtype=int)
    cond_nodes = np.unique(els)
    local = np.searchsorted(cond_nodes, els)
    npe = els.shape[1]
    rows = np.repeat(local[:, :1], npe - 1, axis=1).ravel()
    cols = local[:, 1:].ravel()
    g = sp.coo_matrix((np.ones(len(rows)), (rows, cols)),
                      shape=(len(cond_nodes), len(cond_nodes)))
    _, label = connected_components(g, directed=False)
    pinned = np.zeros(len(cond_nodes), dtype=bool)
    first = np.full(label.max() + 1, len(cond_nodes))
    np.minimum.at(first, label, np.arange(len(cond_nodes)))
    pinned[first] = True                   # smallest node id of each part
    return cond_nodes[~pinned].astype(int)


def _coef(dm, values):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(values, dtype=float)).to(dm.rt.device)
    return N.Coef(ptr(t), 0.0, N.COEF_ELEM, 0), t


def _sub_mesh(mesh, sel):
    return types.SimpleNamespace(nodes=mesh.nodes,
                                 elements=np.asarray(mesh.elements)[sel],
                                 boundaries={}, n_nodes=mesh.n_nodes)


def _scalar_csr(dm, op, values):
    """Node-level CSR (indptr, indices, data) of one scalar operator with a
    per-element coefficient on dm's pattern (host arrays)."""
    import torch
    pat = dm.pattern
    coef, keep = _coef(dm, values)
    vals = torch.empty(max(pat.nnz, 1), dtype=torch.float64, device=dm.rt.device)
    N.check(dm.rt.lib.cfem_assemble(dm.rt.ctx, pat.handle, op, ptr(dm.nodes),
                                    ptr(dm.elems), ctypes.byref(coef), None,
                                    ptr(vals), None, 0, dm.rt.stream()))
    indptr, indices = pat.expand(1)
    del keep
    return (indptr.cpu().numpy().astype(np.int64), indices.cpu().numpy(),
            vals[: pat.nnz].cpu().numpy())


def _componentwise(indptr, indices, datas, n_rows, col_map=None):
    """CSR with row 3p+m holding row p of the node-level CSR for component m
    (data datas[m]); columns 3j+m, or col_map[j] (entries with col_map < 0
    dropped) when given."""
    lens_node = np.diff(indptr)
    row_of = np.repeat(np.arange(n_rows), lens_node)
    if col_map is None:
        keep = np.ones(len(indices), dtype=bool)
    else:
        keep = col_map[indices] >= 0
    kept_per_row = np.bincount(row_of[keep], minlength=n_rows)
    lens = np.repeat(kept_per_row, 3)
    out_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    k_rows = row_of[keep]
    k_idx = indices[keep].astype(np.int64)
    # rank of each kept entry within its node row
    start_kept = np.concatenate([[0], np.cumsum(kept_per_row)])[:-1]
    rank = np.arange(len(k_rows)) - start_kept[k_rows]
    out_idx = np.empty(lens.sum(), dtype=np.int64)
    out_dat = np.empty(lens.sum(), dtype=float)
    for m in range(3):
        pos = out_ptr[3 * k_rows + m] + rank
        out_idx[pos] = (3 * k_idx + m) if col_map is None else col_map[k_idx]
        out_dat[pos] = datas[m][keep]
    return out_ptr, out_idx, out_dat


def _csr(ptr_, idx, dat, shape):
    return sp.csr_matrix((dat, idx.astype(np.int32), ptr_.astype(np.int32)),
                         shape=shape)


def _curl_curl(dm, nu_e):
    import torch
    pat = dm.pattern
    coef, keep = _coef(dm, nu_e)
    vals = torch.empty(max(pat.nnz * 9, 1), dtype=torch.float64, device=dm.rt.device)
    N.check(dm.rt.lib.cfem_assemble_curlcurl(dm.rt.ctx, pat.handle, ptr(dm.nodes),
                                             ptr(dm.elems), coef, ptr(vals), 0,
                                             dm.rt.stream()))
    del keep
    return pat.to_scipy(3, vals[: pat.nnz * 9])


def _assemble_curl_curl_tet10_nu(mesh, nu_e):
    """K (3N, 3N) of the curl-curl operator for per-element nu."""
    nu_e = np.asarray(nu_e, dtype=float)
    if nu_e.shape != (len(mesh.elements),):
        raise ValueError("nu_e needs one value per element")
    return _curl_curl(DeviceMesh(mesh), nu_e)


def assemble_tet10_av(mesh, nu=1.0 / MU0, sigma=0.0, gauge_eps=1e-6):
    """Real blocks of the Tet10 nodal A-V system:
    (K, M, G, S, v_nodes, sig_e, conducting), as the reference returns."""
    n = mesh.n_nodes
    els = np.asarray(mesh.elements)
    if els.ndim != 2 or els.shape[1] != 10:
        raise ValueError("assemble_tet10_av needs a Tet10 mesh")
    nu_e = _element_values(mesh, nu)
    sig_e = _element_values(mesh, sigma)
    conducting = sig_e > 0.0
    sig_max = sig_e.max() if conducting.any() else 0.0
    sig_reg = gauge_eps * sig_max
    v_nodes = _conductor_components(mesh, conducting)
    n_v = len(v_nodes)
    v_col = np.full(n, -1, dtype=np.int64)
    v_col[v_nodes] = np.arange(n_v)

    dm = DeviceMesh(mesh)
    K = _curl_curl(dm, nu_e)

    seff = np.where(conducting, sig_e, sig_reg)
    msel = seff > 0.0
    if msel.any():
        dmm = dm if msel.all() else DeviceMesh(_sub_mesh(mesh, msel))
        ip, ix, dv = _scalar_csr(dmm, N.OP_T10_MASS, seff[msel])
        M = _csr(*_componentwise(ip, ix, [dv, dv, dv], n), (3 * n, 3 * n))
    else:
        M = sp.csr_matrix((3 * n, 3 * n))

    if conducting.any() and n_v:
        dmc = dm if conducting.all() else DeviceMesh(_sub_mesh(mesh, conducting))
        sc = sig_e[conducting]
        parts = [_scalar_csr(dmc, op, sc) for op in
                 (N.OP_T10_NGRAD_X, N.OP_T10_NGRAD_Y, N.OP_T10_NGRAD_Z)]
        ip, ix = parts[0][0], parts[0][1]
        Gs = _csr(*_componentwise(ip, ix, [p[2] for p in parts], n, v_col),
                  (3 * n, n_v))
        sp_, si, sd = _scalar_csr(dmc, N.OP_T10_STIFF, sc)
        Sfull = _csr(sp_, si, sd, (n, n))
        S = Sfull[v_nodes][:, v_nodes].tocsr()
        S.sort_indices()
    else:
        Gs = sp.csr_matrix((3 * n, n_v))
        S = sp.csr_matrix((n_v, n_v))
    return K, M, Gs, S, v_nodes, sig_e, conducting


def _boundary_nodes(mesh, boundary):
    """Outer-boundary node spec (em3d.py:85-105): None -> 'outer', else
    'boundary', else the union of all named sets; a name, a list of names,
    or an index array."""
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


def _js_load(mesh, dm, J_s):
    """A-block load V sum_q w_q J(x_q) N_qp per node and component
    (em3d_tet10.py:322-331), J_s complex allowed."""
    from ..fem.tet10 import quadrature, shape_functions
    Lq, wq = quadrature()
    Nq, _ = shape_functions(Lq)                       # (5, 10)
    pts = dm.sample_points("qp")                      # (M, 5, 3)
    flat = pts.reshape(-1, 3)
    Jq = np.array([np.asarray(J_s(x, y, z), dtype=complex).ravel()
                   for x, y, z in flat]).reshape(pts.shape[0], pts.shape[1], 3)
    els = np.asarray(mesh.elements)
    p = np.asarray(mesh.nodes, dtype=float)[els[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    vol = np.abs(np.linalg.det(J)) / 6.0
    fe = vol[:, None, None] * np.einsum("q,eqm,qp->epm", wq, Jq, Nq)
    rhs = np.zeros(3 * mesh.n_nodes, dtype=complex)
    add_at(rhs, (3 * els[:, :, None] + np.arange(3)).ravel(), fe.ravel())
    return rhs


def solve_eddy_current_tet10(mesh, nu=1.0 / MU0, sigma=0.0, omega=0.0,
                             B_applied=None, J_s=None, boundary=None,
                             a_bc=None, gauge_eps=1e-6, permc_spec=None, *,
                             rtol=1e-10, max_iter=None):
    """Phasor Tet10 nodal A-V eddy-current solve (em3d_tet10.py:267-375);
    returns (a (3N,) complex, v (N,) complex).

    The blocks are assembled on the device; the V rows of
    [[K + i w M, G], [i w G^T, S]] are scaled by 1/(i w), which makes the
    system complex symmetric, and after the reference's Dirichlet
    elimination it is solved by Jacobi-preconditioned COCG on the device
    (cfem_cocg_solve) to rtol relative residual. permc_spec (a SuperLU
    ordering in the reference) is accepted and has no effect. A system that
    does not converge within max_iter raises RuntimeError.
    """
    import torch
    if omega <= 0:
        raise ValueError("omega must be positive (phasor eddy-current "
                         "solve; omega = 0 magnetostatics is out of scope)")
    if B_applied is None and J_s is None:
        raise ValueError("no excitation: pass B_applied (background "
                         "field) or J_s (imposed current density)")
    K, M, Gs, S, v_nodes, sig_e, conducting = assemble_tet10_av(
        mesh, nu=nu, sigma=sigma, gauge_eps=gauge_eps)
    if not conducting.any():
        raise ValueError("no conducting elements (sigma > 0) in mesh")
    return _solve_phasor_with_K_tet10(mesh, K, M, Gs, S, v_nodes, omega, B_applied,
                                      J_s, boundary, a_bc, permc_spec, rtol=rtol,
                                      max_iter=max_iter)


def _solve_phasor_with_K_tet10(mesh, K, M, Gs, S, v_nodes, omega, B_applied, J_s,
                               boundary, a_bc, permc_spec=None, *, rtol=1e-10,
                               max_iter=None, dm=None, js_rhs=None, x0=None):
    """One linear phasor solve with a given curl-curl block K
    (em3d_tet10.py:774-846, used by the nonlinear Picard loop, :938): block
    system with the V rows scaled by 1/(i w), source load, Dirichlet
    elimination as the reference, device COCG; returns (a, v).

    Keyword-only extras for repeated solves on one mesh: dm (its
    DeviceMesh), js_rhs (the A-block source load, computed once), x0 (a
    previous (a, v) used as the initial guess)."""
    import torch
    n = mesh.n_nodes
    n_v = len(v_nodes)
    w = float(omega)
    A_sys = sp.bmat([[K + 1j * w * M, Gs], [Gs.T, S * (1.0 / (1j * w))]],
                    format="csr")
    rhs = np.zeros(3 * n + n_v, dtype=complex)
    dm = dm if dm is not None else DeviceMesh(mesh)
    if js_rhs is not None:
        rhs[:3 * n] += js_rhs
    elif J_s is not None:
        rhs[:3 * n] += _js_load(mesh, dm, J_s)
    fixed = {}
    if B_applied is not None:
        Bv = np.asarray(B_applied, dtype=float)
    for p in _boundary_nodes(mesh, boundary):
        x = mesh.nodes[int(p)]
        val = 0.5 * np.cross(Bv, x) if B_applied is not None else np.zeros(3)
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
    A2 = A_sys[keep][:, keep].tocsr()
    rhs2 = rhs[keep]
    n2 = A2.shape[0]
    dev = dm.rt.device
    d_ip = torch.from_numpy(A2.indptr.astype(np.int32)).to(dev)
    d_ix = torch.from_numpy(A2.indices.astype(np.int32)).to(dev)
    d_a = torch.from_numpy(np.ascontiguousarray(A2.data, dtype=np.complex128).view(np.float64)).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(rhs2, dtype=np.complex128).view(np.float64)).to(dev)
    if x0 is None:
        d_x = torch.zeros(2 * n2, dtype=torch.float64, device=dev)
    else:
        guess = np.concatenate([np.asarray(x0[0], dtype=complex).ravel(),
                                np.asarray(x0[1], dtype=complex)[v_nodes]])[keep]
        d_x = torch.from_numpy(np.ascontiguousarray(guess).view(np.float64)).to(dev)
    st = N.SolveStats()
    # COCG with Jacobi needed ~6,400 iterations at 37 k unknowns (box 10^3)
    mi = max_iter if max_iter is not None else max(5000, 50 * int(np.sqrt(n2)))
    N.check(dm.rt.lib.cfem_cocg_solve(dm.rt.ctx, n2, ptr(d_ip), ptr(d_ix), ptr(d_a),
                                      ptr(d_b), ptr(d_x), float(rtol), int(mi),
                                      ctypes.byref(st), dm.rt.stream()))
    if st.status != N.CFEM_OK:
        raise RuntimeError(f"Tet10 eddy-current solve failed: "
                           f"{N.STATUS_NAMES.get(st.status, st.status)} after "
                           f"{st.iterations} COCG iterations, relative residual "
                           f"{st.relres:.3e}")
    sol = d_x.cpu().numpy().view(np.complex128)
    full = np.zeros(3 * n + n_v, dtype=complex)
    full[keep] = sol
    if len(idx):
        full[idx] = val
    a = full[:3 * n]
    v = np.zeros(n, dtype=complex)
    v[v_nodes] = full[3 * n:]
    _last_info.update(iterations=int(st.iterations), relres=float(st.relres),
                      kernel_ms=float(st.kernel_ms))
    return a, v


_last_info = {}


def last_solve_info():
    """COCG iterations, relative residual and device time of the last
    solve_eddy_current_tet10."""
    return dict(_last_info)


# ------------------------------------------------------ post-processing

def _corner_geometry(mesh):
    """Connectivity (M, 10), corner Jacobians (M, 3, 3) (columns p_k - p_0,
    as element_operators builds them, tet10.py:103-126) and volumes."""
    els = np.asarray(mesh.elements, dtype=np.int64)
    p = np.asarray(mesh.nodes, dtype=float)[els[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    return els, J, np.abs(np.linalg.det(J)) / 6.0


def _keast_operators(mesh):
    """Per element at the Keast-5 points: G (M, 5, 10, 3), N (5, 10),
    xq (M, 5, 3), weights (5,), volumes (M,), connectivity."""
    from ..fem.tet10 import quadrature, shape_functions
    els, J, vol = _corner_geometry(mesh)
    Lq, wq = quadrature()
    Nq, dN = shape_functions(Lq)
    dxi = np.stack([dN[..., 1] - dN[..., 0], dN[..., 2] - dN[..., 0],
                    dN[..., 3] - dN[..., 0]], axis=-1)          # (5, 10, 3)
    G = np.einsum("qpk,ekl->eqpl", dxi, np.linalg.inv(J))
    xq = np.einsum("qc,ecx->eqx", Lq, np.asarray(mesh.nodes, dtype=float)[els[:, :4]])
    return G, Nq, xq, wq, vol, els


def element_flux_density_tet10(mesh, a):
    """B = curl A at every element centroid [T], (M, 3) complex
    (em3d_tet10.py:378-390): B = sum_p grad N_p x a_p with the gradients
    at the centroid (the first Keast point)."""
    from ..fem.tet10 import shape_functions
    a = np.asarray(a, dtype=complex).reshape(-1, 3)
    els, J, _ = _corner_geometry(mesh)
    _, dN = shape_functions(np.full(4, 0.25))
    dxi = np.stack([dN[:, 1] - dN[:, 0], dN[:, 2] - dN[:, 0],
                    dN[:, 3] - dN[:, 0]], axis=-1)              # (10, 3)
    G0 = np.einsum("pk,ekl->epl", dxi, np.linalg.inv(J))        # (M, 10, 3)
    return np.cross(G0, a[els]).sum(axis=1)


def total_joule_power_tet10(mesh, a, v, sigma, omega):
    """Time-averaged Joule power [W] of a phasor field and the per-element
    heating density [W/m^3] (em3d_tet10.py:393-419): E = -i w A - grad V is
    quadratic per element, so with nodal values E_p and the exact Tet10
    mass matrix, P_e = sigma_e V_e / 2 sum_pq M_ref[p, q] Re(E_p . E_q*).
    Returns (P_total, Q_elem); Q is 0 where sigma is 0."""
    from ..fem.tet10 import _MASS_REF
    a = np.asarray(a, dtype=complex).reshape(-1, 3)
    v = np.asarray(v, dtype=complex)
    sig_e = _element_values(mesh, sigma)
    on = sig_e > 0.0
    Q = np.zeros(len(sig_e))
    if not on.any():
        return 0.0, Q
    sub = types.SimpleNamespace(nodes=mesh.nodes, elements=np.asarray(mesh.elements)[on])
    els, _, vol = _corner_geometry(sub)
    grads = _nodal_gradients_all(sub)                           # (m, 10, 10, 3)
    Ep = -1j * float(omega) * a[els] - np.einsum("epjx,ej->epx", grads, v[els])
    re = np.real(np.einsum("epm,eqm->epq", Ep, Ep.conj()))
    P_e = 0.5 * sig_e[on] * vol * np.einsum("pq,epq->e", _MASS_REF, re)
    Q[on] = P_e / vol
    vols_all = _corner_geometry(mesh)[2]
    return float(np.sum(Q * vols_all)), Q


def source_complex_power_tet10(mesh, a, v, J_s, omega):
    """Complex power delivered by the imposed current [VA]
    (em3d_tet10.py:422-451): S = -1/2 sum_e V_e sum_q w_q J_s(x_q)* . E(x_q)
    with the discrete E = -i w A - grad V at the Keast points."""
    a = np.asarray(a, dtype=complex).reshape(-1, 3)
    v = np.asarray(v, dtype=complex)
    G, Nq, xq, wq, vol, els = _keast_operators(mesh)
    flat = xq.reshape(-1, 3)
    Jq = np.array([np.asarray(J_s(x, y, z), dtype=complex).ravel()
                   for x, y, z in flat]).reshape(xq.shape[0], xq.shape[1], 3)
    Eq = (-1j * float(omega) * np.einsum("qp,epm->eqm", Nq, a[els])
          - np.einsum("eqjm,ej->eqm", G, v[els]))
    S = np.sum(vol * np.einsum("q,eqm,eqm->e", wq, Jq.conj(), Eq))
    return -0.5 * complex(S)


def magnetic_energy_tet10(mesh, a, nu=1.0 / MU0, K=None):
    """Time-averaged stored magnetic energy [J] of a phasor A field,
    W = Re(a^H K a) / 4 with the assembled curl-curl matrix
    (em3d_tet10.py:695-713); K is assembled on the device when not given."""
    a = np.asarray(a, dtype=complex).reshape(-1, 3).ravel()
    if K is None:
        K = assemble_tet10_av(mesh, nu=nu)[0]
    return 0.25 * float(np.real(np.vdot(a, K @ a)))


def bh_secant_mu_r(Hmag, bsat=1.9, mu_mag0=200.0):
    """Secant relative permeability of the analytic magnetisation curve
    M(H) = Ms tanh(H / H_ref), Ms = bsat / mu0, H_ref = Ms / mu_mag0
    (em3d_tet10.py:716-743): mu_r = 1 + mu_mag0 tanh(h) / h, h = |H| / H_ref,
    with the series 1 - h^2 / 3 for tanh(h) / h below h = 1e-6."""
    H = np.asarray(Hmag, dtype=float)
    if mu_mag0 == 0.0:
        return np.ones_like(H)
    Ms = float(bsat) / MU0
    h = np.abs(H) / (Ms / float(mu_mag0))
    ratio = np.where(h > 1.0e-6, np.tanh(h) / np.maximum(h, 1.0e-300), 1.0 - h * h / 3.0)
    return 1.0 + float(mu_mag0) * ratio


def _as_fn(q):
    return q if callable(q) else (lambda x, y, z, _q=q: _q)


def _picard(mesh, M, Gs, S, v_nodes, sigma, omega, B_applied, J_s, boundary,
            a_bc, permc_spec, iron_mask, nu_e, mu_target, tol, max_iter, relax,
            rtol, cocg_max_iter):
    """The secant Picard loop shared by the nonlinear phasor solvers
    (em3d_tet10.py:914-967, induction3d_tet10.py:336-371): K rebuilt on the
    device from nu_e (updated in place), a device COCG phasor solve warm-
    started from the previous iterate, centroid |B|, the exact Joule power,
    and nu of the iron elements relaxed towards 1 / (mu0 mu_target(|H|)).
    Returns (a, v, B, Q, iterations, converged, rel_dB, P, cocg iterations)."""
    dm = DeviceMesh(mesh)
    js_rhs = _js_load(mesh, dm, J_s) if J_s is not None else None
    sel = iron_mask if iron_mask.any() else slice(None)
    hist_rel, hist_P, cocg_iters = [], [], []
    B_prev = None
    converged = False
    a = v = B = Q = None
    it = 0
    for it in range(1, max_iter + 1):
        K = _curl_curl(dm, nu_e)
        a, v = _solve_phasor_with_K_tet10(
            mesh, K, M, Gs, S, v_nodes, omega, B_applied, J_s, boundary, a_bc,
            permc_spec, rtol=rtol, max_iter=cocg_max_iter, dm=dm, js_rhs=js_rhs,
            x0=None if a is None else (a, v))
        cocg_iters.append(_last_info["iterations"])
        B = element_flux_density_tet10(mesh, a)
        B_amp = np.sqrt(np.sum(np.abs(B) ** 2, axis=1))
        P, Q = total_joule_power_tet10(mesh, a, v, sigma, omega)
        hist_P.append(P)
        if B_prev is not None:
            denom = max(float(np.linalg.norm(B_amp[sel])), 1e-300)
            rel = float(np.linalg.norm(B_amp[sel] - B_prev[sel]) / denom)
            hist_rel.append(rel)
            if rel < tol:
                converged = True
                break
        if it == max_iter:
            break
        B_prev = B_amp
        if iron_mask.any():
            nu_t = 1.0 / (MU0 * mu_target(B_amp[iron_mask] * nu_e[iron_mask]))
            nu_e[iron_mask] = (1.0 - relax) * nu_e[iron_mask] + relax * nu_t
    return a, v, B, Q, it, converged, hist_rel, hist_P, cocg_iters


def solve_eddy_current_nonlinear_tet10(mesh, nu=1.0 / MU0, sigma=0.0, omega=0.0,
                                       B_applied=None, J_s=None, boundary=None,
                                       a_bc=None, gauge_eps=1e-6, permc_spec=None,
                                       iron=None, bsat=1.9, mu_mag0=200.0,
                                       mu_init=None, tol=1e-3, max_iter=50,
                                       relax=0.5, *, rtol=1e-10, cocg_max_iter=None):
    """Nonlinear (secant B-H) phasor A-V solve by Picard iteration
    (em3d_tet10.py:849-982); returns (a, v, info) as the reference does.

    The sigma blocks (M, G, S) are assembled once; every iteration rebuilds
    K on the device from the per-element reluctivity (the same mesh pattern,
    no pattern rebuild), solves the phasor system by device COCG to rtol,
    warm-started from the previous iterate, and relaxes nu of the iron
    elements towards the curve's secant value at |H| = nu |B| (centroid B).
    Convergence: relative change of |B| over the iron elements (all
    elements without iron) below tol; info carries iterations, converged,
    rel_dB, P (Joule power per solve), mu_r_elem, nu_elem, B_elem,
    iron_mask, relax and tol. permc_spec is accepted and has no effect.
    """
    if omega <= 0:
        raise ValueError("omega must be positive (phasor eddy-current "
                         "solve; omega = 0 magnetostatics is out of scope)")
    if B_applied is None and J_s is None:
        raise ValueError("no excitation: pass B_applied (background "
                         "field) or J_s (imposed current density)")
    if tol <= 0:
        raise ValueError("tol must be positive")
    if max_iter < 1:
        raise ValueError("max_iter must be >= 1")
    if not (0.0 < relax <= 1.0):
        raise ValueError("relax must be in (0, 1]")
    _, M, Gs, S, v_nodes, sig_e, conducting = assemble_tet10_av(
        mesh, nu=1.0, sigma=sigma, gauge_eps=gauge_eps)
    if not conducting.any():
        raise ValueError("no conducting elements (sigma > 0) in mesh")
    nu_e = _element_values(mesh, nu)
    if iron is None:
        iron_mask = np.zeros(len(nu_e), dtype=bool)
    else:
        fn = _as_fn(iron)
        cen = centroids(np.asarray(mesh.nodes, dtype=float), np.asarray(mesh.elements))
        iron_mask = np.array([bool(fn(x, y, z)) for x, y, z in cen], dtype=bool)
    mu_r0 = (1.0 + float(mu_mag0)) if mu_init is None else float(mu_init)
    nu_e[iron_mask] = 1.0 / (MU0 * mu_r0)

    def mu_target(H_amp):
        return bh_secant_mu_r(H_amp, bsat=bsat, mu_mag0=mu_mag0)

    a, v, B, Q, it, converged, hist_rel, hist_P, cocg_iters = _picard(
        mesh, M, Gs, S, v_nodes, sigma, omega, B_applied, J_s, boundary, a_bc,
        permc_spec, iron_mask, nu_e, mu_target, tol, max_iter, relax, rtol,
        cocg_max_iter)
    info = {"iterations": it, "converged": converged,
            "rel_dB": np.array(hist_rel), "P": np.array(hist_P),
            "mu_r_elem": 1.0 / (MU0 * nu_e), "nu_elem": nu_e.copy(),
            "B_elem": B, "iron_mask": iron_mask, "relax": relax, "tol": tol,
            "cocg_iterations": np.array(cocg_iters)}
    return a, v, info


# ------------------------------------------------------ transient (theta)
_THETA_EM = {"be": 1.0, "implicit_euler": 1.0, "cn": 0.5, "crank_nicolson": 0.5}


def _l_nodes():
    from ..mesh.tet10_mesh import EDGES
    L = np.zeros((10, 4))
    L[np.arange(4), np.arange(4)] = 1.0
    for k, (i, j) in enumerate(EDGES):
        L[4 + k, i] = L[4 + k, j] = 0.5
    return L


def _nodal_gradients_all(mesh):
    """grad N_j at node p of every element (em3d_tet10.py:122-137),
    (M, 10, 10, 3)."""
    from ..fem.tet10 import shape_functions
    els = np.asarray(mesh.elements)
    p = np.asarray(mesh.nodes, dtype=float)[els[:, :4]]
    J = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=2)
    _, dN_dL = shape_functions(_l_nodes())
    dN_dxi = np.stack([dN_dL[..., 1] - dN_dL[..., 0], dN_dL[..., 2] - dN_dL[..., 0],
                       dN_dL[..., 3] - dN_dL[..., 0]], axis=-1)
    return np.einsum("pjk,ekl->epjl", dN_dxi, np.linalg.inv(J))


class _JouleDevice:
    """Device tables of the Tet10 Joule-power kernel (cfem_t10_joule_power)
    for one mesh: the reference element's dN_j/dxi at its nodes
    (em3d_tet10.py:122-137), its normalised mass matrix and sigma per
    element."""

    def __init__(self, dm, sig_e):
        import torch
        from ..fem.tet10 import _MASS_REF, shape_functions
        _, dN_dL = shape_functions(_l_nodes())
        dn = np.stack([dN_dL[..., 1] - dN_dL[..., 0], dN_dL[..., 2] - dN_dL[..., 0],
                       dN_dL[..., 3] - dN_dL[..., 0]], axis=-1)
        dev = dm.rt.device
        self.dm = dm
        self.dn = torch.from_numpy(np.ascontiguousarray(dn, dtype=float)).to(dev)
        self.mref = torch.from_numpy(np.ascontiguousarray(_MASS_REF, dtype=float)).to(dev)
        self.sigma = torch.from_numpy(np.ascontiguousarray(sig_e, dtype=float)).to(dev)

    def power(self, a_prev, a_new, vcol, v, h, out, q=None):
        """out[0] = the power of one step (device), q: density per element."""
        rt, dm = self.dm.rt, self.dm
        N.check(rt.lib.cfem_t10_joule_power(
            rt.ctx, dm.n_elems, ptr(dm.elems), ptr(dm.nodes), ptr(self.sigma), ptr(a_prev),
            ptr(a_new), ptr(vcol), ptr(v), float(h), ptr(self.dn), ptr(self.mref), ptr(out),
            ptr(q), rt.stream()))


def transient_joule_power_tet10(mesh, a_prev, a_new, v, sigma, h):
    """Instantaneous Joule power of one transient step and the per-element
    density (em3d_tet10.py:665-692), on the device (one thread per element,
    fixed-order sum)."""
    import torch
    dm = DeviceMesh(mesh)
    dev = dm.rt.device
    n = mesh.n_nodes
    jd = _JouleDevice(dm, _element_values(mesh, sigma))

    def up(a, shape):
        return torch.from_numpy(np.ascontiguousarray(np.reshape(a, shape), dtype=float)).to(dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    q = torch.zeros(mesh.n_elements, dtype=torch.float64, device=dev)
    jd.power(up(a_prev, 3 * n), up(a_new, 3 * n), torch.arange(n, dtype=torch.int64, device=dev),
             up(v, n), h, out, q)
    return float(out.cpu()[0]), q.cpu().numpy()


def transient_eddy_current_tet10(mesh, nu=1.0 / MU0, sigma=0.0, t_end=1.0, dt=0.1,
                                 method="cn", J_s=None, time_scale=None,
                                 B_applied=None, boundary=None, a_bc=None,
                                 gauge_eps=1e-6, history=False, *,
                                 precision="fp64", rtol=None, max_iter=None):
    """Transient Tet10 A-V eddy currents, theta method
    (em3d_tet10.py:479-662); returns the reference's dict (times, P, a_end,
    v_end, and t_hist / a_hist when history is asked for).

    The monolithic step matrix E/h + theta K is made symmetric positive
    definite by scaling its V rows by theta h (the scaled form is
    int sigma |a/sqrt(h) + theta sqrt(h) grad v|^2 + theta a^T K a plus the
    air gauge mass), so every step is one device PCG solve with a solve plan
    kept for the whole march (one CUDA graph launch per step) in place of
    the reference's LU; the Dirichlet values stay in x under a fixed-DOF
    mask. The constraint-consistent V of each step (em3d_tet10.py:485, 527)
    is a second, warm-started device PCG solve on the conductors'
    sigma-Laplacian in place of the reference's LU, and the Joule power a
    device kernel (cfem_t10_joule_power): the fields stay on the GPU for the
    whole march and come back once at its end.
    """
    import torch

    from .. import _driver as D
    from ..device import BlockSystem, PcgPlan, csr_to_device, fixed_mask
    if method not in _THETA_EM:
        raise ValueError(f"unknown method {method!r}; use one of {sorted(_THETA_EM)}")
    theta = _THETA_EM[method]
    if t_end <= 0:
        raise ValueError("t_end must be positive")
    if dt <= 0:
        raise ValueError("dt must be positive")
    if J_s is None and B_applied is None:
        raise ValueError("no excitation: pass J_s and/or B_applied")
    K, M, Gs, S, v_nodes, sig_e, conducting = assemble_tet10_av(
        mesh, nu=nu, sigma=sigma, gauge_eps=gauge_eps)
    if not conducting.any():
        raise ValueError("no conducting elements (sigma > 0) in mesh")
    n = mesh.n_nodes
    n_v = len(v_nodes)
    nx = 3 * n + n_v
    E = sp.bmat([[M, sp.csr_matrix((3 * n, n_v))],
                 [Gs.T, sp.csr_matrix((n_v, n_v))]], format="csr")
    Km = sp.bmat([[K, Gs], [sp.csr_matrix((n_v, 3 * n)), S]], format="csr")
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    h = t_end / n_steps
    scale = sp.diags(np.concatenate([np.ones(3 * n), np.full(n_v, theta * h)]))
    A_l = (scale @ (E / h + theta * Km)).tocsr()
    A_r = (scale @ (E / h - (1.0 - theta) * Km)).tocsr()
    fixed = {}
    Bv = np.asarray(B_applied, dtype=float) if B_applied is not None else None
    for p in _boundary_nodes(mesh, boundary):
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

    dm = DeviceMesh(mesh)
    rt = dm.rt
    lib, ctx = rt.lib, rt.ctx
    dev = rt.device
    lp, li, lv, _ = csr_to_device(rt, A_l)
    rp, ri, rv, _ = csr_to_device(rt, A_r)
    x0 = np.zeros(nx)
    x0[idx] = val
    mask, x = fixed_mask(rt, nx, idx, val, torch.from_numpy(x0).to(dev))
    b = torch.empty(nx, dtype=torch.float64, device=dev)
    f_dev = None
    if J_s is not None:
        f_static = np.real(_js_load(mesh, dm, J_s))
        fh = np.zeros(nx)
        fh[:3 * n] = f_static
        f_dev = torch.from_numpy(fh).to(dev)
    ts = (lambda t: 1.0) if time_scale is None else time_scale
    mode, rtol = D.solver_mode(precision, rtol)
    sysA = BlockSystem(rt, nx, 1, lp, li, lv, b, x, mask, keep=(lp, li, lv))
    plan = PcgPlan([sysA], mode, rtol, max_iter)
    # the constraint-consistent V of each step, S v = -Gs^T (a_new - a_prev) / h
    # (em3d_tet10.py:485, 527): a device FP64 PCG solve (S is the conductors'
    # sigma-Laplacian with one node pinned per part: SPD), warm-started
    vmode, vrtol = D.solver_mode("fp64", None)
    vcol = np.full(n, -1, dtype=np.int64)
    vcol[v_nodes] = np.arange(n_v)
    d_vcol = torch.from_numpy(vcol).to(dev)
    v_b = torch.zeros(max(n_v, 1), dtype=torch.float64, device=dev)
    v_x = torch.zeros(max(n_v, 1), dtype=torch.float64, device=dev)
    planV = None
    if n_v:
        gp_, gi_, gv_, _ = csr_to_device(rt, Gs.T.tocsr())
        sp_, si_, sv_, _ = csr_to_device(rt, S)
        sysV = BlockSystem(rt, n_v, 1, sp_, si_, sv_, v_b, v_x, keep=(sp_, si_, sv_))
        planV = PcgPlan([sysV], vmode, vrtol)
    jd = _JouleDevice(dm, sig_e)
    a_prev_d = x[:3 * n].clone()
    adot = torch.empty(3 * n, dtype=torch.float64, device=dev)

    times = np.linspace(0.0, t_end, n_steps + 1)
    if history is True:
        rec = np.ones(n_steps + 1, dtype=bool)
    elif isinstance(history, (tuple, list)):
        t0h, t1h = history
        rec = (times >= t0h - 1e-12) & (times <= t1h + 1e-12)
        if not rec.any():
            raise ValueError(f"history window {tuple(history)} selects no "
                             f"steps in [0, {t_end}]")
    else:
        rec = np.zeros(n_steps + 1, dtype=bool)
    P_d = torch.zeros(n_steps + 1, dtype=torch.float64, device=dev)
    hist_d = (torch.empty((int(rec.sum()), 3 * n), dtype=torch.float64, device=dev)
              if rec.any() else None)
    nrec = 0
    if rec[0]:
        hist_d[0].copy_(a_prev_d)
        nrec = 1
    infos = []
    try:
        for k in range(1, n_steps + 1):
            N.check(lib.cfem_spmv(ctx, nx, 1, ptr(rp), ptr(ri), ptr(rv), 1.0,
                                  ptr(x), 0.0, ptr(b), rt.stream()))
            if f_dev is not None:
                s = theta * ts(times[k]) + (1.0 - theta) * ts(times[k - 1])
                N.check(lib.cfem_axpby(ctx, nx, 1.0, ptr(b), float(s), ptr(f_dev),
                                       ptr(b), rt.stream()))
            res = plan.solve()
            D.accept(res[0], rtol, f"time step {k}")
            infos.append(res[0])
            if planV is not None:
                N.check(lib.cfem_axpby(ctx, 3 * n, 1.0 / h, ptr(x), -1.0 / h, ptr(a_prev_d),
                                       ptr(adot), rt.stream()))
                N.check(lib.cfem_spmv(ctx, n_v, 1, ptr(gp_), ptr(gi_), ptr(gv_), -1.0,
                                      ptr(adot), 0.0, ptr(v_b), rt.stream()))
                D.accept(planV.solve()[0], vrtol, f"V of time step {k}")
            jd.power(a_prev_d, x, d_vcol, v_x, h, P_d[k:k + 1])
            a_prev_d.copy_(x[:3 * n])
            if rec[k]:
                hist_d[nrec].copy_(a_prev_d)
                nrec += 1
    finally:
        plan.close()
        if planV is not None:
            planV.close()
    D._record(infos)
    P = P_d.cpu().numpy()
    v_end = np.zeros(n)
    if n_v:
        v_end[v_nodes] = v_x.cpu().numpy()
    out = {"times": times, "P": P, "a_end": a_prev_d.cpu().numpy(), "v_end": v_end}
    if hist_d is not None:
        out["t_hist"] = times[rec]
        out["a_hist"] = hist_d.cpu().numpy()
    return out
