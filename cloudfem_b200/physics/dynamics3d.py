"""Transient structural dynamics (Newmark-beta) with the solves on the GPU.

Drop-in for cloudfem/physics/dynamics3d.py:

* ``newmark_integrate`` (:121-197): M u'' + C u' + K u = F(t) for given
  matrices (sparse or dense). The effective stiffness
  K + gamma/(beta h) C + 1/(beta h^2) M is formed once and solved every step
  by a device FP64 PCG solve plan (the reference factorises it once with
  SuperLU); the M and C products of the effective load are device SpMVs.
* ``transient_3d`` (:224-289): the same march on a P1 solid with K, M and
  the Rayleigh damping C = alpha M + beta_r K assembled on the device as
  3x3 blocks of the node pattern; constrained DOFs are held at zero through
  the solver's fixed-DOF mask instead of a reduced system.
* ``modal_superposition_3d`` (:292-341): the modes of ``modal3d`` (device
  shift-invert solves), then the diagonal modal oscillators stepped with
  the same Newmark recurrences, vectorised over modes on the host.
* ``node_series``, ``peak_response``: the reference's history helpers.

Each step's history (U, V, A) is copied to the host, as the reference
returns full histories.
"""

import numpy as np
import scipy.sparse as sp

from .. import _native as N
from .._driver import accept, solver_mode
from ..device import BlockSystem, DeviceMesh, PcgPlan, csr_to_device, fixed_mask, ptr
from .elastic3d import _assemble
from .modal3d import _diag_positions, _fixed_dofs, _mass_values, assemble_mass_3d, solve_modes_3d  # noqa: F401

__all__ = ["NEWMARK_METHODS", "newmark_integrate", "transient_3d",
           "modal_superposition_3d", "node_series", "peak_response"]

#: Named Newmark parameter sets: name -> (beta, gamma) (dynamics3d.py:82-85).
NEWMARK_METHODS = {"average": (0.25, 0.5), "linear": (1.0 / 6.0, 0.5)}


def _newmark_params(method, beta, gamma):
    if beta is None or gamma is None:
        if method not in NEWMARK_METHODS:
            raise ValueError(f"unknown method {method!r}; use one of "
                             f"{sorted(NEWMARK_METHODS)} or pass beta/gamma explicitly")
        b0, g0 = NEWMARK_METHODS[method]
        beta = b0 if beta is None else beta
        gamma = g0 if gamma is None else gamma
    if beta <= 0.0:
        raise ValueError("Newmark beta must be positive")
    return float(beta), float(gamma)


def _as_force_fn(load, n):
    if load is None:
        return lambda t: np.zeros(n)
    if callable(load):
        def fn(t, _load=load):
            F = np.asarray(_load(t), dtype=float).ravel()
            if F.shape != (n,):
                raise ValueError(f"load callable returned shape {F.shape}, expected ({n},)")
            return F
        return fn
    F = np.asarray(load, dtype=float).ravel()
    if F.shape != (n,):
        raise ValueError(f"constant load has shape {F.shape}, expected ({n},)")
    return lambda t: F


def _coefficients(beta, gamma, h):
    a1 = 1.0 / (beta * h * h)
    a2 = 1.0 / (beta * h)
    a3 = 1.0 / (2.0 * beta) - 1.0
    a4 = gamma / (beta * h)
    a5 = gamma / beta - 1.0
    a6 = h * (gamma / (2.0 * beta) - 1.0)
    return a1, a2, a3, a4, a5, a6


class _Operator:
    """A (block) CSR matrix on the device with y = A x products."""

    def __init__(self, rt, n_rows, bs, row_ptr, col, vals):
        self.rt, self.n_rows, self.bs = rt, n_rows, bs
        self.row_ptr, self.col, self.vals = row_ptr, col, vals

    def mul(self, x, y):
        if self.vals.numel() == 0:                  # an all-zero matrix (no damping)
            return y.zero_()
        rt = self.rt

        def p(v):
            return v if isinstance(v, N._vp) else ptr(v)
        N.check(rt.lib.cfem_spmv(rt.ctx, self.n_rows, self.bs, p(self.row_ptr),
                                 p(self.col), ptr(self.vals), 1.0, ptr(x), 0.0, ptr(y),
                                 rt.stream()))
        return y


def _march(rt, n, Mop, Cop, Kop, Khat_sys, M_sys, F, t_end, n_steps, u, v, beta, gamma,
           mask):
    """The Newmark recurrences of dynamics3d.py:170-196 on device vectors
    (products and solves by the library; the O(n) vector updates as
    elementwise device operations); Khat_sys / M_sys are BlockSystems whose
    b and x are the work vectors, mask the fixed DOFs (held at zero)."""
    import torch
    h = t_end / n_steps
    a1, a2, a3, a4, a5, a6 = _coefficients(beta, gamma, h)
    dev = rt.device
    mode, rtol = solver_mode("fp64", None)

    def dvec(a):
        t = torch.from_numpy(np.array(a, dtype=float)).to(dev)
        if mask is not None:
            t[mask.bool()] = 0.0
        return t

    u = dvec(u)
    v = dvec(v)
    w1 = torch.empty(n, dtype=torch.float64, device=dev)
    w2 = torch.empty(n, dtype=torch.float64, device=dev)
    # initial acceleration from M a0 = F(0) - C v0 - K u0
    rhs = dvec(F(0.0)) - Cop.mul(v, w1) - Kop.mul(u, w2)
    M_sys.b.copy_(rhs)
    M_sys.x.zero_()
    plan_M = PcgPlan([M_sys], mode, rtol)
    try:
        accept(plan_M.solve()[0], rtol, "initial acceleration")
    finally:
        plan_M.close()
    a = M_sys.x.clone()
    times = [0.0]
    U, V, A = [u.cpu().numpy()], [v.cpu().numpy()], [a.cpu().numpy()]
    plan = PcgPlan([Khat_sys], mode, rtol)
    t = 0.0
    try:
        for _ in range(n_steps):
            t_next = t + h
            Feff = (dvec(F(t_next)) + Mop.mul(a1 * u + a2 * v + a3 * a, w1)
                    + Cop.mul(a4 * u + a5 * v + a6 * a, w2))
            Khat_sys.b.copy_(Feff)
            Khat_sys.x.copy_(u)                        # previous step as the guess
            accept(plan.solve()[0], rtol, f"Newmark step {len(times)}")
            u_next = Khat_sys.x.clone()
            a_next = a1 * (u_next - u) - a2 * v - a3 * a
            v = v + h * ((1.0 - gamma) * a + gamma * a_next)
            u, a = u_next, a_next
            t = t_next
            times.append(t)
            U.append(u.cpu().numpy())
            V.append(v.cpu().numpy())
            A.append(a.cpu().numpy())
    finally:
        plan.close()
    times[-1] = t_end
    return np.array(times), np.array(U), np.array(V), np.array(A)


def _csr(A):
    A = sp.csr_matrix(A, dtype=float)
    A.sum_duplicates()
    A.sort_indices()
    return A


def newmark_integrate(M, C, K, load, t_end, dt, u0=None, v0=None, method="average",
                      beta=None, gamma=None):
    """Integrate M u'' + C u' + K u = F(t) with Newmark-beta
    (dynamics3d.py:121-197); returns (times, U, V, A). M, C (or None), K:
    sparse matrices or dense arrays; load: None, an (n,) array or F(t)."""
    import torch
    beta, gamma = _newmark_params(method, beta, gamma)
    M = _csr(M)
    K = _csr(K)
    n = M.shape[0]
    C = _csr((n, n)) if C is None else _csr(C)
    F = _as_force_fn(load, n)
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    h = t_end / n_steps
    a1, _, _, a4, _, _ = _coefficients(beta, gamma, h)
    Khat = _csr(K + a4 * C + a1 * M)
    rt = N.runtime()
    dev = rt.device

    def op(A):
        ip, ix, vv, _ = csr_to_device(rt, A)
        return _Operator(rt, n, 1, ip, ix, vv)

    Mop, Cop, Kop, Hop = op(M), op(C), op(K), op(Khat)

    def system(o):
        b = torch.zeros(n, dtype=torch.float64, device=dev)
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        return BlockSystem(rt, n, 1, o.row_ptr, o.col, o.vals, b, x,
                           keep=(o.row_ptr, o.col, o.vals))

    u = np.zeros(n) if u0 is None else np.broadcast_to(np.asarray(u0, dtype=float), (n,))
    v = np.zeros(n) if v0 is None else np.broadcast_to(np.asarray(v0, dtype=float), (n,))
    return _march(rt, n, Mop, Cop, Kop, system(Hop), system(Mop), F, t_end, n_steps,
                  u, v, beta, gamma, None)


def _check_homogeneous_bc(mesh, bc):
    """Only zero prescribed displacements (dynamics3d.py:200-221)."""
    if not bc:
        return
    for name, vals in bc.items():
        for v in vals:
            if v is None:
                continue
            if callable(v):
                ids = np.arange(mesh.n_nodes) if name == "all" else np.asarray(mesh.boundaries[name])
                for i in ids:
                    x, y, z = mesh.nodes[int(i)]
                    if v(x, y, z) != 0.0:
                        raise ValueError("transient_3d supports only homogeneous "
                                         "Dirichlet BCs (prescribed value 0)")
            elif float(v) != 0.0:
                raise ValueError("transient_3d supports only homogeneous "
                                 "Dirichlet BCs (prescribed value 0)")


def _block_mass(dm, m, lumped):
    """3x3 blocks m_ij I of the mass on the node pattern (device)."""
    import torch
    pat = dm.pattern
    Mb = torch.zeros(pat.nnz, 3, 3, dtype=torch.float64, device=dm.rt.device)
    if lumped:
        idx = _diag_positions(dm)
        for c in range(3):
            Mb[idx, c, c] = m
    else:
        for c in range(3):
            Mb[:, c, c] = m
    return Mb.reshape(-1)


def transient_3d(mesh, E, nu, rho, bc=None, t_end=1.0, dt=0.01, load=None, u0=None, v0=None,
                 method="average", beta=None, gamma=None, rayleigh=(0.0, 0.0), lumped=False):
    """Transient dynamics of a P1 solid by direct Newmark integration
    (dynamics3d.py:224-289); returns (times, U, V, A) on the full 3N DOFs,
    zero at the constrained ones."""
    import torch
    _check_homogeneous_bc(mesh, bc)
    beta, gamma = _newmark_params(method, beta, gamma)
    dm = DeviceMesh(mesh)
    rt = dm.rt
    pat = dm.pattern
    nnz9 = pat.nnz * 9
    K, _ = _assemble(dm, mesh, N.OP_P1_ELAST, E, nu, None, None, None, 0.0, 0.0, False)
    M = _block_mass(dm, _mass_values(dm, rho, lumped), lumped)
    alpha_r, beta_r = rayleigh
    C = torch.empty_like(K)
    N.check(rt.lib.cfem_axpby(rt.ctx, nnz9, float(alpha_r), ptr(M), float(beta_r), ptr(K),
                              ptr(C), rt.stream()))
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    h = t_end / n_steps
    a1, _, _, a4, _, _ = _coefficients(beta, gamma, h)
    KM = torch.empty_like(K)
    N.check(rt.lib.cfem_axpby(rt.ctx, nnz9, 1.0, ptr(K), a1, ptr(M), ptr(KM), rt.stream()))
    Khat = torch.empty_like(K)                 # K + a4 C + a1 M
    N.check(rt.lib.cfem_axpby(rt.ctx, nnz9, 1.0, ptr(KM), a4, ptr(C), ptr(Khat), rt.stream()))
    del KM
    n3 = 3 * mesh.n_nodes
    fixed = _fixed_dofs(mesh, bc) if bc else np.zeros(0, dtype=int)

    def op(vals):
        return _Operator(rt, dm.n_nodes, 3, pat.row_ptr, pat.col, vals)

    def system(vals):
        mask, x = fixed_mask(rt, n3, fixed, np.zeros(len(fixed)))
        b = torch.zeros(n3, dtype=torch.float64, device=rt.device)
        return BlockSystem(rt, dm.n_nodes, 3, pat.row_ptr, pat.col, vals, b, x, mask), mask

    khat_sys, mask = system(Khat)
    m_sys, _ = system(M)
    F = _as_force_fn(load, n3)
    u = np.zeros(n3) if u0 is None else np.broadcast_to(np.asarray(u0, dtype=float), (n3,))
    v = np.zeros(n3) if v0 is None else np.broadcast_to(np.asarray(v0, dtype=float), (n3,))
    return _march(rt, n3, op(M), op(C), op(K), khat_sys, m_sys, F, t_end, n_steps, u, v,
                  beta, gamma, mask)


def _newmark_diagonal(m, c, k, F, t_end, dt, q0, r0, beta, gamma):
    """The Newmark recurrences for a diagonal system (one scalar oscillator
    per entry), vectorised on the host."""
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    h = t_end / n_steps
    a1, a2, a3, a4, a5, a6 = _coefficients(beta, gamma, h)
    khat = k + a4 * c + a1 * m
    u, v = q0.astype(float).copy(), r0.astype(float).copy()
    a = (F(0.0) - c * v - k * u) / m
    times, U, V, A = [0.0], [u.copy()], [v.copy()], [a.copy()]
    t = 0.0
    for _ in range(n_steps):
        t_next = t + h
        Feff = F(t_next) + m * (a1 * u + a2 * v + a3 * a) + c * (a4 * u + a5 * v + a6 * a)
        u_next = Feff / khat
        a_next = a1 * (u_next - u) - a2 * v - a3 * a
        v = v + h * ((1.0 - gamma) * a + gamma * a_next)
        u, a = u_next, a_next
        t = t_next
        times.append(t)
        U.append(u.copy())
        V.append(v.copy())
        A.append(a.copy())
    times[-1] = t_end
    return np.array(times), np.array(U), np.array(V), np.array(A)


def modal_superposition_3d(mesh, E, nu, rho, bc=None, t_end=1.0, dt=0.01, load=None,
                           u0=None, v0=None, n_modes=12, method="average", beta=None,
                           gamma=None, rayleigh=(0.0, 0.0), lumped=False):
    """Transient dynamics by modal superposition (dynamics3d.py:292-341):
    the lowest n_modes modes (device shift-invert solves), each modal
    coordinate a Newmark-stepped scalar oscillator with Rayleigh damping."""
    _check_homogeneous_bc(mesh, bc)
    beta, gamma = _newmark_params(method, beta, gamma)
    freqs, modes = solve_modes_3d(mesh, E, nu, rho, bc=bc, n_modes=n_modes, lumped=lumped)
    M = assemble_mass_3d(mesh, rho, lumped=lumped)
    n3 = 3 * mesh.n_nodes
    omega2 = (2.0 * np.pi * freqs) ** 2
    alpha_r, beta_r = rayleigh
    F_full = _as_force_fn(load, n3)
    q0 = (modes.T @ (M @ np.broadcast_to(np.asarray(u0, dtype=float), (n3,)))
          if u0 is not None else np.zeros(n_modes))
    r0 = (modes.T @ (M @ np.broadcast_to(np.asarray(v0, dtype=float), (n3,)))
          if v0 is not None else np.zeros(n_modes))
    times, Q, Qd, Qdd = _newmark_diagonal(np.ones(n_modes), alpha_r + beta_r * omega2, omega2,
                                          lambda t: modes.T @ F_full(t), t_end, dt, q0, r0,
                                          beta, gamma)
    return times, Q @ modes.T, Qd @ modes.T, Qdd @ modes.T


def node_series(history, node, comp):
    """(S + 1,) series of component comp of node from a (S + 1, 3N) history."""
    return history[:, 3 * int(node) + int(comp)]


def peak_response(times, U):
    """(peak per DOF, time of the overall peak, DOF attaining it)."""
    peak = np.abs(U).max(axis=0)
    s, dof = np.unravel_index(np.argmax(np.abs(U)), U.shape)
    return peak, float(times[s]), int(dof)
