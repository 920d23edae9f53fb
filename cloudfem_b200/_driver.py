"""Device-side drivers shared by the drop-in modules: steady solves of
scalar (bs = 1) and nodal-block (bs = 3) systems, and the theta-method
march used by the transient heat solvers.

Solver options accepted by every ``solve_*`` / ``transient_*`` entry point
as keyword-only extras (the reference signatures are unchanged):

precision : "fp64" (default, plain FP64 Jacobi-PCG) or "mixed" (FP32 PCG
    with FP64 true residual, solution update and convergence test).
rtol : relative residual target ||b - A x|| <= rtol ||b_lift|| on the free
    DOFs (default 1e-15 for fp64, 1e-10 for mixed). The FP64 solve also
    stops at the round-off floor of its residual (about 2 eps |A||x|, the
    accuracy of a direct solver's answer), so the fp64 default means "as
    accurate as the reference's SuperLU solve".
max_iter : iteration cap (default grows with the system size).
"""

import threading

import numpy as np

from . import _native as N
from .device import BlockSystem, PcgPlan, fixed_mask, pcg, raise_for

PRECISION = {"fp64": N.SOLVE_FP64, "mixed": N.SOLVE_MIXED}
DEFAULT_RTOL = {"fp64": 1e-15, "mixed": 1e-10}

_tls = threading.local()


def last_solve_info():
    """SolveResult records of this thread's most recent device solve."""
    return list(getattr(_tls, "last", []))


def _record(results):
    _tls.last = results


def solver_mode(precision, rtol):
    if precision not in PRECISION:
        raise ValueError(f"unknown precision {precision!r}; use 'fp64' or "
                         "'mixed'")
    return PRECISION[precision], (DEFAULT_RTOL[precision] if rtol is None
                                  else float(rtol))


def accept(res, rtol, what):
    """Raise RuntimeError unless the solve converged.

    The reference raises RuntimeError when its solve fails
    (cloudfem/physics/em3d_tet10.py:360-367). A solve that stopped short of
    its target - iteration cap, or no progress over several true-residual
    replacements - is reported the same way, with the residual it reached
    (rtol is named in the message); it is never returned as a result.
    """
    if res.status == N.CFEM_OK:
        return
    raise_for(res, f"{what} (target relative residual {rtol:.1e})")


def solve_block(dm, bs, vals, rhs, fixed_idx, fixed_val, precision="fp64",
                rtol=None, max_iter=None, x0=None, what="solve"):
    """Solve the assembled system on dm's node pattern; returns device x."""
    mode, rtol = solver_mode(precision, rtol)
    pat = dm.pattern
    n = dm.n_nodes * bs
    mask, x = fixed_mask(dm.rt, n, fixed_idx, fixed_val, x0)
    sysm = BlockSystem(dm.rt, dm.n_nodes, bs, pat.row_ptr, pat.col, vals, rhs,
                       x, mask)
    res = pcg([sysm], mode, rtol, max_iter)
    _record(res)
    accept(res[0], rtol, what)
    return x


def solve_csr(rt, indptr, indices, data, rhs, fixed_idx, fixed_val, n,
              precision="fp64", rtol=None, max_iter=None, what="solve"):
    """Solve a general scalar CSR system (device arrays)."""
    mode, rtol = solver_mode(precision, rtol)
    mask, x = fixed_mask(rt, n, fixed_idx, fixed_val)
    sysm = BlockSystem(rt, n, 1, indptr, indices, data, rhs, x, mask)
    res = pcg([sysm], mode, rtol, max_iter)
    _record(res)
    accept(res[0], rtol, what)
    return x


THETA = {"be": 1.0, "implicit_euler": 1.0, "cn": 0.5, "crank_nicolson": 0.5}


def n_steps_of(t_end, dt):
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    return n_steps


def theta_march(dm, K, C, F, fixed_idx, fixed_val, t_end, n_steps, T0, theta,
                precision="fp64", rtol=None, max_iter=None, load_fn=None,
                keep_history=True):
    """(C + theta h K) T+ = (C - (1-theta) h K) T + h F, one device solve
    per step with the previous field as the initial guess
    (tet_heat.py:239-274, tet10.py:509-548). With keep_history=False the
    fields stay on the device and (times, final device field) is returned."""
    import torch
    rt = dm.rt
    lib, ctx = rt.lib, rt.ctx
    mode, rtol = solver_mode(precision, rtol)
    n = dm.n_nodes
    h = t_end / n_steps
    pat = dm.pattern
    nnz = pat.nnz
    A = torch.empty_like(K)
    R = torch.empty_like(K)
    N.check(lib.cfem_axpby(ctx, nnz, 1.0, N.ptr(C), theta * h, N.ptr(K),
                           N.ptr(A), rt.stream()))
    N.check(lib.cfem_axpby(ctx, nnz, 1.0, N.ptr(C), -(1.0 - theta) * h,
                           N.ptr(K), N.ptr(R), rt.stream()))
    T0h = (np.full(n, T0, dtype=float) if np.isscalar(T0)
           else np.asarray(T0, dtype=float).copy())
    if T0h.shape != (n,):
        raise ValueError(f"T0 must be a scalar or ({n},) array")
    T = torch.from_numpy(T0h).to(rt.device)
    mask, T = fixed_mask(rt, n, fixed_idx, fixed_val, T)
    b = torch.empty(n, dtype=torch.float64, device=rt.device)
    sysA = BlockSystem(rt, n, 1, pat.row_ptr, pat.col, A, b, T, mask)
    # one solve plan for the whole march (the reference factorises A_sys
    # once, tet_heat.py:254): every step reuses its working copies and graphs
    plan = PcgPlan([sysA], mode, rtol, max_iter)
    hist = np.empty((n_steps + 1, n)) if keep_history else None
    if keep_history:
        hist[0] = T.cpu().numpy()
    infos = []
    try:
        for step in range(n_steps):
            Fs = F if load_fn is None else load_fn(step, h)
            N.check(lib.cfem_spmv(ctx, n, 1, pat.row_ptr, pat.col, N.ptr(R), 1.0,
                                  N.ptr(T), 0.0, N.ptr(b), rt.stream()))
            N.check(lib.cfem_axpby(ctx, n, 1.0, N.ptr(b), h, N.ptr(Fs), N.ptr(b),
                                   rt.stream()))
            res = plan.solve()
            accept(res[0], rtol, f"time step {step + 1}")
            infos.append(res[0])
            if keep_history:
                hist[step + 1] = T.cpu().numpy()
    finally:
        plan.close()
    _record(infos)
    times = np.cumsum(np.concatenate([[0.0], np.full(n_steps, h)]))
    times[-1] = t_end
    return times, (hist if keep_history else T)
