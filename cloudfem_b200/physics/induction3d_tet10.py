"""Staggered EM -> heat induction heating of Tet10 steel parts on the GPU.

Drop-in for cloudfem/physics/induction3d_tet10.py:

* the BIG-M4/M10 material laws (:126-221): ``curie_step_T``,
  ``steel_sigma_T``, ``bh_secant_mu_r_HT``, ``steel_cp_T``,
  ``steel_enthalpy_T`` - closed-form functions of T, restated;
* ``solve_eddy_current_nonlinear_tet10_T`` (:242-371): the secant B-H Picard
  loop at a frozen element temperature field (conductivity and the Curie
  switch from T), K rebuilt on the device every iteration and each linear
  phasor solve by device COCG warm-started from the previous iterate;
* ``induction_heating_3d_tet10`` (:407-639): per EM interval a nonlinear
  A-V solve, the element Joule density as a nodal heat load, and theta-
  method heat steps on the workpiece submesh. The heat march stays on the
  device: K and C of the submesh assembled once (C again per interval when
  the capacity follows T), one solve plan per capacity matrix (the reference
  factorises once), each step an FP64 SpMV for the right-hand side and one
  plan solve, where the reference runs a SuperLU back-substitution.

The energy account, the per-interval history and the returned dict follow
the reference field by field.
"""

import numpy as np
from scipy.special import erf

from .. import _native as N
from .._driver import THETA, solver_mode
from ..device import BlockSystem, DeviceMesh, PcgPlan, centroids, ptr
from ..mesh.tet10_mesh import Tet10Mesh
from . import em3d_tet10 as em
from .em3d_tet10 import MU0, bh_secant_mu_r

__all__ = [
    "curie_step_T", "steel_sigma_T", "bh_secant_mu_r_HT",
    "steel_cp_T", "steel_enthalpy_T",
    "solve_eddy_current_nonlinear_tet10_T",
    "induction_heating_3d_tet10",
    "TC_CURIE", "W_STEP_CURIE", "SIG_HI", "SIG_LO", "T_SIG", "W_SIG",
]

# Default constants of the BIG-M4/M10 laws (induction3d_tet10.py:114-121).
TC_CURIE = 770.0
W_STEP_CURIE = 15.0
SIG_HI = 6.0e6
SIG_LO = 1.0e6
T_SIG = 550.0
W_SIG = 150.0


def curie_step_T(T, t_curie=TC_CURIE, w_step=W_STEP_CURIE):
    """Curie switch 0.5 (1 - tanh((T - Tc) / w)): 1 well below Tc, 0 above."""
    return 0.5 * (1.0 - np.tanh((np.asarray(T, dtype=float) - float(t_curie))
                                / float(w_step)))


def steel_sigma_T(T, sig_hi=SIG_HI, sig_lo=SIG_LO, t_sig=T_SIG, w_sig=W_SIG):
    """Conductivity [S/m]: sig_lo + (sig_hi - sig_lo) * tanh switch at t_sig."""
    sw = 0.5 * (1.0 - np.tanh((np.asarray(T, dtype=float) - float(t_sig)) / float(w_sig)))
    return float(sig_lo) + (float(sig_hi) - float(sig_lo)) * sw


def bh_secant_mu_r_HT(Hmag, T, bsat=1.9, mu_mag0=200.0, t_curie=TC_CURIE,
                      w_step=W_STEP_CURIE):
    """mu_r(|H|, T) = 1 + (mu_r(|H|) - 1) * curie_step_T(T)."""
    return 1.0 + (bh_secant_mu_r(Hmag, bsat=bsat, mu_mag0=mu_mag0) - 1.0) * \
        curie_step_T(T, t_curie=t_curie, w_step=w_step)


def steel_cp_T(T, rho_cp=3.768e6, cp_slope=0.0, t_ref=20.0, cp_peak_h=0.0,
               cp_peak_w=25.0, t_curie=TC_CURIE):
    """Volumetric heat capacity: rho_cp (1 + cp_slope (T - t_ref)) plus a
    Gaussian peak of height cp_peak_h and width cp_peak_w at t_curie."""
    T = np.asarray(T, dtype=float)
    c = float(rho_cp) * (1.0 + float(cp_slope) * (T - float(t_ref)))
    if float(cp_peak_h) != 0.0 and float(cp_peak_w) > 0.0:
        z = (T - float(t_curie)) / float(cp_peak_w)
        c = c + float(cp_peak_h) * np.exp(-0.5 * z * z)
    return c


def steel_enthalpy_T(T, t_ref=20.0, rho_cp=3.768e6, cp_slope=0.0, cp_peak_h=0.0,
                     cp_peak_w=25.0, t_curie=TC_CURIE):
    """Volumetric enthalpy relative to t_ref: the integral of steel_cp_T in
    closed form (polynomial part, and erf for the Gaussian peak)."""
    T = np.asarray(T, dtype=float)
    dT = T - float(t_ref)
    H = float(rho_cp) * (dT + 0.5 * float(cp_slope) * dT * dT)
    h, w = float(cp_peak_h), float(cp_peak_w)
    if h != 0.0 and w > 0.0:
        s2 = np.sqrt(2.0)
        H = H + h * w * np.sqrt(np.pi / 2.0) * (
            erf((T - float(t_curie)) / (w * s2)) - erf((float(t_ref) - float(t_curie)) / (w * s2)))
    return H


def _iron_mask(mesh, iron):
    if iron is None:
        raise ValueError("iron predicate is required: it marks the steel "
                         "elements whose mu and sigma follow the temperature-"
                         "dependent BIG-M4/M10 laws")
    cen = centroids(np.asarray(mesh.nodes, dtype=float), np.asarray(mesh.elements))
    return np.array([bool(iron(x, y, z)) for x, y, z in cen], dtype=bool), cen


def solve_eddy_current_nonlinear_tet10_T(mesh, T_elem, omega, B_applied=None, J_s=None,
                                         boundary=None, a_bc=None, gauge_eps=1e-6,
                                         permc_spec=None, iron=None, bsat=1.9,
                                         mu_mag0=200.0, t_curie=TC_CURIE,
                                         w_step=W_STEP_CURIE, sig_hi=SIG_HI,
                                         sig_lo=SIG_LO, t_sig=T_SIG, w_sig=W_SIG,
                                         mu_init=None, nu_init=None, tol=1e-3,
                                         max_iter=50, relax=0.5, *, rtol=1e-10,
                                         cocg_max_iter=None):
    """Nonlinear B-H phasor A-V solve at a frozen element temperature field
    (induction3d_tet10.py:242-371); returns (a, v, info) with info as the
    reference's (plus cocg_iterations).

    Iron elements take sigma = steel_sigma_T(T_elem) and the secant target
    mu_r = bh_secant_mu_r_HT(|H|, T_elem); the others are air (sigma 0,
    nu 1/mu0). nu_init: per-element reluctivity to start from (a warm start
    from the previous interval). permc_spec has no effect (device COCG)."""
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
    n_el = len(mesh.elements)
    T_elem = np.asarray(T_elem, dtype=float)
    if T_elem.shape != (n_el,):
        raise ValueError(f"T_elem must have shape ({n_el},), got {T_elem.shape}")
    iron_mask, _ = _iron_mask(mesh, iron)
    if not iron_mask.any():
        raise ValueError("iron predicate selects no elements")
    sig_e = np.zeros(n_el)
    sig_e[iron_mask] = steel_sigma_T(T_elem[iron_mask], sig_hi=sig_hi, sig_lo=sig_lo,
                                     t_sig=t_sig, w_sig=w_sig)
    _, M, Gs, S, v_nodes, sig_e, conducting = em.assemble_tet10_av(
        mesh, nu=1.0, sigma=sig_e, gauge_eps=gauge_eps)
    if not conducting.any():
        raise ValueError("no conducting elements (sigma > 0) in mesh")
    if nu_init is not None:
        nu_e = np.asarray(nu_init, dtype=float).copy()
        if nu_e.shape != (n_el,):
            raise ValueError("nu_init must be a per-element array")
    else:
        nu_e = np.full(n_el, 1.0 / MU0)
        mu_r0 = (1.0 + float(mu_mag0)) if mu_init is None else float(mu_init)
        nu_e[iron_mask] = 1.0 / (MU0 * mu_r0)
    T_iron = T_elem[iron_mask]

    def mu_target(H_amp):
        return bh_secant_mu_r_HT(H_amp, T_iron, bsat=bsat, mu_mag0=mu_mag0,
                                 t_curie=t_curie, w_step=w_step)

    a, v, B, Q, it, converged, hist_rel, hist_P, cocg_iters = em._picard(
        mesh, M, Gs, S, v_nodes, sig_e, omega, B_applied, J_s, boundary, a_bc,
        permc_spec, iron_mask, nu_e, mu_target, tol, max_iter, relax, rtol,
        cocg_max_iter)
    info = {"iterations": it, "converged": converged,
            "rel_dB": np.array(hist_rel), "P": np.array(hist_P),
            "mu_r_elem": 1.0 / (MU0 * nu_e), "nu_elem": nu_e.copy(),
            "B_elem": B, "Q_elem": Q, "sigma_elem": sig_e.copy(),
            "T_elem": T_elem.copy(), "iron_mask": iron_mask,
            "relax": relax, "tol": tol, "cocg_iterations": np.array(cocg_iters)}
    return a, v, info


def _centroid_lookup(centroids, values):
    """Callable(x, y, z) -> the value of the nearest centroid
    (induction3d_tet10.py:216-230): exact at the centroids themselves,
    where the element fields are evaluated. Takes scalars or arrays."""
    from scipy.spatial import cKDTree
    tree = cKDTree(np.asarray(centroids, dtype=float))
    vals = np.asarray(values, dtype=float)

    def fn(x, y, z):
        pts = np.stack(np.broadcast_arrays(np.asarray(x, dtype=float), np.asarray(y, dtype=float),
                                           np.asarray(z, dtype=float)), axis=-1)
        _, idx = tree.query(pts)
        out = vals[idx]
        return float(out) if np.ndim(out) == 0 else out

    return fn


def _element_source_load(sub, Q_sub):
    """Nodal load of an element-constant heat source Q_sub [W/m^3]
    (induction3d_tet10.py:390-404): V Q_e sum_q w_q N_q per element, the
    f-assembly of assemble_tet10, on the device."""
    dm = DeviceMesh(sub)
    _, F = dm.assemble(N.OP_T10_STIFF, coef=0.0,
                       load=np.ascontiguousarray(np.asarray(Q_sub, dtype=float)))
    return F.cpu().numpy()


def _extract_submesh_tet10(mesh, elem_mask):
    """The masked Tet10 elements as a standalone Tet10Mesh (boundary tags
    not carried over), with the used node ids and the element ids
    (induction3d_tet10.py:374-387)."""
    elem_idx = np.where(np.asarray(elem_mask, dtype=bool))[0]
    els = np.asarray(mesh.elements)[elem_idx]
    used, inv = np.unique(els, return_inverse=True)
    n_corners = int(np.sum(used < mesh.n_corners)) if hasattr(mesh, "n_corners") else None
    sub = Tet10Mesh(np.asarray(mesh.nodes)[used], inv.reshape(-1, 10), n_corners=n_corners)
    return sub, used, elem_idx


class _HeatMarch:
    """Theta-method heat steps on the device for one capacity matrix:
    A = C + theta h K and R = C - (1 - theta) h K on the submesh pattern,
    one FP64 solve plan on A (built once, as the reference factorises once,
    induction3d_tet10.py:499-515); each step b = R T + h F_Q, then A T = b."""

    def __init__(self, dm, K, C, theta, h):
        import torch
        rt = dm.rt
        self.dm, self.h = dm, float(h)
        pat = dm.pattern
        self.A = torch.empty_like(K)
        self.R = torch.empty_like(K)
        N.check(rt.lib.cfem_axpby(rt.ctx, pat.nnz, 1.0, ptr(C), theta * h, ptr(K),
                                  ptr(self.A), rt.stream()))
        N.check(rt.lib.cfem_axpby(rt.ctx, pat.nnz, 1.0, ptr(C), -(1.0 - theta) * h,
                                  ptr(K), ptr(self.R), rt.stream()))
        n = dm.n_nodes
        self.T = torch.zeros(n, dtype=torch.float64, device=rt.device)
        self.b = torch.empty(n, dtype=torch.float64, device=rt.device)
        mode, self.rtol = solver_mode("fp64", None)
        sysA = BlockSystem(rt, n, 1, pat.row_ptr, pat.col, self.A, self.b, self.T)
        self.plan = PcgPlan([sysA], mode, self.rtol)

    def advance(self, T_start, F_Q, n_sub):
        from .._driver import accept
        rt, pat = self.dm.rt, self.dm.pattern
        n = self.dm.n_nodes
        self.T.copy_(T_start)
        for _ in range(n_sub):
            N.check(rt.lib.cfem_spmv(rt.ctx, n, 1, pat.row_ptr, pat.col, ptr(self.R), 1.0,
                                     ptr(self.T), 0.0, ptr(self.b), rt.stream()))
            N.check(rt.lib.cfem_axpby(rt.ctx, n, 1.0, ptr(self.b), self.h, ptr(F_Q),
                                      ptr(self.b), rt.stream()))
            accept(self.plan.solve()[0], self.rtol, "induction heat step")
        return self.T.clone()

    def close(self):
        self.plan.close()


def _row_sums(dm, vals):
    """C ones on the device, as a host vector (C symmetric: ones^T C)."""
    import torch
    rt, pat = dm.rt, dm.pattern
    ones = torch.ones(dm.n_nodes, dtype=torch.float64, device=rt.device)
    out = torch.empty_like(ones)
    N.check(rt.lib.cfem_spmv(rt.ctx, dm.n_nodes, 1, pat.row_ptr, pat.col, ptr(vals), 1.0,
                             ptr(ones), 0.0, ptr(out), rt.stream()))
    return out.cpu().numpy()


def induction_heating_3d_tet10(mesh, omega, B_applied=None, J_s=None, boundary=None,
                               a_bc=None, iron=None, T0=20.0, t_end=1.0, dt=0.01,
                               em_every=5, k_th=30.0, rho_cp=3.768e6, method="be",
                               stagger_iter=1, stagger_tol=None, em_tol=1e-3,
                               em_max_iter=50, em_relax=0.5, gauge_eps=1e-6,
                               permc_spec=None, **law_kwargs):
    """Staggered EM -> heat induction heating of the iron part
    (induction3d_tet10.py:407-639); returns the reference's dict.

    Per EM interval (em_every heat steps): the nonlinear A-V solve at the
    interval-start temperatures (warm-started from the previous interval's
    reluctivity), the iron elements' Joule density as an element-constant
    heat source on the workpiece submesh, and theta-method heat steps on the
    device; stagger_iter > 1 repeats the interval with the EM solve at the
    new temperatures until the temperatures move by less than stagger_tol.
    law_kwargs: the material-law parameters (bsat, mu_mag0, t_curie, w_step,
    sig_hi, sig_lo, t_sig, w_sig) and the capacity law (cp_slope,
    cp_peak_h, cp_peak_w); with a temperature-dependent capacity, C is
    rebuilt from the interval-start element temperatures each interval."""
    import torch
    if iron is None:
        raise ValueError("iron predicate is required (it defines the workpiece)")
    if method not in THETA:
        raise ValueError(f"unknown method {method!r}; use one of {sorted(THETA)}")
    if em_every < 1:
        raise ValueError("em_every must be >= 1")
    if stagger_iter < 1:
        raise ValueError("stagger_iter must be >= 1")
    theta = THETA[method]
    t_curie = float(law_kwargs.get("t_curie", TC_CURIE))
    cp_slope = float(law_kwargs.pop("cp_slope", 0.0))
    cp_peak_h = float(law_kwargs.pop("cp_peak_h", 0.0))
    cp_peak_w = float(law_kwargs.pop("cp_peak_w", 25.0))
    if cp_peak_h != 0.0 and cp_peak_w <= 0.0:
        raise ValueError("cp_peak_w must be positive when cp_peak_h != 0 "
                         f"(got cp_peak_h={cp_peak_h}, cp_peak_w={cp_peak_w})")
    cp_varying = cp_slope != 0.0 or (cp_peak_h != 0.0 and cp_peak_w > 0.0)

    iron_mask, _ = _iron_mask(mesh, iron)
    sub, used_nodes, iron_idx = _extract_submesh_tet10(mesh, iron_mask)
    vols_sub = sub.element_volumes()
    dm = DeviceMesh(sub)
    rt = dm.rt
    K_th, _ = dm.assemble(N.OP_T10_STIFF, coef=k_th, load=None)
    C1, _ = dm.assemble(N.OP_T10_MASS, coef=1.0)
    w1 = _row_sums(dm, C1)                              # ones^T C1
    n_steps = int(np.ceil(t_end / dt - 1e-12))
    if n_steps < 1:
        raise ValueError("t_end must be positive")
    h_step = t_end / n_steps
    els = np.asarray(sub.elements)

    def elem_temps(T_nodes):
        return T_nodes[els].mean(axis=1)

    march = None
    if not cp_varying:
        C_const, _ = dm.assemble(N.OP_T10_MASS, coef=rho_cp)
        march = _HeatMarch(dm, K_th, C_const, theta, h_step)
    T = np.full(sub.n_nodes, float(T0))
    times, T_hist, T_elem_hist = [0.0], [T.copy()], [elem_temps(T)]
    history = []
    E_in = 0.0
    gain_disc = 0.0
    nu_warm = None
    a = v = em_info = None
    marches = []
    try:
        n_intervals = int(np.ceil(n_steps / em_every))
        for iv in range(n_intervals):
            n_sub = min(em_every, n_steps - iv * em_every)
            T_start = T.copy()
            if cp_varying:
                c_e = steel_cp_T(elem_temps(T_start), rho_cp=rho_cp, cp_slope=cp_slope,
                                 cp_peak_h=cp_peak_h, cp_peak_w=cp_peak_w, t_curie=t_curie)
                C_iv, _ = dm.assemble(N.OP_T10_MASS, coef=c_e)
                step = _HeatMarch(dm, K_th, C_iv, theta, h_step)
                marches.append(step)
                w_iv = _row_sums(dm, C_iv)
            else:
                step = march
            d_T_start = torch.from_numpy(T_start).to(rt.device)
            T_est = T_start.copy()
            T_trial = None
            dT_stagger = None
            for s in range(stagger_iter):
                T_elem = np.full(len(mesh.elements), float(T0))
                T_elem[iron_idx] = elem_temps(T_est)
                a, v, em_info = solve_eddy_current_nonlinear_tet10_T(
                    mesh, T_elem, omega, B_applied=B_applied, J_s=J_s, boundary=boundary,
                    a_bc=a_bc, gauge_eps=gauge_eps, permc_spec=permc_spec, iron=iron,
                    tol=em_tol, max_iter=em_max_iter, relax=em_relax, nu_init=nu_warm,
                    **law_kwargs)
                nu_warm = em_info["nu_elem"]
                _, F_Q = dm.assemble(N.OP_T10_STIFF, coef=0.0,
                                     load=np.ascontiguousarray(em_info["Q_elem"][iron_idx]))
                T_new = step.advance(d_T_start, F_Q, n_sub).cpu().numpy()
                if T_trial is not None:
                    dT_stagger = float(np.max(np.abs(T_new - T_trial)))
                T_trial = T_est = T_new
                if stagger_tol is not None and dT_stagger is not None and \
                        dT_stagger < stagger_tol:
                    break
            T = T_trial
            P_used = float(em_info["P"][-1])
            E_in += P_used * (n_sub * h_step)
            if cp_varying:
                gain_disc += float(w_iv @ (T - T_start))
            Te = elem_temps(T)
            mu_iron = em_info["mu_r_elem"][iron_idx]
            history.append({
                "t_end": times[-1] + n_sub * h_step, "P": P_used,
                "em_iterations": em_info["iterations"],
                "em_converged": bool(em_info["converged"]),
                "stagger_passes": s + 1, "stagger_dT": dT_stagger,
                "T_elem_mean": float(Te.mean()), "T_elem_max": float(Te.max()),
                "frac_above_Tc": float(np.mean(Te > t_curie)),
                "mu_r_iron_mean": float(mu_iron.mean()),
                "mu_r_iron_min": float(mu_iron.min()),
                "mu_r_iron": mu_iron.copy(),
                "Q_iron": em_info["Q_elem"][iron_idx].copy(),
            })
            times.append(times[-1] + n_sub * h_step)
            T_hist.append(T.copy())
            T_elem_hist.append(Te.copy())
    finally:
        for m in ([march] if march is not None else []) + marches:
            m.close()
    if not cp_varying:
        enthalpy_gain = float(rho_cp * (w1 @ (T - float(T0))))
        enthalpy_gain_phys = enthalpy_gain
    else:
        enthalpy_gain = gain_disc
        H_end = steel_enthalpy_T(T, t_ref=float(T0), rho_cp=rho_cp, cp_slope=cp_slope,
                                 cp_peak_h=cp_peak_h, cp_peak_w=cp_peak_w, t_curie=t_curie)
        enthalpy_gain_phys = float(w1 @ H_end)
    balance_rel = (E_in - enthalpy_gain) / E_in if E_in > 0 else 0.0
    return {"times": np.array(times), "T_hist": np.array(T_hist),
            "T_elem_hist": np.array(T_elem_hist), "history": history,
            "E_in": E_in, "enthalpy_gain": enthalpy_gain,
            "enthalpy_gain_phys": enthalpy_gain_phys, "cp_varying": bool(cp_varying),
            "balance_rel": balance_rel, "submesh": sub, "iron_idx": iron_idx,
            "used_nodes": used_nodes, "iron_volumes": vols_sub, "a": a, "v": v,
            "em_info": em_info}
