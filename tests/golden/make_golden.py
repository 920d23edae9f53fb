"""Generate the golden-vector fixtures by running the reference package.

Usage (from the repository root, with the reference checkout readable)::

    python tests/golden/make_golden.py /path/to/CloudFEM

The reference (zhangkalin627-svg/CloudFEM, pure Python on NumPy/SciPy)
is imported unchanged from the given path and called on the small cases
of ``cases.py``. Every output array is written to ``ref_fixtures.npz``
next to this script. The fixtures pin both the oracle and the CUDA path;
nothing at test time reads the reference itself.

Sparse matrices are stored as ``<name>__indptr/__indices/__data``.
Dirichlet-modified matrices are stored after ``eliminate_zeros()``,
because the reference's column zeroing keeps an explicit dense block of
zeros (``cloudfem/fem/tet_poisson.py:106``) that carries no information.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases as C  # noqa: E402


def main(ref_path):
    sys.path.insert(0, ref_path)
    from cloudfem.mesh.tet_mesh import box_mesh
    from cloudfem.mesh.tet10_mesh import box_mesh_tet10, tet4_to_tet10
    from cloudfem.fem import tet_poisson as tp
    from cloudfem.fem import tet_heat as th
    from cloudfem.fem import tet10 as t10
    from cloudfem.physics import elastic3d as e3
    from cloudfem.physics import elastic_tet10 as e10
    from cloudfem.physics import em3d_tet10 as em

    out = {}

    def put(name, arr):
        out[name] = np.asarray(arr)

    def put_csr(name, A, eliminate=False):
        A = A.tocsr().copy()
        if eliminate:
            A.eliminate_zeros()
        A.has_sorted_indices  # noqa: B018
        put(name + "__indptr", A.indptr.astype(np.int64))
        put(name + "__indices", A.indices.astype(np.int64))
        put(name + "__data", A.data)
        put(name + "__shape", np.array(A.shape, dtype=np.int64))

    def put_mesh(name, m):
        put(name + "__nodes", m.nodes)
        put(name + "__elements", m.elements)
        for s in C.FACES:
            put(name + "__bnd_" + s, m.boundaries[s])

    # ---------------- P1 scalar ----------------
    nx, ny, nz, xl, yl, zl = C.P1_BOX
    m = box_mesh(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    put_mesh("p1", m)
    put("p1__volumes", m.element_volumes())
    A, b = tp.assemble(m, k=C.k_fn, f=C.f_fn)
    put_csr("p1_K", A)
    put("p1_F", b)
    A0, b0 = tp.assemble(m, k=2.5, f=1.0)
    put_csr("p1_Kconst", A0)
    put("p1_Fconst", b0)
    bc = {"xmin": 0.0, "zmax": C.bc_fn}
    Abc, bbc = tp.apply_dirichlet(A, b, m, bc)
    put_csr("p1_Kbc", Abc, eliminate=True)
    put("p1_Fbc", bbc)
    put("p1_u", tp.solve_tet_poisson(m, k=C.k_fn, f=C.f_fn, bc=bc))
    g, vol = tp._tet_gradients(m.nodes[m.elements[7]])
    put("p1_grad7", g)
    put("p1_vol7", np.array(vol))

    mc = box_mesh(C.P1_CUBE, C.P1_CUBE, C.P1_CUBE)
    put("p1cube_u", tp.solve_tet_poisson(
        mc, k=1.0, f=C.f_sss, bc={s: 0.0 for s in C.FACES}))

    Cm = th.assemble_mass_tet(m, rho_cp=C.rho_fn)
    put_csr("p1_C", Cm)
    Kr, Fr = th.assemble_boundary_terms(
        m, neumann={"xmax": C.q_fn, "ymin": 2.0},
        robin={"zmin": (C.h_fn, C.tinf_fn), "xmin": (4.0, 10.0)})
    put_csr("p1_Krobin", Kr)
    put("p1_Frobin", Fr)
    put("p1_faces_zmin", th._boundary_faces(m, "zmin"))
    put("p1_faces3_xmax", e3.boundary_faces(m, "xmax"))
    times, hist = th.transient_heat_tet(
        m, k=C.k_fn, rho_cp=C.rho_fn, f=C.f_fn, bc={"xmin": 0.0},
        robin={"xmax": (C.h_fn, C.tinf_fn)}, neumann={"ymax": 1.5},
        t_end=0.3, dt=0.1, T0=5.0, method="cn")
    put("p1_tr_times", times)
    put("p1_tr_hist", hist)
    times, hist = th.transient_heat_tet(
        m, k=1.0, rho_cp=1.0, f=0.0, robin={s: (25.0, 20.0) for s in C.FACES},
        t_end=0.2, dt=0.1, T0=C.t_nodal(m.n_nodes), method="be")
    put("p1_tr2_hist", hist)

    # ---------------- Tet10 scalar ----------------
    nx, ny, nz, xl, yl, zl = C.TET10_BOX
    m10 = box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    put_mesh("t10", m10)
    m4 = box_mesh(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    conv = tet4_to_tet10(m4)
    put_mesh("t10conv", conv)
    Lq, wq = t10.quadrature()
    put("t10_Lq", Lq)
    put("t10_wq", wq)
    Ns, dNs = t10.shape_functions(Lq)
    put("t10_N", Ns)
    put("t10_dN", dNs)
    G, N, xq, vol = t10.element_operators(m10, m10.elements[5])
    put("t10_op5_G", G)
    put("t10_op5_xq", xq)
    put("t10_op5_vol", np.array(vol))
    put("t10_MASS_REF", t10._MASS_REF)
    A, b = t10.assemble_tet10(m10, k=C.k_fn, f=C.f_fn)
    put_csr("t10_K", A)
    put("t10_F", b)
    put_csr("t10_C", t10.assemble_mass_tet10(m10, rho_cp=C.rho_fn))
    Kr, Fr = t10.assemble_boundary_terms_tet10(
        m10, neumann={"xmax": C.q_fn, "zmin": 2.0},
        robin={"ymax": (C.h_fn, C.tinf_fn)})
    put_csr("t10_Krobin", Kr)
    put("t10_Frobin", Fr)
    put("t10_faces_ymax", t10._boundary_faces10(m10, "ymax"))
    put("t10_faces10e_xmin", e10.boundary_faces10(m10, "xmin"))
    bc10 = {"xmin": C.bc_fn, "zmax": 0.5}
    Abc, bbc = tp.apply_dirichlet(A, b, m10, bc10)
    put_csr("t10_Kbc", Abc, eliminate=True)
    put("t10_Fbc", bbc)
    put("t10_u", t10.solve_tet10_poisson(m10, k=C.k_fn, f=C.f_fn, bc=bc10))
    times, hist = t10.transient_heat_tet10(
        m10, k=C.k_fn, rho_cp=C.rho_fn, f=1.0, bc={"zmin": 1.0},
        neumann={"xmax": lambda x, y, z, t: 2.0 * t + x},
        robin={"ymin": (3.0, 0.5)}, t_end=0.2, dt=0.05, T0=0.0,
        method="cn")
    put("t10_tr_times", times)
    put("t10_tr_hist", hist)

    # ---------------- P1 elasticity ----------------
    E, nu = 210e9, 0.3
    put("el_D", e3.constitutive_3d(E, nu))
    Tn = C.t_nodal(m.n_nodes)
    A, b = e3.assemble_elasticity_3d(
        m, E, nu, body=(C.bx_fn, None, -7.8e4),
        traction={"xmax": (0.0, 1e5, C.q_fn)}, T=Tn, alpha=1.2e-5,
        T_ref=20.0)
    put_csr("e3_K", A)
    put("e3_F", b)
    bcv = {"xmin": (0.0, 0.0, 0.0), "zmin": (None, None, 0.0),
           "ymax": (None, 1e-4, None)}
    put("e3_u", e3.apply_dirichlet_vec3(A, b, m, bcv))
    ux, uy, uz = e3.solve_elasticity_3d(
        m, E, nu, bc={"xmin": (0.0, 0.0, 0.0)},
        traction={"xmax": (0.0, 0.0, -1e6)})
    put("e3_sol", np.stack([ux, uy, uz]))
    sig, eps = e3.element_stress_strain_3d(
        m, (ux, uy, uz), E, nu, T=C.t_fn, alpha=1e-5, T_ref=20.0)
    put("e3_sig", sig)
    put("e3_eps", eps)
    put("e3_vm", e3.von_mises_3d(sig))

    # ---------------- Tet10 elasticity ----------------
    nx, ny, nz, xl, yl, zl = C.TET10_BEAM
    mb = box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    put_mesh("beam", mb)
    Tb = C.t_nodal(mb.n_nodes)
    A, b = e10.assemble_elasticity_tet10(
        mb, E, nu, body=(None, C.bx_fn, -7.8e4),
        traction={"xmax": (0.0, 0.0, -1e6), "ymin": (C.q_fn, None, 0.0)},
        T=Tb, alpha=1.2e-5, T_ref=20.0)
    put_csr("e10_K", A)
    put("e10_F", b)
    A2, b2 = e10.assemble_elasticity_tet10(mb, E, nu, T=C.t_fn, alpha=1e-5)
    put("e10_Fthermal_fn", b2)
    ux, uy, uz = e10.solve_elasticity_tet10(
        mb, E, nu, bc={"xmin": (0.0, 0.0, 0.0)},
        traction={"xmax": (0.0, 0.0, -1e6)})
    put("e10_sol", np.stack([ux, uy, uz]))
    sig, eps = e10.element_stress_tet10(mb, (ux, uy, uz), E, nu,
                                        T=Tb, alpha=1e-5, T_ref=20.0)
    put("e10_sig", sig)
    put("e10_eps", eps)

    # ---------------- Tet10 A-V eddy-current blocks ----------------
    nx, ny, nz, xl, yl, zl = C.AV_BOX
    ma = box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    K, M, Gs, S, v_nodes, sig_e, cond = em.assemble_tet10_av(
        ma, nu=C.nu_fn, sigma=C.sigma_fn, gauge_eps=1e-6)
    put_csr("av_K", K)
    put_csr("av_M", M)
    put_csr("av_G", Gs)
    put_csr("av_S", S)
    put("av_vnodes", v_nodes)
    put("av_sig_e", sig_e)
    put("av_cond", cond)

    # ---------------- Tet10 A-V phasor solve (SuperLU) ----------------
    mp = box_mesh_tet10(C.AVP_N, C.AVP_N, C.AVP_N)
    a, v = em.solve_eddy_current_tet10(mp, nu=C.nu_fn, sigma=C.AVP_SIGMA,
                                       omega=C.AVP_OMEGA, J_s=C.avp_js,
                                       boundary=list(C.FACES))
    put("avp_a", a)
    put("avp_v", v)
    # post-processing of the phasor field (em3d_tet10.py:378-451, 695-713)
    put("avp_B", em.element_flux_density_tet10(mp, a))
    P, Q = em.total_joule_power_tet10(mp, a, v, C.AVP_SIGMA, C.AVP_OMEGA)
    put("avp_P", np.array(P))
    put("avp_Q", Q)
    put("avp_S", np.array(em.source_complex_power_tet10(mp, a, v, C.avp_js,
                                                         C.AVP_OMEGA)))
    put("avp_Wm", np.array(em.magnetic_energy_tet10(mp, a, nu=C.nu_fn)))
    put("bh_mu_r", em.bh_secant_mu_r(C.BH_H))
    put("bh_mu_r_soft", em.bh_secant_mu_r(C.BH_H, bsat=1.2, mu_mag0=50.0))

    # ---------------- Tet10 nonlinear (secant B-H) phasor A-V ----------------
    mn = box_mesh_tet10(C.AVN_N, C.AVN_N, C.AVN_N)
    a, v, info = em.solve_eddy_current_nonlinear_tet10(
        mn, sigma=C.avn_sigma, omega=C.AVN_OMEGA, B_applied=C.AVN_B,
        iron=C.avn_iron, boundary=list(C.FACES), **C.AVN_KW)
    put("avn_a", a)
    put("avn_v", v)
    put("avn_iterations", np.array(info["iterations"]))
    put("avn_converged", np.array(info["converged"]))
    put("avn_rel_dB", info["rel_dB"])
    put("avn_P", info["P"])
    put("avn_mu_r", info["mu_r_elem"])
    put("avn_B", info["B_elem"])

    # ---------------- induction heating (EM -> heat, staggered) ----------------
    from cloudfem.physics import induction3d_tet10 as ind
    mi = box_mesh_tet10(C.IND_N, C.IND_N, C.IND_N)
    for tag, kw in (("ind", C.IND_KW), ("ind2", C.IND_KW2)):
        res = ind.induction_heating_3d_tet10(mi, iron=C.ind_iron, **kw)
        put(tag + "_times", res["times"])
        put(tag + "_T_hist", res["T_hist"])
        put(tag + "_P", np.array([h["P"] for h in res["history"]]))
        put(tag + "_em_iterations", np.array([h["em_iterations"] for h in res["history"]]))
        put(tag + "_E_in", np.array(res["E_in"]))
        put(tag + "_balance_rel", np.array(res["balance_rel"]))
        put(tag + "_enthalpy_gain", np.array(res["enthalpy_gain"]))
        put(tag + "_mu_r_iron", res["history"][-1]["mu_r_iron"])
    Tt = 20.0 + 900.0 * np.linspace(0.0, 1.0, 9)
    put("law_sigma", ind.steel_sigma_T(Tt))
    put("law_step", ind.curie_step_T(Tt))
    put("law_mu_HT", ind.bh_secant_mu_r_HT(C.BH_H, Tt))
    put("law_cp", ind.steel_cp_T(Tt, cp_slope=1e-3, cp_peak_h=2e6))
    put("law_H", ind.steel_enthalpy_T(Tt, cp_slope=1e-3, cp_peak_h=2e6))

    # ---------------- P1 modal analysis and Newmark dynamics ----------------
    from cloudfem.physics import dynamics3d as dyn
    from cloudfem.physics import modal3d as mod
    nx, ny, nz, xl, yl, zl = C.DYN_BOX
    md = box_mesh(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    put_csr("dyn_M", mod.assemble_mass_3d(md, C.DYN_RHO))
    put_csr("dyn_Ml", mod.assemble_mass_3d(md, C.DYN_RHO, lumped=True))
    for lumped in (False, True):
        fr, modes = mod.solve_modes_3d(md, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC,
                                       n_modes=6, lumped=lumped)
        put("dyn_freqs" + ("_l" if lumped else ""), fr)
        put("dyn_modes" + ("_l" if lumped else ""), modes)
    for tag, kw in (("avg", dict(method="average")),
                    ("lin", dict(method="linear", rayleigh=(5.0, 1e-6)))):
        times, U, V, A = dyn.transient_3d(md, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC,
                                          t_end=C.DYN_T_END, dt=C.DYN_DT,
                                          load=C.dyn_load(md), **kw)
        put("dyn_" + tag + "_times", times)
        put("dyn_" + tag + "_U", U[:, ::7])
        put("dyn_" + tag + "_V", V[-1])
        put("dyn_" + tag + "_A", A[-1])
    times, U, V, A = dyn.modal_superposition_3d(
        md, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC, t_end=C.DYN_T_END,
        dt=C.DYN_DT, load=C.dyn_load(md), n_modes=6, rayleigh=(5.0, 1e-6))
    put("dyn_ms_U", U[:, ::7])
    # single-DOF oscillator through the low-level core
    times, U, V, A = dyn.newmark_integrate(np.array([[2.0]]), np.array([[0.3]]),
                                           np.array([[50.0]]), lambda t: np.array([np.sin(3 * t)]),
                                           2.0, 0.05, u0=1.0, v0=0.0)
    put("dyn_sdof_U", U.ravel())
    put("dyn_sdof_A", A.ravel())

    # ---------------- Tet10 A-V transient (theta method, LU) ----------------
    mt = box_mesh_tet10(C.AVT_N, C.AVT_N, C.AVT_N)
    res = em.transient_eddy_current_tet10(
        mt, nu=C.nu_fn, sigma=C.sigma_fn, t_end=C.AVT_T_END, dt=C.AVT_DT,
        method="cn", J_s=C.avt_js, time_scale=C.avt_scale,
        boundary=list(C.FACES))
    put("avt_P", res["P"])
    put("avt_a_end", res["a_end"])
    put("avt_v_end", res["v_end"])

    path = os.path.join(HERE, "ref_fixtures.npz")
    np.savez_compressed(path, **out)
    size = os.path.getsize(path)
    print(f"wrote {path}: {len(out)} arrays, {size / 1024:.0f} KiB")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the CloudFEM checkout>")
    main(sys.argv[1])
