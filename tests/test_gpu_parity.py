"""CUDA path vs the reference's golden vectors and the oracle.

Integer structure (indptr / indices, face lists, meshes) must match bit
for bit; matrix and load values within 1e-12 of the largest entry; FP64
solutions within 1e-10 relative (the reference's SuperLU answer is itself
only pinned to round-off times the condition number).
"""

import numpy as np
import pytest

import cases as C
from conftest import assert_close, assert_csr_equal, golden_csr

pytestmark = pytest.mark.gpu

E, NU = 210e9, 0.3
SOL_RTOL = 1e-10


@pytest.fixture(scope="module")
def cf():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import cloudfem_b200.fem.tet10 as t10
    import cloudfem_b200.fem.tet_heat as th
    import cloudfem_b200.fem.tet_poisson as tp
    import cloudfem_b200.mesh as mesh
    import cloudfem_b200.physics.elastic3d as e3
    import cloudfem_b200.physics.elastic_tet10 as e10

    class NS:
        pass
    ns = NS()
    ns.tp, ns.th, ns.t10, ns.e3, ns.e10, ns.mesh = tp, th, t10, e3, e10, mesh
    return ns


def _box(spec, fn):
    nx, ny, nz, xl, yl, zl = spec
    return fn(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)


def test_p1_assemble(cf, golden):
    m = _box(C.P1_BOX, cf.mesh.box_mesh)
    A, b = cf.tp.assemble(m, k=C.k_fn, f=C.f_fn)
    assert_csr_equal(A, golden_csr(golden, "p1_K"))
    assert_close(b, golden["p1_F"], 1e-12, "p1 rhs")
    A, b = cf.tp.assemble(m, k=2.5, f=1.0)
    assert_csr_equal(A, golden_csr(golden, "p1_Kconst"))
    assert_close(b, golden["p1_Fconst"], 1e-12, "p1 const rhs")


def test_p1_dirichlet_and_solve(cf, golden):
    m = _box(C.P1_BOX, cf.mesh.box_mesh)
    A, b = cf.tp.assemble(m, k=C.k_fn, f=C.f_fn)
    bc = {"xmin": 0.0, "zmax": C.bc_fn}
    Abc, bbc = cf.tp.apply_dirichlet(A, b, m, bc)
    assert_csr_equal(Abc, golden_csr(golden, "p1_Kbc"), eliminate=True)
    assert_close(bbc, golden["p1_Fbc"], 1e-12, "p1 lifted rhs")
    u = cf.tp.solve_tet_poisson(m, k=C.k_fn, f=C.f_fn, bc=bc)
    assert_close(u, golden["p1_u"], SOL_RTOL, "p1 solution")
    mc = cf.mesh.box_mesh(C.P1_CUBE, C.P1_CUBE, C.P1_CUBE)
    u = cf.tp.solve_tet_poisson(mc, f=C.f_sss, bc={s: 0.0 for s in C.FACES})
    assert_close(u, golden["p1cube_u"], SOL_RTOL, "p1 cube solution")


def test_p1_heat_terms_and_faces(cf, golden):
    m = _box(C.P1_BOX, cf.mesh.box_mesh)
    assert_csr_equal(cf.th.assemble_mass_tet(m, rho_cp=C.rho_fn),
                     golden_csr(golden, "p1_C"))
    K, F = cf.th.assemble_boundary_terms(
        m, neumann={"xmax": C.q_fn, "ymin": 2.0},
        robin={"zmin": (C.h_fn, C.tinf_fn), "xmin": (4.0, 10.0)})
    assert_csr_equal(K, golden_csr(golden, "p1_Krobin"))
    assert_close(F, golden["p1_Frobin"], 1e-12, "robin load")
    np.testing.assert_array_equal(cf.th._boundary_faces(m, "zmin"),
                                  golden["p1_faces_zmin"])
    np.testing.assert_array_equal(cf.e3.boundary_faces(m, "xmax"),
                                  golden["p1_faces3_xmax"])


def test_p1_transient(cf, golden):
    m = _box(C.P1_BOX, cf.mesh.box_mesh)
    times, hist = cf.th.transient_heat_tet(
        m, k=C.k_fn, rho_cp=C.rho_fn, f=C.f_fn, bc={"xmin": 0.0},
        robin={"xmax": (C.h_fn, C.tinf_fn)}, neumann={"ymax": 1.5},
        t_end=0.3, dt=0.1, T0=5.0, method="cn")
    np.testing.assert_array_equal(times, golden["p1_tr_times"])
    assert_close(hist, golden["p1_tr_hist"], SOL_RTOL, "p1 transient")
    _, hist = cf.th.transient_heat_tet(
        m, robin={s: (25.0, 20.0) for s in C.FACES}, t_end=0.2, dt=0.1,
        T0=C.t_nodal(m.n_nodes), method="be")
    assert_close(hist, golden["p1_tr2_hist"], SOL_RTOL, "p1 robin transient")


def test_tet10_scalar(cf, golden):
    m = _box(C.TET10_BOX, cf.mesh.box_mesh_tet10)
    A, b = cf.t10.assemble_tet10(m, k=C.k_fn, f=C.f_fn)
    assert_csr_equal(A, golden_csr(golden, "t10_K"))
    assert_close(b, golden["t10_F"], 1e-12, "t10 rhs")
    assert_csr_equal(cf.t10.assemble_mass_tet10(m, rho_cp=C.rho_fn),
                     golden_csr(golden, "t10_C"))
    K, F = cf.t10.assemble_boundary_terms_tet10(
        m, neumann={"xmax": C.q_fn, "zmin": 2.0},
        robin={"ymax": (C.h_fn, C.tinf_fn)})
    assert_csr_equal(K, golden_csr(golden, "t10_Krobin"))
    assert_close(F, golden["t10_Frobin"], 1e-12, "t10 robin load")
    np.testing.assert_array_equal(cf.t10._boundary_faces10(m, "ymax"),
                                  golden["t10_faces_ymax"])
    np.testing.assert_array_equal(cf.e10.boundary_faces10(m, "xmin"),
                                  golden["t10_faces10e_xmin"])


def test_tet10_solve_and_transient(cf, golden):
    m = _box(C.TET10_BOX, cf.mesh.box_mesh_tet10)
    A, b = cf.t10.assemble_tet10(m, k=C.k_fn, f=C.f_fn)
    bc10 = {"xmin": C.bc_fn, "zmax": 0.5}
    Abc, bbc = cf.tp.apply_dirichlet(A, b, m, bc10)
    assert_csr_equal(Abc, golden_csr(golden, "t10_Kbc"), eliminate=True)
    assert_close(bbc, golden["t10_Fbc"], 1e-12, "t10 lifted rhs")
    u = cf.t10.solve_tet10_poisson(m, k=C.k_fn, f=C.f_fn, bc=bc10)
    assert_close(u, golden["t10_u"], SOL_RTOL, "t10 solution")
    times, hist = cf.t10.transient_heat_tet10(
        m, k=C.k_fn, rho_cp=C.rho_fn, f=1.0, bc={"zmin": 1.0},
        neumann={"xmax": lambda x, y, z, t: 2.0 * t + x},
        robin={"ymin": (3.0, 0.5)}, t_end=0.2, dt=0.05, T0=0.0, method="cn")
    np.testing.assert_array_equal(times, golden["t10_tr_times"])
    assert_close(hist, golden["t10_tr_hist"], SOL_RTOL, "t10 transient")


def test_p1_elasticity(cf, golden):
    m = _box(C.P1_BOX, cf.mesh.box_mesh)
    A, b = cf.e3.assemble_elasticity_3d(
        m, E, NU, body=(C.bx_fn, None, -7.8e4),
        traction={"xmax": (0.0, 1e5, C.q_fn)}, T=C.t_nodal(m.n_nodes),
        alpha=1.2e-5, T_ref=20.0)
    assert_csr_equal(A, golden_csr(golden, "e3_K"))
    assert_close(b, golden["e3_F"], 1e-12, "e3 rhs")
    bcv = {"xmin": (0.0, 0.0, 0.0), "zmin": (None, None, 0.0),
           "ymax": (None, 1e-4, None)}
    u = cf.e3.apply_dirichlet_vec3(A, b, m, bcv)
    assert_close(u, golden["e3_u"], SOL_RTOL, "e3 reduced solve")
    sol = cf.e3.solve_elasticity_3d(m, E, NU, bc={"xmin": (0.0, 0.0, 0.0)},
                                    traction={"xmax": (0.0, 0.0, -1e6)})
    assert_close(np.stack(sol), golden["e3_sol"], SOL_RTOL, "e3 solution")
    sig, eps = cf.e3.element_stress_strain_3d(
        m, tuple(golden["e3_sol"]), E, NU, T=C.t_fn, alpha=1e-5, T_ref=20.0)
    assert_close(sig, golden["e3_sig"], 1e-12, "e3 stress")
    assert_close(eps, golden["e3_eps"], 1e-12, "e3 strain")


def test_tet10_elasticity(cf, golden):
    m = _box(C.TET10_BEAM, cf.mesh.box_mesh_tet10)
    A, b = cf.e10.assemble_elasticity_tet10(
        m, E, NU, body=(None, C.bx_fn, -7.8e4),
        traction={"xmax": (0.0, 0.0, -1e6), "ymin": (C.q_fn, None, 0.0)},
        T=C.t_nodal(m.n_nodes), alpha=1.2e-5, T_ref=20.0)
    assert_csr_equal(A, golden_csr(golden, "e10_K"))
    assert_close(b, golden["e10_F"], 1e-12, "e10 rhs")
    _, b2 = cf.e10.assemble_elasticity_tet10(m, E, NU, T=C.t_fn, alpha=1e-5)
    assert_close(b2, golden["e10_Fthermal_fn"], 1e-12, "e10 thermal rhs")
    sol = cf.e10.solve_elasticity_tet10(m, E, NU, bc={"xmin": (0.0, 0.0, 0.0)},
                                        traction={"xmax": (0.0, 0.0, -1e6)})
    assert_close(np.stack(sol), golden["e10_sol"], 1e-9, "e10 solution")
    sig, eps = cf.e10.element_stress_tet10(
        m, tuple(golden["e10_sol"]), E, NU, T=C.t_nodal(m.n_nodes),
        alpha=1e-5, T_ref=20.0)
    assert_close(sig, golden["e10_sig"], 1e-11, "e10 stress")
    assert_close(eps, golden["e10_eps"], 1e-11, "e10 strain")


def test_mixed_precision_matches_fp64(cf):
    m = cf.mesh.box_mesh_tet10(16, 2, 2, xlim=(0, 0.8), ylim=(0, 0.1),
                               zlim=(0, 0.1))
    kw = dict(bc={"xmin": (0.0, 0.0, 0.0)},
              traction={"xmax": (0.0, 0.0, -1e6)})
    u64 = np.stack(cf.e10.solve_elasticity_tet10(m, E, NU, **kw))
    u32 = np.stack(cf.e10.solve_elasticity_tet10(m, E, NU, precision="mixed",
                                                 rtol=1e-10, **kw))
    err = np.linalg.norm(u32 - u64) / np.linalg.norm(u64)
    assert err <= 1e-8, err


# ------------------------------------------------------- Tet10 A-V blocks
def test_av_blocks_golden(cf, golden):
    """assemble_tet10_av against the reference's blocks on the golden case
    (structure bit-exact, values 1e-12 of the largest entry)."""
    from cloudfem_b200.physics import em3d_tet10 as em
    nx, ny, nz, xl, yl, zl = C.AV_BOX
    m = cf.mesh.box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    K, M, Gs, S, v_nodes, sig_e, cond = em.assemble_tet10_av(
        m, nu=C.nu_fn, sigma=C.sigma_fn, gauge_eps=1e-6)
    g = golden
    assert_csr_equal(K, golden_csr(g, "av_K"))
    assert_csr_equal(M, golden_csr(g, "av_M"))
    assert_csr_equal(Gs, golden_csr(g, "av_G"))
    assert_csr_equal(S, golden_csr(g, "av_S"))
    np.testing.assert_array_equal(v_nodes, g["av_vnodes"])
    np.testing.assert_array_equal(sig_e, g["av_sig_e"])
    np.testing.assert_array_equal(cond, g["av_cond"])


@pytest.mark.parametrize("gauge", [1e-6, 0.0])
def test_av_blocks_vs_oracle(cf, gauge):
    """A larger box with two separate conductors (two pinned V nodes) and,
    with gauge 0, a mass block restricted to the conductors."""
    from cloudfem_b200.physics import em3d_tet10 as em
    from oracle import cfem_oracle as O

    def sigma(x, y, z):
        x = np.asarray(x)
        return np.where((x < 0.3) | (x > 0.75), 3.5e7, 0.0)

    m = cf.mesh.box_mesh_tet10(6, 3, 2, xlim=(0, 1.5), ylim=(0, 0.5), zlim=(0, 0.4))
    mo = O.box_mesh_tet10(6, 3, 2, (0, 1.5), (0, 0.5), (0, 0.4))
    ours = em.assemble_tet10_av(m, nu=C.nu_fn, sigma=sigma, gauge_eps=gauge)
    ref = O.assemble_tet10_av(mo, nu=C.nu_fn, sigma=sigma, gauge_eps=gauge)
    for a, b in zip(ours[:4], ref[:4]):
        assert_csr_equal(a, b)
    np.testing.assert_array_equal(ours[4], ref[4])
    np.testing.assert_array_equal(ours[5], ref[5])
    np.testing.assert_array_equal(ours[6], ref[6])
    # K alone from per-element nu (the nonlinear solver's rebuild)
    cen = m.nodes[np.asarray(m.elements)[:, :4]].mean(axis=1)
    nu_e = np.array([C.nu_fn(*c) for c in cen])
    assert_csr_equal(em._assemble_curl_curl_tet10_nu(m, nu_e), ref[0])


# stated tolerance: COCG to 1e-10 relative residual agrees with SuperLU's
# answer to 1e-8 relative
AVP_TOL = 1e-8


def test_av_phasor_golden(cf, golden):
    """Phasor A-V solve (device COCG) against the reference's SuperLU answer."""
    from cloudfem_b200.physics import em3d_tet10 as em
    m = cf.mesh.box_mesh_tet10(C.AVP_N, C.AVP_N, C.AVP_N)
    a, v = em.solve_eddy_current_tet10(m, nu=C.nu_fn, sigma=C.AVP_SIGMA,
                                       omega=C.AVP_OMEGA, J_s=C.avp_js,
                                       boundary=list(C.FACES))
    for mine, ref in ((a, golden["avp_a"]), (v, golden["avp_v"])):
        assert np.linalg.norm(mine - ref) <= AVP_TOL * np.linalg.norm(ref)


def test_av_phasor_conductor_in_air(cf):
    """Half-conducting box in a background field (gauge-regularised air,
    pinned V node) against the oracle's SuperLU solve."""
    from cloudfem_b200.physics import em3d_tet10 as em
    from oracle import cfem_oracle as O
    m = cf.mesh.box_mesh_tet10(4, 4, 4)
    mo = O.box_mesh_tet10(4, 4, 4)
    kw = dict(nu=C.nu_fn, sigma=C.sigma_fn, omega=C.AVP_OMEGA, B_applied=(0.0, 0.0, 1e-3))
    a, v = em.solve_eddy_current_tet10(m, **kw)
    ao, vo = O.solve_eddy_current_tet10(mo, **kw)
    assert np.linalg.norm(a - ao) <= 1e-7 * np.linalg.norm(ao)
    assert np.linalg.norm(v - vo) <= 1e-7 * np.linalg.norm(vo)
    with pytest.raises(ValueError):
        em.solve_eddy_current_tet10(m, nu=C.nu_fn, sigma=0.0, omega=1.0, B_applied=(0, 0, 1))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_av_transient_golden(cf, golden, precision):
    """Transient A-V eddy currents (theta method; device PCG on the
    symmetrised step matrix) against the reference's LU march."""
    from cloudfem_b200.physics import em3d_tet10 as em
    m = cf.mesh.box_mesh_tet10(C.AVT_N, C.AVT_N, C.AVT_N)
    r = em.transient_eddy_current_tet10(
        m, nu=C.nu_fn, sigma=C.sigma_fn, t_end=C.AVT_T_END, dt=C.AVT_DT,
        method="cn", J_s=C.avt_js, time_scale=C.avt_scale,
        boundary=list(C.FACES), precision=precision)
    tol = 1e-9 if precision == "fp64" else 1e-7
    assert np.abs(r["P"] - golden["avt_P"]).max() <= tol * np.abs(golden["avt_P"]).max()
    for k in ("a_end", "v_end"):
        ref = golden["avt_" + k]
        assert np.linalg.norm(r[k] - ref) <= tol * np.linalg.norm(ref)


def test_t10_joule_power_kernel_vs_oracle(cf):
    """The device Joule-power kernel (cfem_t10_joule_power) against the
    oracle's restatement of em3d_tet10.py:665-692 on seeded fields over a
    mesh with conducting and non-conducting elements: power within 1e-12,
    per-element densities entry-wise within 1e-12, and bitwise the same on a
    repeat (fixed-order sum)."""
    from cloudfem_b200.physics import em3d_tet10 as em
    from oracle import cfem_oracle as O
    m = cf.mesh.box_mesh_tet10(4, 3, 3)
    mo = O.box_mesh_tet10(4, 3, 3)
    rng = np.random.default_rng(7)
    n = m.n_nodes
    a0, a1, v = rng.normal(size=3 * n), rng.normal(size=3 * n), rng.normal(size=n)
    P, Q = em.transient_joule_power_tet10(m, a0, a1, v, C.sigma_fn, 0.01)
    Po, Qo = O.transient_joule_power_tet10(mo, a0, a1, v, C.sigma_fn, 0.01)
    assert (Q == 0).any() and (Q > 0).any()
    assert abs(P - Po) <= 1e-12 * abs(Po), (P, Po)
    assert np.all(np.abs(Q - Qo) <= 1e-12 * np.abs(Qo) + 1e-300)
    P2, _ = em.transient_joule_power_tet10(m, a0, a1, v, C.sigma_fn, 0.01)
    assert P2 == P


def test_element_source_load_sums_to_power(cf):
    """_element_source_load (induction3d_tet10.py:390-404) on the device
    against the reference formula evaluated on the host per element
    (vol Q_e sum_q w_q N_q, scattered to the element's nodes), and
    ones . F = sum_e Q_e V_e."""
    from cloudfem_b200.fem.tet10 import element_operators, quadrature
    from cloudfem_b200.physics.induction3d_tet10 import _element_source_load
    m = cf.mesh.box_mesh_tet10(3, 2, 2)
    Q = np.random.default_rng(3).uniform(1e5, 1e6, m.n_elements)
    F = _element_source_load(m, Q)
    _, wq = quadrature()
    ref = np.zeros(m.n_nodes)
    for e, el in enumerate(np.asarray(m.elements)):
        _, Nq, _, vol = element_operators(m, el)
        np.add.at(ref, el, vol * Q[e] * (Nq * wq[:, None]).sum(axis=0))
    assert np.abs(F - ref).max() <= 1e-12 * np.abs(ref).max()
    assert abs(F.sum() - float(Q @ m.element_volumes())) <= 1e-12 * F.sum()


def test_av_magnetic_energy_golden(cf, golden):
    """W_m = Re(a^H K a)/4 with K assembled on the device."""
    from cloudfem_b200.physics import em3d_tet10 as em
    m = cf.mesh.box_mesh_tet10(C.AVP_N, C.AVP_N, C.AVP_N)
    W = em.magnetic_energy_tet10(m, golden["avp_a"], nu=C.nu_fn)
    Wg = float(golden["avp_Wm"])
    assert abs(W - Wg) <= 1e-12 * abs(Wg)


def test_av_nonlinear_picard_golden(cf, golden):
    """Secant B-H Picard loop (K rebuilt on the device each iteration,
    device COCG per linear solve) against the reference's SuperLU loop:
    same iteration count and convergence flag; fields, power history and
    permeabilities within the linear solves' accuracy."""
    from cloudfem_b200.physics import em3d_tet10 as em
    g = golden
    m = cf.mesh.box_mesh_tet10(C.AVN_N, C.AVN_N, C.AVN_N)
    a, v, info = em.solve_eddy_current_nonlinear_tet10(
        m, sigma=C.avn_sigma, omega=C.AVN_OMEGA, B_applied=C.AVN_B,
        iron=C.avn_iron, boundary=list(C.FACES), **C.AVN_KW)
    assert info["iterations"] == int(g["avn_iterations"])
    assert info["converged"] == bool(g["avn_converged"])
    tol = 1e-8
    assert np.linalg.norm(a - g["avn_a"]) <= tol * np.linalg.norm(g["avn_a"])
    assert np.linalg.norm(v - g["avn_v"]) <= tol * np.linalg.norm(g["avn_v"])
    assert_close(info["P"], g["avn_P"], tol, "power history")
    assert_close(info["mu_r_elem"], g["avn_mu_r"], tol, "mu_r")
    assert_close(np.abs(info["B_elem"]), np.abs(g["avn_B"]), tol, "|B|")
    assert np.abs(info["rel_dB"] - g["avn_rel_dB"]).max() <= 1e-6 * g["avn_rel_dB"].max()


@pytest.mark.parametrize("tag", ["ind", "ind2"])
def test_induction_heating_golden(cf, golden, tag):
    """Staggered EM -> heat induction heating (device Picard A-V solves and
    device heat march) against the reference's SuperLU/LU chain: constant
    capacity with backward Euler, and T-dependent capacity with Crank-
    Nicolson and two stagger passes per interval."""
    from cloudfem_b200.physics import induction3d_tet10 as ind
    g = golden
    kw = dict(C.IND_KW if tag == "ind" else C.IND_KW2)
    m = cf.mesh.box_mesh_tet10(C.IND_N, C.IND_N, C.IND_N)
    res = ind.induction_heating_3d_tet10(m, iron=C.ind_iron, **kw)
    np.testing.assert_array_equal(res["times"], g[tag + "_times"])
    assert [h["em_iterations"] for h in res["history"]] == list(g[tag + "_em_iterations"])
    tol = 1e-8
    assert_close(res["T_hist"], g[tag + "_T_hist"], tol, "temperatures")
    assert_close([h["P"] for h in res["history"]], g[tag + "_P"], tol, "power")
    assert abs(res["E_in"] - float(g[tag + "_E_in"])) <= tol * float(g[tag + "_E_in"])
    assert abs(res["balance_rel"]) <= 1e-9
    assert_close(res["history"][-1]["mu_r_iron"], g[tag + "_mu_r_iron"], tol, "mu_r")


def test_boundary_faces_on_device_against_oracle(cf):
    """Device face dedup (two stable radix sorts of corner triples) against
    the oracle's dict-order restatement: every face of a 24^3 P1 box and a
    Tet10 box, named sets and 'interior' sets whose faces occur twice."""
    from cloudfem_b200.device import DeviceMesh
    from oracle import cfem_oracle as O
    m = cf.mesh.box_mesh(24, 20, 16)
    mo = O.Mesh(m.nodes, m.elements, m.boundaries)
    dm = DeviceMesh(m)
    for name in C.FACES:
        np.testing.assert_array_equal(dm.boundary_faces(name), O.boundary_faces_p1(mo, name))
    # a node set containing interior faces: the x < 0.5 half of the box
    half = np.nonzero(m.nodes[:, 0] <= 0.5)[0]
    m.boundaries["half"] = half
    mo.boundaries["half"] = half
    np.testing.assert_array_equal(DeviceMesh(m).boundary_faces("half"),
                                  O.boundary_faces_p1(mo, "half"))
    m10 = cf.mesh.box_mesh_tet10(6, 5, 4)
    mo10 = O.Mesh(m10.nodes, m10.elements, m10.boundaries)
    dm10 = DeviceMesh(m10)
    for name in ("xmin", "ymax", "zmin"):
        np.testing.assert_array_equal(dm10.boundary_faces(name, tet10=True),
                                      O.boundary_faces10(mo10, name))
