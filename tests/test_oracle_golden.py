"""Pin the CPU oracle to the reference's own outputs (golden fixtures)."""

import numpy as np
import pytest

import cases as C
from conftest import assert_close, assert_csr_equal, golden_csr
from oracle import cfem_oracle as O

E, NU = 210e9, 0.3


@pytest.fixture(scope="module")
def p1():
    nx, ny, nz, xl, yl, zl = C.P1_BOX
    return O.box_mesh(nx, ny, nz, xl, yl, zl)


@pytest.fixture(scope="module")
def t10():
    nx, ny, nz, xl, yl, zl = C.TET10_BOX
    return O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)


@pytest.fixture(scope="module")
def beam():
    nx, ny, nz, xl, yl, zl = C.TET10_BEAM
    return O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)


def _check_mesh(golden, name, m):
    np.testing.assert_array_equal(m.nodes, golden[name + "__nodes"])
    np.testing.assert_array_equal(m.elements, golden[name + "__elements"])
    for s in C.FACES:
        np.testing.assert_array_equal(m.boundaries[s],
                                      golden[name + "__bnd_" + s])


def test_meshes_bit_exact(golden, p1, t10, beam):
    _check_mesh(golden, "p1", p1)
    _check_mesh(golden, "t10", t10)
    _check_mesh(golden, "beam", beam)
    nx, ny, nz, xl, yl, zl = C.TET10_BOX
    _check_mesh(golden, "t10conv",
                O.tet4_to_tet10(O.box_mesh(nx, ny, nz, xl, yl, zl)))
    assert_close(p1.element_volumes(), golden["p1__volumes"], 1e-15)


def test_p1_assembly(golden, p1):
    A, b = O.assemble_p1(p1, k=C.k_fn, f=C.f_fn)
    assert_csr_equal(A, golden_csr(golden, "p1_K"))
    assert_close(b, golden["p1_F"], 1e-13)
    A, b = O.assemble_p1(p1, k=2.5, f=1.0)
    assert_csr_equal(A, golden_csr(golden, "p1_Kconst"))
    assert_close(b, golden["p1_Fconst"], 1e-13)
    g, vol = O.tet_gradients(p1.nodes[p1.elements[7:8]])
    assert_close(g[0], golden["p1_grad7"], 1e-14)
    assert_close(vol[0], golden["p1_vol7"], 1e-15)


def test_p1_dirichlet_and_solve(golden, p1):
    A, b = O.assemble_p1(p1, k=C.k_fn, f=C.f_fn)
    bc = {"xmin": 0.0, "zmax": C.bc_fn}
    Abc, bbc = O.apply_dirichlet(A, b, p1, bc)
    assert_csr_equal(Abc, golden_csr(golden, "p1_Kbc"), eliminate=True)
    assert_close(bbc, golden["p1_Fbc"], 1e-13)
    u = O.solve_p1_poisson(p1, k=C.k_fn, f=C.f_fn, bc=bc)
    assert_close(u, golden["p1_u"], 1e-12)
    mc = O.box_mesh(C.P1_CUBE, C.P1_CUBE, C.P1_CUBE)
    u = O.solve_p1_poisson(mc, f=C.f_sss, bc={s: 0.0 for s in C.FACES})
    assert_close(u, golden["p1cube_u"], 1e-12)


def test_p1_heat_terms(golden, p1):
    assert_csr_equal(O.assemble_mass_p1(p1, rho_cp=C.rho_fn),
                     golden_csr(golden, "p1_C"))
    K, F = O.assemble_boundary_terms_p1(
        p1, neumann={"xmax": C.q_fn, "ymin": 2.0},
        robin={"zmin": (C.h_fn, C.tinf_fn), "xmin": (4.0, 10.0)})
    assert_csr_equal(K, golden_csr(golden, "p1_Krobin"))
    assert_close(F, golden["p1_Frobin"], 1e-13)
    np.testing.assert_array_equal(O.boundary_faces_p1(p1, "zmin"),
                                  golden["p1_faces_zmin"])
    np.testing.assert_array_equal(O.boundary_faces_p1(p1, "xmax"),
                                  golden["p1_faces3_xmax"])


def test_p1_transient(golden, p1):
    times, hist = O.transient_heat_p1(
        p1, k=C.k_fn, rho_cp=C.rho_fn, f=C.f_fn, bc={"xmin": 0.0},
        robin={"xmax": (C.h_fn, C.tinf_fn)}, neumann={"ymax": 1.5},
        t_end=0.3, dt=0.1, T0=5.0, method="cn")
    assert_close(times, golden["p1_tr_times"], 0.0)
    assert_close(hist, golden["p1_tr_hist"], 1e-12)
    _, hist = O.transient_heat_p1(
        p1, robin={s: (25.0, 20.0) for s in C.FACES}, t_end=0.2, dt=0.1,
        T0=C.t_nodal(p1.n_nodes), method="be")
    assert_close(hist, golden["p1_tr2_hist"], 1e-12)


def test_tet10_helpers(golden, t10):
    Lq, wq = O.quadrature()
    assert_close(Lq, golden["t10_Lq"], 0.0)
    assert_close(wq, golden["t10_wq"], 0.0)
    N, dN = O.shape_functions(Lq)
    assert_close(N, golden["t10_N"], 0.0)
    assert_close(dN, golden["t10_dN"], 0.0)
    assert_close(O.MASS_REF, golden["t10_MASS_REF"], 1e-15)
    G, _, xq, vol = O.element_operators_all(t10)
    assert_close(G[5], golden["t10_op5_G"], 1e-14)
    assert_close(xq[5], golden["t10_op5_xq"], 1e-15)
    assert_close(vol[5], golden["t10_op5_vol"], 1e-15)


def test_tet10_assembly(golden, t10):
    A, b = O.assemble_tet10(t10, k=C.k_fn, f=C.f_fn)
    assert_csr_equal(A, golden_csr(golden, "t10_K"))
    assert_close(b, golden["t10_F"], 1e-13)
    assert_csr_equal(O.assemble_mass_tet10(t10, rho_cp=C.rho_fn),
                     golden_csr(golden, "t10_C"))
    K, F = O.assemble_boundary_terms_tet10(
        t10, neumann={"xmax": C.q_fn, "zmin": 2.0},
        robin={"ymax": (C.h_fn, C.tinf_fn)})
    assert_csr_equal(K, golden_csr(golden, "t10_Krobin"))
    assert_close(F, golden["t10_Frobin"], 1e-13)
    np.testing.assert_array_equal(O.boundary_faces10(t10, "ymax"),
                                  golden["t10_faces_ymax"])
    np.testing.assert_array_equal(O.boundary_faces10(t10, "xmin"),
                                  golden["t10_faces10e_xmin"])


def test_tet10_dirichlet_solve_transient(golden, t10):
    A, b = O.assemble_tet10(t10, k=C.k_fn, f=C.f_fn)
    bc10 = {"xmin": C.bc_fn, "zmax": 0.5}
    Abc, bbc = O.apply_dirichlet(A, b, t10, bc10)
    assert_csr_equal(Abc, golden_csr(golden, "t10_Kbc"), eliminate=True)
    assert_close(bbc, golden["t10_Fbc"], 1e-13)
    u = O.solve_tet10_poisson(t10, k=C.k_fn, f=C.f_fn, bc=bc10)
    assert_close(u, golden["t10_u"], 1e-12)
    times, hist = O.transient_heat_tet10(
        t10, k=C.k_fn, rho_cp=C.rho_fn, f=1.0, bc={"zmin": 1.0},
        neumann={"xmax": lambda x, y, z, t: 2.0 * t + x},
        robin={"ymin": (3.0, 0.5)}, t_end=0.2, dt=0.05, T0=0.0,
        method="cn")
    assert_close(times, golden["t10_tr_times"], 0.0)
    assert_close(hist, golden["t10_tr_hist"], 1e-12)


def test_p1_elasticity(golden, p1):
    assert_close(O.constitutive_3d(E, NU), golden["el_D"], 0.0)
    A, b = O.assemble_elasticity_p1(
        p1, E, NU, body=(C.bx_fn, None, -7.8e4),
        traction={"xmax": (0.0, 1e5, C.q_fn)}, T=C.t_nodal(p1.n_nodes),
        alpha=1.2e-5, T_ref=20.0)
    assert_csr_equal(A, golden_csr(golden, "e3_K"))
    assert_close(b, golden["e3_F"], 1e-13)
    bcv = {"xmin": (0.0, 0.0, 0.0), "zmin": (None, None, 0.0),
           "ymax": (None, 1e-4, None)}
    assert_close(O.apply_dirichlet_vec3(A, b, p1, bcv), golden["e3_u"],
                 1e-11)
    sol = O.solve_elasticity_p1(p1, E, NU, bc={"xmin": (0.0, 0.0, 0.0)},
                                traction={"xmax": (0.0, 0.0, -1e6)})
    assert_close(np.stack(sol), golden["e3_sol"], 1e-11)
    sig, eps = O.element_stress_strain_p1(p1, sol, E, NU, T=C.t_fn,
                                          alpha=1e-5, T_ref=20.0)
    assert_close(sig, golden["e3_sig"], 1e-10)
    assert_close(eps, golden["e3_eps"], 1e-10)
    assert_close(O.von_mises_3d(golden["e3_sig"]), golden["e3_vm"], 1e-15)


def test_tet10_elasticity(golden, beam):
    A, b = O.assemble_elasticity_tet10(
        beam, E, NU, body=(None, C.bx_fn, -7.8e4),
        traction={"xmax": (0.0, 0.0, -1e6), "ymin": (C.q_fn, None, 0.0)},
        T=C.t_nodal(beam.n_nodes), alpha=1.2e-5, T_ref=20.0)
    assert_csr_equal(A, golden_csr(golden, "e10_K"))
    assert_close(b, golden["e10_F"], 1e-13)
    _, b2 = O.assemble_elasticity_tet10(beam, E, NU, T=C.t_fn, alpha=1e-5)
    assert_close(b2, golden["e10_Fthermal_fn"], 1e-13)
    sol = O.solve_elasticity_tet10(beam, E, NU, bc={"xmin": (0.0, 0.0, 0.0)},
                                   traction={"xmax": (0.0, 0.0, -1e6)})
    assert_close(np.stack(sol), golden["e10_sol"], 1e-10)
    sig, eps = O.element_stress_tet10(beam, sol, E, NU,
                                      T=C.t_nodal(beam.n_nodes), alpha=1e-5,
                                      T_ref=20.0)
    assert_close(sig, golden["e10_sig"], 1e-9)
    assert_close(eps, golden["e10_eps"], 1e-9)


def test_av_blocks(golden):
    nx, ny, nz, xl, yl, zl = C.AV_BOX
    m = O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)
    K, M, Gs, S, v_nodes, sig_e, cond = O.assemble_tet10_av(
        m, nu=C.nu_fn, sigma=C.sigma_fn, gauge_eps=1e-6)
    assert_csr_equal(K, golden_csr(golden, "av_K"))
    assert_csr_equal(M, golden_csr(golden, "av_M"))
    assert_csr_equal(Gs, golden_csr(golden, "av_G"))
    assert_csr_equal(S, golden_csr(golden, "av_S"))
    np.testing.assert_array_equal(v_nodes, golden["av_vnodes"])
    np.testing.assert_array_equal(sig_e, golden["av_sig_e"])
    np.testing.assert_array_equal(cond, golden["av_cond"])


def test_av_phasor_solve(golden):
    m = O.box_mesh_tet10(C.AVP_N, C.AVP_N, C.AVP_N)
    a, v = O.solve_eddy_current_tet10(m, nu=C.nu_fn, sigma=C.AVP_SIGMA,
                                      omega=C.AVP_OMEGA, J_s=C.avp_js,
                                      boundary=list(C.FACES))
    for mine, ref in ((a, golden["avp_a"]), (v, golden["avp_v"])):
        assert np.linalg.norm(mine - ref) <= 1e-10 * np.linalg.norm(ref)


def test_av_transient(golden):
    m = O.box_mesh_tet10(C.AVT_N, C.AVT_N, C.AVT_N)
    r = O.transient_eddy_current_tet10(
        m, nu=C.nu_fn, sigma=C.sigma_fn, t_end=C.AVT_T_END, dt=C.AVT_DT,
        method="cn", J_s=C.avt_js, time_scale=C.avt_scale, boundary=list(C.FACES))
    assert np.abs(r["P"] - golden["avt_P"]).max() <= 1e-10 * np.abs(golden["avt_P"]).max()
    for k in ("a_end", "v_end"):
        ref = golden["avt_" + k]
        assert np.linalg.norm(r[k] - ref) <= 1e-10 * np.linalg.norm(ref)
