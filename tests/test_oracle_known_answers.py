"""Pin the CPU oracle a second way: the analytic known answers that the
reference's own tests check for this path (affine and quadratic exactness,
manufactured convergence rates, shape-function and mass identities, the
elastic patch, clamped uniform heating, the capacity matrix total, a
transient started at its steady state). Each test cites the reference test
whose criterion it restates; the golden fixtures pin the oracle to the
reference's outputs, these pin it to the mathematics."""

import numpy as np
import pytest

import cases as C
from oracle import cfem_oracle as O


def _affine(x, y, z):
    return 1.0 + 2.0 * x - y + 3.0 * z


def test_p1_affine_solution_is_exact():
    """tests/test_tet.py:24-32: P1 reproduces an affine field to 1e-10."""
    m = O.box_mesh(6, 6, 6)
    u = O.solve_p1_poisson(m, k=1.0, f=0.0, bc={s: _affine for s in C.FACES})
    exact = _affine(*m.nodes.T)
    assert np.max(np.abs(u - exact)) < 1e-10


def test_p1_manufactured_rate():
    """tests/test_tet.py:35-69: second-order nodal convergence for
    u = sin(pi x) sin(pi y) sin(pi z), f = 3 pi^2 u (rate in (1.7, 2.3))."""
    def f(x, y, z):
        return 3 * np.pi ** 2 * np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)

    errs = []
    for n in (4, 8):
        m = O.box_mesh(n, n, n)
        u = O.solve_p1_poisson(m, k=1.0, f=f, bc={s: 0.0 for s in C.FACES})
        x, y, z = m.nodes.T
        exact = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        errs.append(np.sqrt(np.mean((u - exact) ** 2)))
    rate = np.log2(errs[0] / errs[1])
    assert 1.7 < rate < 2.3, rate


def test_tet10_shape_quadrature_and_mass_identities():
    """tests/test_tet10.py:75-105: partition of unity of the quadratic
    shape functions and of their derivatives, Keast weights summing to 1,
    and the reference mass summing to the element volume (1e-13)."""
    rng = np.random.default_rng(0)
    L = rng.random((50, 4))
    L /= L.sum(axis=1, keepdims=True)
    N, _ = O.shape_functions(L)
    assert np.max(np.abs(N.sum(axis=1) - 1.0)) < 1e-13
    # reference-coordinate derivatives of the sum vanish
    assert np.max(np.abs(O._dN_dxi(L).sum(axis=1))) < 1e-13
    _, wq = O.quadrature()
    assert abs(wq.sum() - 1.0) < 1e-14
    Mref = O.mass_reference()
    assert abs(Mref.sum() - 1.0) < 1e-13
    assert np.max(np.abs(Mref - Mref.T)) == 0.0
    m = O.box_mesh_tet10(2, 2, 2, (0.0, 2.0), (0.0, 1.0), (0.0, 0.5))
    M = O.assemble_mass_tet10(m, rho_cp=3.0)
    assert abs(M.sum() - 3.0 * 1.0) < 1e-12


def test_tet10_quadratic_patch():
    """tests/test_tet10.py:131-206: Tet10 reproduces a quadratic field
    (u = x^2 + 2 y^2 - z^2 + x y, -lap u = -4) to 1e-11."""
    def u_ex(x, y, z):
        return x * x + 2 * y * y - z * z + x * y

    m = O.box_mesh_tet10(3, 3, 3)
    u = O.solve_tet10_poisson(m, k=1.0, f=-4.0, bc={s: u_ex for s in C.FACES})
    assert np.max(np.abs(u - u_ex(*m.nodes.T))) < 1e-11


def test_tet10_elastic_affine_patch():
    """tests/test_tet10.py:263-342: an affine displacement imposed on the
    whole boundary is reproduced in the interior without body load."""
    Ag = np.array([[1e-3, 2e-4, -1e-4], [3e-4, -5e-4, 1e-4], [0.0, 1e-4, 2e-3]])
    bg = np.array([1e-3, -2e-3, 5e-4])

    def comp(c):
        return lambda x, y, z: Ag[c, 0] * x + Ag[c, 1] * y + Ag[c, 2] * z + bg[c]

    m = O.box_mesh_tet10(3, 2, 2, (0.0, 1.0), (0.0, 0.5), (0.0, 0.5))
    bc = {s: (comp(0), comp(1), comp(2)) for s in C.FACES}
    ux, uy, uz = O.solve_elasticity_tet10(m, 210e9, 0.3, bc=bc)
    exact = m.nodes @ Ag.T + bg
    got = np.stack([ux, uy, uz], axis=1)
    assert np.max(np.abs(got - exact)) < 1e-12 * np.max(np.abs(exact))


def test_p1_clamped_uniform_heating():
    """tests/test_elastic3d.py:105-123: a body clamped on all faces and
    heated uniformly does not move, and every element carries the
    hydrostatic stress -E alpha dT / (1 - 2 nu)."""
    E, nu, alpha, dT = 200e9, 0.3, 1.2e-5, 50.0
    m = O.box_mesh(3, 3, 3)
    u = O.solve_elasticity_p1(m, E, nu, bc={s: (0.0, 0.0, 0.0) for s in C.FACES},
                              T=np.full(m.n_nodes, dT), alpha=alpha, T_ref=0.0)
    assert max(np.max(np.abs(c)) for c in u) < 1e-15
    out = O.element_stress_strain_p1(m, u, E, nu, T=np.full(m.n_nodes, dT), alpha=alpha,
                                     T_ref=0.0)
    sig = out[0] if isinstance(out, tuple) else out
    sig = np.asarray(sig)
    want = -E * alpha * dT / (1.0 - 2.0 * nu)
    np.testing.assert_allclose(sig[:, :3], want, rtol=1e-10)
    assert np.max(np.abs(sig[:, 3:])) < 1e-6 * abs(want)


def test_p1_capacity_matrix_total():
    """tests/test_transient3d.py:83-92: the consistent capacity matrix sums
    to rho_cp times the volume and is symmetric."""
    m = O.box_mesh(3, 2, 4, (0.0, 2.0), (0.0, 1.0), (0.0, 0.5))
    C_ = O.assemble_mass_p1(m, rho_cp=3.6e6)
    assert abs(C_.sum() - 3.6e6 * 1.0) < 1e-12 * 3.6e6
    assert abs(C_ - C_.T).max() == 0.0


@pytest.mark.parametrize("method", ["cn", "be"])
def test_tet10_transient_stays_at_steady_state(method):
    """tests/test_tet10.py:344-387: started from the steady solution of its
    source and boundary data, the theta march does not drift (1e-12)."""
    m = O.box_mesh_tet10(2, 2, 2)
    bc = {s: _affine for s in C.FACES}
    u_ss = O.solve_tet10_poisson(m, k=2.0, f=5.0, bc=bc)
    _, hist = O.transient_heat_tet10(m, k=2.0, rho_cp=3.0, f=5.0, bc=bc,
                                     t_end=1.0, dt=0.1, T0=u_ss, method=method)
    assert np.max(np.abs(hist[-1] - u_ss)) < 1e-12 * np.max(np.abs(u_ss))
