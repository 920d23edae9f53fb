"""The reference's helpers that other modules import (and that a drop-in
must therefore provide) match the oracle on the CPU: P1 gradients, the
Tet10 shape functions, quadrature, per-element operators and reference
mass, Dirichlet value maps, the isotropic constitutive matrix, the strain-
displacement matrices and DOF maps, and the centroid / Keast sample
points."""

import numpy as np
import pytest

import cases as C
from oracle import cfem_oracle as O

pytest.importorskip("torch")   # the package imports torch for device buffers


def _mesh10():
    from cloudfem_b200.mesh import box_mesh_tet10
    return box_mesh_tet10(2, 2, 1, xlim=(0.0, 2.0), ylim=(0.0, 1.0), zlim=(0.0, 0.5))


def test_p1_gradients():
    from cloudfem_b200.fem.tet_poisson import _tet_gradients
    m = O.box_mesh(2, 2, 2, (0.0, 2.0), (0.0, 1.0), (0.0, 3.0))
    p = m.nodes[m.elements]
    Gref, vref = O.tet_gradients(p)
    for e in range(len(p)):
        G, v = _tet_gradients(p[e])
        np.testing.assert_allclose(G, Gref[e], rtol=1e-13, atol=1e-13)
        assert abs(v - vref[e]) <= 1e-15 * vref[e] * 10


def test_tet10_shape_quadrature_operators_mass():
    from cloudfem_b200.fem import tet10 as T
    rng = np.random.default_rng(1)
    L = rng.random((20, 4))
    L /= L.sum(axis=1, keepdims=True)
    for a, b in zip(T.shape_functions(L), O.shape_functions(L)):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(T.quadrature(), O.quadrature()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(T._MASS_REF, O.mass_reference(), rtol=0, atol=1e-15)
    m = _mesh10()
    om = O.Mesh(m.nodes, m.elements, m.boundaries)
    Gall, Nall, xall, vall = O.element_operators_all(om)
    for e in (0, 5, len(m.elements) - 1):
        G, Nq, xq, vol = T.element_operators(m, m.elements[e])
        np.testing.assert_allclose(G, Gall[e], rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(Nq, Nall)
        np.testing.assert_allclose(xq, xall[e], rtol=1e-14, atol=1e-15)
        assert abs(vol - vall[e]) <= 1e-14 * vall[e]


def test_dirichlet_values_later_names_win():
    from cloudfem_b200.fem.tet10 import _dirichlet_values
    m = _mesh10()
    om = O.Mesh(m.nodes, m.elements, m.boundaries)
    bc = {"xmin": 1.0, "ymin": lambda x, y, z: x + 2.0 * z, "xmax": 3.5}
    assert _dirichlet_values(m, bc) == O.dirichlet_values(om, bc)


def test_elastic_helpers():
    from cloudfem_b200.physics import elastic3d as E3
    from cloudfem_b200.physics import elastic_tet10 as E10
    np.testing.assert_array_equal(E3.constitutive_3d(210e9, 0.3),
                                  O.constitutive_3d(210e9, 0.3))
    rng = np.random.default_rng(2)
    for nn, sd in ((4, E3._strain_displacement), (10, E10._strain_displacement10)):
        G = rng.normal(size=(nn, 3))
        np.testing.assert_array_equal(sd(G), O.strain_displacement(G))
    el = np.array([7, 3, 11, 0, 5, 9, 2, 4, 8, 1])
    np.testing.assert_array_equal(E3._dof_map(el[:4]), O.dof_map(el[:4]))
    np.testing.assert_array_equal(E10._dof_map10(el), O.dof_map(el))


def test_sample_points():
    from cloudfem_b200.device import centroids, keast_points
    m = _mesh10()
    om = O.Mesh(m.nodes, m.elements, m.boundaries)
    _, _, xq, _ = O.element_operators_all(om)
    np.testing.assert_allclose(keast_points(m.nodes, m.elements), xq, rtol=1e-14, atol=1e-15)
    p1 = O.box_mesh(*C.P1_BOX)
    np.testing.assert_allclose(centroids(p1.nodes, p1.elements),
                               p1.nodes[p1.elements].mean(axis=1), rtol=0, atol=1e-15)


def test_coefficient_evaluation_in_chunks():
    """Callables are called on chunks of points: the values equal one call
    on all points bitwise (and the reference's pointwise values); scalars,
    constant-returning and scalar-only callables keep their meaning."""
    from cloudfem_b200 import device as D
    rng = np.random.default_rng(3)
    pts = rng.random((3 * D.EVAL_CHUNK + 17, 4, 3))
    f = lambda x, y, z: np.sin(3 * x) * y + np.exp(-z)  # noqa: E731
    v = D.evaluate(f, pts)
    assert v.shape == (3 * D.EVAL_CHUNK + 17, 4)
    np.testing.assert_array_equal(v, f(pts[..., 0], pts[..., 1], pts[..., 2]))
    calls = []

    def counted(x, y, z):
        calls.append(np.size(x))
        return x + y + z
    D.evaluate(counted, pts)
    assert max(calls) == D.EVAL_CHUNK and sum(calls) == pts.size // 3
    assert D.evaluate(2.5, pts) == 2.5
    np.testing.assert_array_equal(D.evaluate(lambda x, y, z: 7.0, pts), np.full(pts.shape[:-1], 7.0))
    few = pts[:5, :1]
    scalar_only = lambda x, y, z: float(x) * 2.0 + (1.0 if y > 0.5 else 0.0)  # noqa: E731
    want = [scalar_only(*p) for p in few.reshape(-1, 3)]
    np.testing.assert_array_equal(D.evaluate(scalar_only, few).ravel(), want)
