"""Product meshers reproduce the reference meshes bit for bit."""

import numpy as np

import cases as C
from cloudfem_b200.mesh import box_mesh, box_mesh_tet10, tet4_to_tet10


def _check(golden, name, m):
    np.testing.assert_array_equal(m.nodes, golden[name + "__nodes"])
    np.testing.assert_array_equal(m.elements, golden[name + "__elements"])
    for s in C.FACES:
        np.testing.assert_array_equal(m.boundaries[s],
                                      golden[name + "__bnd_" + s])


def _box(spec, fn):
    nx, ny, nz, xl, yl, zl = spec
    return fn(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)


def test_box_mesh(golden):
    m = _box(C.P1_BOX, box_mesh)
    _check(golden, "p1", m)
    np.testing.assert_allclose(m.element_volumes(), golden["p1__volumes"],
                               rtol=0, atol=1e-16)


def test_tet10_meshes(golden):
    _check(golden, "t10", _box(C.TET10_BOX, box_mesh_tet10))
    _check(golden, "beam", _box(C.TET10_BEAM, box_mesh_tet10))
    _check(golden, "t10conv", tet4_to_tet10(_box(C.TET10_BOX, box_mesh)))


def test_mesh_sizes_of_benchmark_configs():
    m = box_mesh(20, 20, 20)
    assert m.n_nodes == 9261 and m.n_elements == 48000
    mb = box_mesh_tet10(8, 1, 1)
    assert mb.n_elements == 48


def test_add_at_matches_numpy():
    from cloudfem_b200._faces import add_at
    rng = np.random.default_rng(6)
    idx = rng.integers(0, 300, 5000)
    for v in (rng.random(5000), rng.random(5000) * (1 - 0.5j)):
        a = np.zeros(300, dtype=v.dtype)
        b = a.copy()
        np.add.at(a, idx, v)
        add_at(b, idx, v)
        np.testing.assert_allclose(b, a, rtol=1e-14, atol=0)
