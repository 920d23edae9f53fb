"""Host-side boundary-face integrals of the product (`cloudfem_b200._faces`)
against the oracle on the same face lists, on the CPU: P1 Neumann, Robin
and traction (centroid rules), Tet10 Neumann (time-dependent flux), Robin
and traction (Dunavant-6 and 3-point rules)."""

import numpy as np
import pytest

import cases as C
from oracle import cfem_oracle as O


@pytest.fixture(scope="module")
def faces():
    pytest.importorskip("torch")   # the package's device module imports it
    from cloudfem_b200 import _faces
    return _faces


def _q(x, y, z):
    return 1.0 + x * y - 0.5 * z


def _h(x, y, z):
    return 10.0 + 5.0 * x


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.max(np.abs(b)))


def _csr_close(A, B):
    d = (A - B).tocsr()
    d.eliminate_zeros()
    scale = max(1.0, abs(B).max())
    assert d.nnz == 0 or abs(d).max() <= 1e-13 * scale


def test_p1_neumann_robin(faces):
    m = O.box_mesh(3, 2, 2, (0.0, 2.0), (0.0, 1.0), (0.0, 0.5))
    n = m.n_nodes
    Kref, Fref = O.assemble_boundary_terms_p1(
        m, neumann={"xmax": _q, "ymin": 2.5}, robin={"zmin": (_h, 20.0), "xmin": (25.0, _q)})
    F = np.zeros(n)
    rows, cols, data = [], [], []
    faces.p1_neumann(m.nodes, O.boundary_faces_p1(m, "xmax"), _q, F)
    faces.p1_neumann(m.nodes, O.boundary_faces_p1(m, "ymin"), 2.5, F)
    faces.p1_robin(m.nodes, O.boundary_faces_p1(m, "zmin"), _h, 20.0, F, rows, cols, data)
    faces.p1_robin(m.nodes, O.boundary_faces_p1(m, "xmin"), 25.0, _q, F, rows, cols, data)
    _close(F, Fref)
    _csr_close(faces.coo_csr(rows, cols, data, n), Kref)


def test_p1_traction(faces):
    m = O.box_mesh(2, 2, 3)
    trac = {"xmax": (0.0, None, lambda x, y, z: -1e6 * (1.0 + y)), "zmin": (3.0, 2.0, 1.0)}
    ref = np.zeros(3 * m.n_nodes)
    O._traction_p1(m, trac, ref)
    got = np.zeros(3 * m.n_nodes)
    for name, comps in trac.items():
        faces.p1_traction(m.nodes, O.boundary_faces_p1(m, name), comps, got)
    _close(got, ref)


def test_tet10_neumann_time_dependent_and_robin(faces):
    m = O.box_mesh_tet10(2, 2, 2)
    n = m.n_nodes

    def qt(x, y, z, t):
        return (1.0 + x) * np.cos(3.0 * t) + y * z

    for t in (0.0, 0.3):
        ref = O.neumann_load_tet10(m, {"xmin": qt, "zmax": _q, "ymax": 4.0}, t)
        F = np.zeros(n)
        for name, q in (("xmin", qt), ("zmax", _q), ("ymax", 4.0)):
            faces.t10_neumann(m.nodes, O.boundary_faces10(m, name), q, t, F)
        _close(F, ref)
    Kref, Fref = O.robin_terms_tet10(m, {"ymin": (_h, 20.0), "zmin": (25.0, _q)})
    F = np.zeros(n)
    rows, cols, data = [], [], []
    faces.t10_robin(m.nodes, O.boundary_faces10(m, "ymin"), _h, 20.0, F, rows, cols, data)
    faces.t10_robin(m.nodes, O.boundary_faces10(m, "zmin"), 25.0, _q, F, rows, cols, data)
    _close(F, Fref)
    _csr_close(faces.coo_csr(rows, cols, data, n), Kref)


def test_tet10_traction(faces):
    nx, ny, nz, xl, yl, zl = C.TET10_BEAM
    m = O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)
    trac = {"xmax": (0.0, None, lambda x, y, z: -1e6 * (1.0 + z)), "ymin": (1.0, 2.0, 3.0)}
    _, r1 = O.assemble_elasticity_tet10(m, 210e9, 0.3, traction=trac)
    _, r0 = O.assemble_elasticity_tet10(m, 210e9, 0.3)
    got = np.zeros(3 * m.n_nodes)
    for name, comps in trac.items():
        faces.t10_traction(m.nodes, O.boundary_faces10(m, name), comps, got)
    _close(got, r1 - r0)
