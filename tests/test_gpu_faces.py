"""Boundary-face integrals on the device (`cloudfem_b200._faces`:
cfem_face_geometry, cfem_face_integrate) against the oracle on the same
face lists: P1 Neumann, Robin and traction (centroid rules), Tet10
Neumann (time-dependent flux), Robin and traction (Dunavant-6 and 3-point
rules); loads and matrices within 1e-13 of the largest entry, and
bitwise the same on a repeat (stable-sorted, fixed-order sums)."""

import numpy as np
import pytest

import cases as C
from oracle import cfem_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


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


def _dev_faces(torch, f):
    return torch.from_numpy(np.ascontiguousarray(f, dtype=np.int64)).to("cuda")


def _run(torch, m, rule, neumann, robin, ncomp=1, faces_of=None):
    """Device loads (and Robin matrix) over the oracle's face lists."""
    from cloudfem_b200 import _faces
    from cloudfem_b200.device import DeviceMesh
    dm = DeviceMesh(m)
    F = torch.zeros(ncomp * m.n_nodes, dtype=torch.float64, device="cuda")
    K = torch.zeros(dm.pattern.nnz, dtype=torch.float64, device="cuda")
    flist = []
    for name, specs in neumann:
        _faces.add_load(dm, _dev_faces(torch, faces_of(m, name)), rule, specs, F)
    for name, (h, tinf) in robin:
        f = faces_of(m, name)
        _faces.add_robin(dm, _dev_faces(torch, f), rule, h, tinf, F, K)
        flist.append(f)
    Kh = _faces.face_csr(dm, flist, K) if flist else None
    return F.cpu().numpy(), Kh


def test_p1_neumann_robin(torch):
    from cloudfem_b200 import _faces
    m = O.box_mesh(3, 2, 2, (0.0, 2.0), (0.0, 1.0), (0.0, 0.5))
    Kref, Fref = O.assemble_boundary_terms_p1(
        m, neumann={"xmax": _q, "ymin": 2.5}, robin={"zmin": (_h, 20.0), "xmin": (25.0, _q)})
    args = (_faces.P1, [("xmax", [_q]), ("ymin", [2.5])],
            [("zmin", (_h, 20.0)), ("xmin", (25.0, _q))])
    F, K = _run(torch, m, *args, faces_of=O.boundary_faces_p1)
    _close(F, Fref)
    _csr_close(K, Kref)
    F2, K2 = _run(torch, m, *args, faces_of=O.boundary_faces_p1)
    assert np.array_equal(F, F2) and np.array_equal(K.data, K2.data)


def test_p1_traction(torch):
    from cloudfem_b200 import _faces
    m = O.box_mesh(2, 2, 3)
    trac = {"xmax": (0.0, None, lambda x, y, z: -1e6 * (1.0 + y)), "zmin": (3.0, 2.0, 1.0)}
    ref = np.zeros(3 * m.n_nodes)
    O._traction_p1(m, trac, ref)
    got, _ = _run(torch, m, _faces.P1, [(k, list(v)) for k, v in trac.items()], [], ncomp=3,
                  faces_of=O.boundary_faces_p1)
    _close(got, ref)


def test_tet10_neumann_time_dependent_and_robin(torch):
    from cloudfem_b200 import _faces
    from cloudfem_b200.fem.tet10 import _flux_at
    m = O.box_mesh_tet10(2, 2, 2)

    def qt(x, y, z, t):
        return (1.0 + x) * np.cos(3.0 * t) + y * z

    for t in (0.0, 0.3):
        ref = O.neumann_load_tet10(m, {"xmin": qt, "zmax": _q, "ymax": 4.0}, t)
        F, _ = _run(torch, m, _faces.T10,
                    [(name, [_flux_at(q, t)]) for name, q in
                     (("xmin", qt), ("zmax", _q), ("ymax", 4.0))], [],
                    faces_of=O.boundary_faces10)
        _close(F, ref)
    Kref, Fref = O.robin_terms_tet10(m, {"ymin": (_h, 20.0), "zmin": (25.0, _q)})
    F, K = _run(torch, m, _faces.T10, [], [("ymin", (_h, 20.0)), ("zmin", (25.0, _q))],
                faces_of=O.boundary_faces10)
    _close(F, Fref)
    _csr_close(K, Kref)


def test_tet10_traction(torch):
    from cloudfem_b200 import _faces
    nx, ny, nz, xl, yl, zl = C.TET10_BEAM
    m = O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)
    trac = {"xmax": (0.0, None, lambda x, y, z: -1e6 * (1.0 + z)), "ymin": (1.0, 2.0, 3.0)}
    _, r1 = O.assemble_elasticity_tet10(m, 210e9, 0.3, traction=trac)
    _, r0 = O.assemble_elasticity_tet10(m, 210e9, 0.3)
    got, _ = _run(torch, m, _faces.T10_TRACTION, [(k, list(v)) for k, v in trac.items()], [],
                  ncomp=3, faces_of=O.boundary_faces10)
    _close(got, r1 - r0)
