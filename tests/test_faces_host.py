"""Host parts of the boundary-face integrals (no GPU): the quadrature rules
the device kernels take against the oracle's tables (themselves pinned to
the reference), the Robin mass tables, the time-dependence detection of
flux functions (tet10.py:366-381) and the host scatter helper."""

import numpy as np
import pytest

from oracle import cfem_oracle as O

pytest.importorskip("torch")   # the package imports torch for device buffers


def test_rules_match_the_oracle_tables():
    from cloudfem_b200 import _faces as Fc
    np.testing.assert_array_equal(Fc.TRI_L6, O.TRI_L6)
    np.testing.assert_array_equal(Fc.TRI_W6, O.TRI_W6)
    np.testing.assert_array_equal(Fc.TRI_L3, O.TRI_L3)
    np.testing.assert_array_equal(Fc.TRI_W3, O.TRI_W3)
    np.testing.assert_allclose(Fc.face_shape6(O.TRI_L6), O.face_shape6(O.TRI_L6), rtol=0, atol=1e-15)
    # the 6-node shape functions interpolate: partition of unity, nodal values
    assert np.abs(Fc.FACE_N6.sum(axis=1) - 1.0).max() < 1e-14
    corners_mids = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1],
                             [.5, .5, 0], [0, .5, .5], [.5, 0, .5]])
    np.testing.assert_allclose(Fc.face_shape6(corners_mids), np.eye(6), atol=1e-15)


def test_robin_mass_tables():
    """P1: the exact face mass (1 + d_ij) / 12 per unit area; Tet10: the
    Dunavant-6 tables sum to the exact quadratic-triangle mass (degree 4 is
    integrated exactly)."""
    from cloudfem_b200 import _faces as Fc
    np.testing.assert_allclose(Fc.P1.mt[0].sum(), 1.0, rtol=1e-15)
    m6 = np.einsum("q,qab->ab", Fc.T10.w, Fc.T10.mt)
    # exact mass of the 6-node triangle (unit area): corners 6/180, mids 32/180,
    # corner-corner -1/180, corner-opposite-mid -4/180, others 0, mid-mid 16/180
    exact = np.array([[6, -1, -1, 0, -4, 0], [-1, 6, -1, 0, 0, -4], [-1, -1, 6, -4, 0, 0],
                      [0, 0, -4, 32, 16, 16], [-4, 0, 0, 16, 32, 16], [0, -4, 0, 16, 16, 32]],
                     float) / 180.0
    np.testing.assert_allclose(m6, exact, atol=1e-13)
    assert Fc.T10_TRACTION.mt is None and Fc.T10_TRACTION.nq == 3


def test_flux_function_time_dependence():
    from cloudfem_b200._faces import flux_fn
    f, td = flux_fn(2.5)
    assert not td and f(0, 0, 0, 9.0) == 2.5
    f, td = flux_fn(lambda x, y, z: x + y)
    assert not td and f(1.0, 2.0, 0.0, 7.0) == 3.0
    f, td = flux_fn(lambda x, y, z, t: t * x)
    assert td and f(2.0, 0.0, 0.0, 3.0) == 6.0


def test_add_at_sums_repeats_like_numpy():
    from cloudfem_b200._faces import add_at
    rng = np.random.default_rng(1)
    idx = rng.integers(0, 7, 50)
    vals = rng.random(50)
    F, G = np.zeros(7), np.zeros(7)
    add_at(F, idx, vals)
    np.add.at(G, idx, vals)
    np.testing.assert_allclose(F, G, rtol=1e-14)
    Fc, Gc = np.zeros(7, complex), np.zeros(7, complex)
    add_at(Fc, idx, vals * (1 + 2j))
    np.add.at(Gc, idx, vals * (1 + 2j))
    np.testing.assert_allclose(Fc, Gc, rtol=1e-14)
