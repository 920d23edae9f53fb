"""Host post-processing of the A-V phasor field against the reference's
golden values (computed by the reference on its own SuperLU solution of the
phasor golden case): centroid flux density, exact Joule power and its
per-element density, the source's complex power, and the B-H model curve."""

import numpy as np
import pytest

import cases as C
from conftest import assert_close


def test_phasor_postprocessing_matches_reference(golden):
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics import em3d_tet10 as em
    m = box_mesh_tet10(C.AVP_N, C.AVP_N, C.AVP_N)
    a, v = golden["avp_a"], golden["avp_v"]
    assert_close(em.element_flux_density_tet10(m, a), golden["avp_B"], 1e-12, "B")
    P, Q = em.total_joule_power_tet10(m, a, v, C.AVP_SIGMA, C.AVP_OMEGA)
    assert abs(P - float(golden["avp_P"])) <= 1e-12 * abs(float(golden["avp_P"]))
    assert_close(Q, golden["avp_Q"], 1e-12, "Q")
    S = em.source_complex_power_tet10(m, a, v, C.avp_js, C.AVP_OMEGA)
    Sg = complex(golden["avp_S"])
    assert abs(S - Sg) <= 1e-12 * abs(Sg)


def test_joule_power_without_conductor_is_zero():
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics import em3d_tet10 as em
    m = box_mesh_tet10(2, 2, 2)
    a = np.ones(3 * m.n_nodes, dtype=complex)
    P, Q = em.total_joule_power_tet10(m, a, np.zeros(m.n_nodes), 0.0, 1.0)
    assert P == 0.0 and not Q.any()


def test_bh_curve_matches_reference(golden):
    from cloudfem_b200.physics import em3d_tet10 as em
    assert_close(em.bh_secant_mu_r(C.BH_H), golden["bh_mu_r"], 1e-15, "mu_r")
    assert_close(em.bh_secant_mu_r(C.BH_H, bsat=1.2, mu_mag0=50.0),
                 golden["bh_mu_r_soft"], 1e-15, "mu_r soft")
    assert np.array_equal(em.bh_secant_mu_r(C.BH_H, mu_mag0=0.0), np.ones(len(C.BH_H)))


def test_induction_material_laws_match_reference(golden):
    from cloudfem_b200.physics import induction3d_tet10 as ind
    Tt = 20.0 + 900.0 * np.linspace(0.0, 1.0, 9)
    assert_close(ind.steel_sigma_T(Tt), golden["law_sigma"], 1e-15, "sigma(T)")
    assert_close(ind.curie_step_T(Tt), golden["law_step"], 1e-15, "Curie step")
    assert_close(ind.bh_secant_mu_r_HT(C.BH_H, Tt), golden["law_mu_HT"], 1e-15, "mu_r(H, T)")
    assert_close(ind.steel_cp_T(Tt, cp_slope=1e-3, cp_peak_h=2e6), golden["law_cp"], 1e-15, "cp(T)")
    assert_close(ind.steel_enthalpy_T(Tt, cp_slope=1e-3, cp_peak_h=2e6), golden["law_H"],
                 1e-14, "H(T)")


def test_centroid_lookup_scalar_and_array():
    """The nearest-centroid coefficient of the induction chain
    (induction3d_tet10.py:216-230) answers scalars with floats and arrays
    element-wise (so device assembly samples it in one call)."""
    pytest.importorskip("torch")
    from cloudfem_b200.physics.induction3d_tet10 import _centroid_lookup
    cen = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.0, 1.0, 0.0]])
    fn = _centroid_lookup(cen, [3.0, 5.0, 7.0])
    assert fn(0.1, 0.0, 0.0) == 3.0 and isinstance(fn(0.1, 0.0, 0.0), float)
    got = fn(np.array([0.9, 0.1, 0.0]), np.array([1.0, 0.0, 0.9]), np.array([1.0, 0.0, 0.1]))
    np.testing.assert_array_equal(got, [5.0, 3.0, 7.0])
