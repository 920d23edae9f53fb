"""Host logic of the dynamics module: the Newmark parameter sets, load
normalisation, the vectorised diagonal recurrences that step the modal
coordinates (against the reference's single-DOF history), the boundary
check and the history helpers. No GPU."""

import numpy as np
import pytest

import cases as C
from conftest import rel_err


def test_newmark_params():
    from cloudfem_b200.physics.dynamics3d import NEWMARK_METHODS, _newmark_params
    assert _newmark_params("average", None, None) == NEWMARK_METHODS["average"]
    assert _newmark_params("linear", None, None) == (1.0 / 6.0, 0.5)
    assert _newmark_params("bogus", 0.3, 0.6) == (0.3, 0.6)
    assert _newmark_params("average", None, 0.6) == (0.25, 0.6)
    with pytest.raises(ValueError, match="unknown method"):
        _newmark_params("bogus", None, None)
    with pytest.raises(ValueError, match="positive"):
        _newmark_params("average", 0.0, 0.5)


def test_force_fn_shapes():
    from cloudfem_b200.physics.dynamics3d import _as_force_fn
    assert not _as_force_fn(None, 4)(0.3).any()
    np.testing.assert_array_equal(_as_force_fn(np.arange(4.0), 4)(1.0), np.arange(4.0))
    assert _as_force_fn(lambda t: [t, 2 * t], 2)(0.5).tolist() == [0.5, 1.0]
    with pytest.raises(ValueError, match="shape"):
        _as_force_fn(np.zeros(3), 4)
    with pytest.raises(ValueError, match="returned shape"):
        _as_force_fn(lambda t: np.zeros(3), 4)(0.0)


def test_diagonal_recurrences_match_reference_sdof(golden):
    """The modal stepping (one scalar oscillator per entry) reproduces the
    reference's single-DOF history, and is exact per entry when vectorised."""
    from cloudfem_b200.physics.dynamics3d import _newmark_diagonal
    F = lambda t: np.array([np.sin(3 * t)])  # noqa: E731
    times, U, V, A = _newmark_diagonal(np.array([2.0]), np.array([0.3]), np.array([50.0]), F,
                                       2.0, 0.05, np.array([1.0]), np.array([0.0]), 0.25, 0.5)
    assert len(times) == 41 and times[-1] == 2.0
    assert rel_err(U.ravel(), golden["dyn_sdof_U"]) <= 1e-13
    assert rel_err(A.ravel(), golden["dyn_sdof_A"]) <= 1e-13
    # three independent oscillators at once == one at a time
    m, c, k = np.array([2.0, 1.0, 3.0]), np.array([0.3, 0.0, 1.0]), np.array([50.0, 4.0, 9.0])
    F3 = lambda t: np.array([np.sin(3 * t), 1.0, np.cos(t)])  # noqa: E731
    _, U3, _, _ = _newmark_diagonal(m, c, k, F3, 1.0, 0.1, np.ones(3), np.zeros(3), 1 / 6, 0.5)
    for j in range(3):
        _, Uj, _, _ = _newmark_diagonal(m[j:j + 1], c[j:j + 1], k[j:j + 1],
                                        lambda t, j=j: F3(t)[j:j + 1], 1.0, 0.1,
                                        np.ones(1), np.zeros(1), 1 / 6, 0.5)
        np.testing.assert_array_equal(U3[:, j], Uj[:, 0])


def test_diagonal_energy_conserved_average_acceleration():
    """Undamped, unloaded: the average-acceleration rule conserves
    k u^2 + m v^2 exactly (up to round-off)."""
    from cloudfem_b200.physics.dynamics3d import _newmark_diagonal
    m, k = np.array([1.0, 2.0]), np.array([100.0, 3.0])
    _, U, V, _ = _newmark_diagonal(m, np.zeros(2), k, lambda t: np.zeros(2), 5.0, 0.07,
                                   np.array([1.0, -0.5]), np.array([0.0, 2.0]), 0.25, 0.5)
    energy = k * U ** 2 + m * V ** 2
    assert np.abs(energy / energy[0] - 1.0).max() < 1e-12


def test_homogeneous_bc_check():
    from cloudfem_b200.mesh import box_mesh
    from cloudfem_b200.physics.dynamics3d import _check_homogeneous_bc
    m = box_mesh(2, 1, 1)
    _check_homogeneous_bc(m, None)
    _check_homogeneous_bc(m, {"xmin": (0.0, None, lambda x, y, z: 0.0)})
    with pytest.raises(ValueError, match="homogeneous"):
        _check_homogeneous_bc(m, {"xmin": (0.0, 1.0, None)})
    with pytest.raises(ValueError, match="homogeneous"):
        _check_homogeneous_bc(m, {"xmin": (lambda x, y, z: y, None, None)})


def test_fixed_dofs_and_history_helpers():
    from cloudfem_b200.mesh import box_mesh
    from cloudfem_b200.physics.dynamics3d import node_series, peak_response
    from cloudfem_b200.physics.modal3d import _fixed_dofs
    nx, ny, nz, xl, yl, zl = C.DYN_BOX
    m = box_mesh(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    xmin = np.asarray(m.boundaries["xmin"])
    fixed = _fixed_dofs(m, {"xmin": (0.0, None, 0.0)})
    np.testing.assert_array_equal(fixed, np.sort(np.concatenate([3 * xmin, 3 * xmin + 2])))
    H = np.zeros((4, 3 * m.n_nodes))
    H[2, 3 * 5 + 1] = -7.0
    H[1, 3 * 2] = 3.0
    np.testing.assert_array_equal(node_series(H, 5, 1), [0, 0, -7.0, 0])
    peak, t_peak, dof = peak_response(np.array([0.0, 0.1, 0.2, 0.3]), H)
    assert t_peak == 0.2 and dof == 16 and peak[6] == 3.0 and peak[16] == 7.0
