"""Host logic of the solve drivers (no GPU): precision modes and default
tolerances, the step count of the time marches (the reference's rounding,
tet_heat.py:234, tet10.py:504, em3d_tet10.py:557), and how solver statuses
become errors: nothing short of convergence is returned as a result."""

import pytest

pytest.importorskip("torch")   # the package imports torch for device buffers


def _result(status, iterations=7, relres=3.5e-6):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import SolveResult
    st = N.SolveStats()
    st.status, st.iterations, st.relres = status, iterations, relres
    return SolveResult(st)


def test_solver_mode_and_default_tolerances():
    from cloudfem_b200 import _native as N
    from cloudfem_b200._driver import solver_mode
    assert solver_mode("fp64", None) == (N.SOLVE_FP64, 1e-15)
    assert solver_mode("mixed", None) == (N.SOLVE_MIXED, 1e-10)
    assert solver_mode("mixed", 1e-8) == (N.SOLVE_MIXED, 1e-8)
    with pytest.raises(ValueError, match="unknown precision"):
        solver_mode("fp16", None)


@pytest.mark.parametrize("t_end, dt, want", [(1.0, 0.1, 10), (1.0, 0.3, 4), (0.3, 0.1, 3),
                                             (2.0, 0.05, 40), (1e-3, 1.0, 1)])
def test_step_count_follows_the_reference(t_end, dt, want):
    import numpy as np

    from cloudfem_b200._driver import n_steps_of
    assert n_steps_of(t_end, dt) == want == int(np.ceil(t_end / dt - 1e-12))


def test_step_count_rejects_non_positive_end():
    from cloudfem_b200._driver import n_steps_of
    with pytest.raises(ValueError, match="positive"):
        n_steps_of(0.0, 0.1)


def test_statuses_become_errors():
    from cloudfem_b200 import _native as N
    from cloudfem_b200._driver import accept
    accept(_result(N.CFEM_OK), 1e-10, "solve")
    with pytest.raises(RuntimeError, match=r"not converged.*7 iterations.*3\.500e-06") as e:
        accept(_result(N.CFEM_ERR_NOT_CONVERGED), 1e-10, "time step 3")
    assert "time step 3" in str(e.value) and "1.0e-10" in str(e.value)
    with pytest.raises(RuntimeError, match="singular or indefinite"):
        accept(_result(N.CFEM_ERR_BREAKDOWN), 1e-10, "solve")
    with pytest.raises(RuntimeError, match="timed out|timeout"):
        accept(_result(N.CFEM_ERR_TIMEOUT), 1e-10, "solve")
