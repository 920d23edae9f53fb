"""Failure detection on the device, in forms that cannot hurt the GPU.

* Non-finite input (a NaN conductivity injected on the host) is caught by
  the solver's finiteness checks and raised as RuntimeError.
* A solve that stops short of its target (iteration cap) raises
  RuntimeError; it is never returned as a result.
* The persistent scheduler's grid barrier has a bounded wait. With a short
  limit and one phantom block that never arrives (CFEM_PARAM_BARRIER_HOLD),
  every wait runs out: the launch returns, the host reads
  CFEM_ERR_TIMEOUT, and the same context then solves normally.
"""

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def test_nan_coefficient_raises(torch):
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(6, 6, 6)

    def k(x, y, z):
        x = np.asarray(x, dtype=float)
        return np.where(x > 0.9, np.nan, 1.0)

    with pytest.raises(RuntimeError, match="breakdown"):
        solve_tet_poisson(m, k=k, f=1.0, bc={"xmin": 0.0})


def test_iteration_cap_raises(torch):
    from cloudfem_b200.fem.tet10 import solve_tet10_poisson
    from cloudfem_b200.mesh import box_mesh_tet10
    m = box_mesh_tet10(6, 6, 6)
    with pytest.raises(RuntimeError, match="not converged"):
        solve_tet10_poisson(m, k=1.0, f=1.0, bc={s: 0.0 for s in C.FACES},
                            max_iter=5)


def test_grid_barrier_timeout_then_recovery(torch):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    rt = N.runtime()
    m = box_mesh(12, 12, 12)
    kw = dict(k=C.k_fn, f=C.f_fn, bc={"xmin": 0.0, "zmax": C.bc_fn})
    ref = solve_tet_poisson(m, **kw)
    old = (rt.lib.cfem_ctx_get_param(rt.ctx, N.PARAM_BARRIER_TIMEOUT_US),
           rt.lib.cfem_ctx_get_param(rt.ctx, N.PARAM_BARRIER_HOLD))
    assert old == (4000000, 0)
    N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_PERSISTENT))
    try:
        rt.set_param(N.PARAM_BARRIER_TIMEOUT_US, 20000)     # 20 ms
        rt.set_param(N.PARAM_BARRIER_HOLD, 1)
        with pytest.raises(N.CfemError) as info:
            solve_tet_poisson(m, **kw)
        assert info.value.status == N.CFEM_ERR_TIMEOUT
        rt.set_param(N.PARAM_BARRIER_HOLD, 0)
        rt.set_param(N.PARAM_BARRIER_TIMEOUT_US, old[0])
        u = solve_tet_poisson(m, **kw)
        assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()
    finally:
        rt.set_param(N.PARAM_BARRIER_HOLD, 0)
        rt.set_param(N.PARAM_BARRIER_TIMEOUT_US, old[0])
        N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_AUTO))
    with pytest.raises(ValueError):
        rt.set_param(N.PARAM_BARRIER_HOLD, 2)
    with pytest.raises(ValueError):
        rt.set_param(N.PARAM_BARRIER_TIMEOUT_US, 0)
    with pytest.raises(ValueError):
        rt.set_param(N.PARAM_SELL3_LANES, 8)   # slices must hold a chunk's rows
