"""The allocation-free solver entry point against the allocating one.

cfem_pcg_solve_noalloc exists for callers that cannot allocate device
memory while solving (an application that has reserved the whole HBM
budget for its own pools, or a latency-bound loop that cannot take
cudaMalloc's implicit synchronisation); its workspace is a fixed device
array inside libcfem. Here it is called through the C ABI twice in a row on
the same systems and must reproduce cfem_pcg_solve's solution within the
suite's solution tolerance each time (the array keeps the previous call's
contents, so the second call checks that it is cleared). This file is
collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu

SOL_RTOL = 1e-10
MIXED_RTOL = 1e-8


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _elastic_system(torch):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import (BlockSystem, DeviceMesh, fixed_mask,
                                      fixed_vector)
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics.elastic3d import _assemble
    m = box_mesh_tet10(12, 2, 2, xlim=(0, 0.6), ylim=(0, 0.1), zlim=(0, 0.1))
    dm = DeviceMesh(m)
    vals, rhs = _assemble(dm, m, N.OP_T10_ELAST, 210e9, 0.3, None,
                          {"xmax": (0.0, 0.0, -1e6)}, None, 0.0, 0.0, True)
    idx, v = fixed_vector(m, {"xmin": (0.0, 0.0, 0.0)})

    def make():
        mask, x = fixed_mask(dm.rt, 3 * m.n_nodes, idx, v)
        pat = dm.pattern
        return BlockSystem(dm.rt, m.n_nodes, 3, pat.row_ptr, pat.col, vals,
                           rhs, x, mask, keep=(dm,))
    return make


def _heat_system(torch):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import (BlockSystem, DeviceMesh, fixed_mask,
                                      fixed_scalar)
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(10, 9, 8)
    dm = DeviceMesh(m)
    vals, rhs = dm.assemble(N.OP_P1_STIFF, coef=C.k_fn, load=C.f_fn)
    idx, v = fixed_scalar(m, {"xmin": 0.0, "zmax": C.bc_fn})

    def make():
        mask, x = fixed_mask(dm.rt, m.n_nodes, idx, v)
        pat = dm.pattern
        return BlockSystem(dm.rt, m.n_nodes, 1, pat.row_ptr, pat.col, vals,
                           rhs, x, mask, keep=(dm,))
    return make


def _big_heat_system(torch):
    """P1 box 50^3 (132,651 rows, 8,291 row chunks): more chunks than one
    resident wave of the persistent kernel has warps, so every warp loops
    over several chunks per phase."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import (BlockSystem, DeviceMesh, fixed_mask,
                                      fixed_scalar)
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(50, 50, 50)
    dm = DeviceMesh(m)
    vals, rhs = dm.assemble(N.OP_P1_STIFF, coef=C.k_fn, load=C.f_fn)
    idx, v = fixed_scalar(m, {"xmin": 0.0, "zmax": C.bc_fn})

    def make():
        mask, x = fixed_mask(dm.rt, m.n_nodes, idx, v)
        pat = dm.pattern
        return BlockSystem(dm.rt, m.n_nodes, 1, pat.row_ptr, pat.col, vals,
                           rhs, x, mask, keep=(dm,))
    return make


def _pool_reserved(rt, keep):
    """Bytes the library's device pool holds after trimming it to `keep`.
    The pool keeps what it frees (release threshold unlimited), so with
    keep = 2^64 - 1 any allocation made since the last trim shows up here."""
    from cloudfem_b200 import _native as N
    v = ctypes.c_uint64()
    N.check(rt.lib.cfem_ctx_trim(rt.ctx, ctypes.c_uint64(keep), ctypes.byref(v)))
    return v.value


def _call_noalloc(system, mode, rtol):
    """One call of cfem_pcg_solve_noalloc through the C ABI."""
    from cloudfem_b200 import _native as N
    rt = system.rt
    ls = system.linsys(mode, rtol, 20000)
    st = N.SolveStats()
    N.check(rt.lib.cfem_pcg_solve_noalloc(rt.ctx, ctypes.byref(ls),
                                          ctypes.byref(st), rt.stream()))
    return st


@pytest.mark.parametrize("kind", ["elastic", "heat"])
@pytest.mark.parametrize("mode_name", ["fp64", "mixed"])
def test_noalloc_matches_allocating_solver(torch, kind, mode_name):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import pcg
    mode = N.SOLVE_FP64 if mode_name == "fp64" else N.SOLVE_MIXED
    rtol = 1e-12 if mode_name == "fp64" else 1e-10
    make = _elastic_system(torch) if kind == "elastic" else _heat_system(torch)
    ref = make()
    r = pcg([ref], mode, rtol=rtol, max_iter=20000)[0]
    assert r.status == 0, r
    x_ref = ref.x.cpu().numpy()
    systems = [make() for _ in range(2)]
    for sys_ in systems:
        sys_.vals32 = ref.vals32          # same FP32 operator, made once
    rt = ref.rt
    before = _pool_reserved(rt, 0)
    for call, sys_ in enumerate(systems):
        st = _call_noalloc(sys_, mode, rtol)
        assert st.status == 0, f"call {call}: status {st.status}"
        x = sys_.x.cpu().numpy()
        err = np.abs(x - x_ref).max() / np.abs(x_ref).max()
        assert err <= SOL_RTOL, f"call {call}: rel diff {err:.3e}"
        assert st.iterations == r.iterations
    assert _pool_reserved(rt, 2 ** 64 - 1) == before, "the library allocated"


@pytest.mark.parametrize("mode_name", ["fp64", "mixed"])
def test_noalloc_strided_grid_matches_allocating_solver(torch, mode_name):
    """A system with many more row chunks than the persistent grid has warps
    (each warp strides over several chunks per phase) against cfem_pcg_solve
    on the persistent scheduler (same kernels: same iterations, bitwise the
    same solution) and on its default scheduler (within the tolerance)."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import pcg
    mode = N.SOLVE_FP64 if mode_name == "fp64" else N.SOLVE_MIXED
    rtol = 1e-12 if mode_name == "fp64" else 1e-10
    make = _big_heat_system(torch)
    auto = make()
    r_auto = pcg([auto], mode, rtol=rtol, max_iter=20000)[0]
    assert r_auto.status == 0, r_auto
    rt = auto.rt
    pers = make()
    pers.vals32 = auto.vals32
    N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_PERSISTENT))
    try:
        r_pers = pcg([pers], mode, rtol=rtol, max_iter=20000)[0]
    finally:
        N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_AUTO))
    assert r_pers.status == 0, r_pers
    x_pers = pers.x.cpu().numpy()
    x_auto = auto.x.cpu().numpy()
    systems = [make() for _ in range(2)]
    for sys_ in systems:
        sys_.vals32 = auto.vals32
    before = _pool_reserved(rt, 0)
    for call, sys_ in enumerate(systems):
        st = _call_noalloc(sys_, mode, rtol)
        assert st.status == 0, f"call {call}: status {st.status}"
        x = sys_.x.cpu().numpy()
        assert st.iterations == r_pers.iterations
        assert np.array_equal(x, x_pers), f"call {call}"
        # another scheduler sums in another order: the suite's tolerance
        # for the precision (FP64 1e-10, mixed 1e-8)
        tol = SOL_RTOL if mode_name == "fp64" else MIXED_RTOL
        err = np.abs(x - x_auto).max() / np.abs(x_auto).max()
        assert err <= tol, f"call {call}: rel diff {err:.3e}"
    assert _pool_reserved(rt, 2 ** 64 - 1) == before, "the library allocated"


def test_noalloc_rejects_systems_beyond_capacity(torch):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem
    rt = N.runtime()
    cap = int(rt.lib.cfem_pcg_noalloc_capacity())
    assert cap == 32 << 20
    n = cap // 8          # more FP64 vector bytes than the whole array
    dev = rt.device
    rp = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    col = torch.zeros(1, dtype=torch.int32, device=dev)
    v = torch.zeros(1, dtype=torch.float64, device=dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    big = BlockSystem(rt, n, 1, rp, col, v, b, x)
    with pytest.raises(ValueError, match="scratch"):
        _call_noalloc(big, N.SOLVE_FP64, 1e-8)
