"""Solver properties on the GPU: determinism, batch independence, error
reporting, and full-size checks through size-independent properties."""

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


def _poisson_system(torch, n, k=1.0, seed=0):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem, DeviceMesh, fixed_mask
    from cloudfem_b200.mesh import box_mesh_tet10
    m = box_mesh_tet10(n, n, n)
    dm = DeviceMesh(m)
    rng = np.random.default_rng(seed)
    kc = np.exp(rng.normal(0.0, 1.0, (n, n, n)))

    def kf(x, y, z):
        i = np.minimum((x * n).astype(int), n - 1)
        j = np.minimum((y * n).astype(int), n - 1)
        kk = np.minimum((z * n).astype(int), n - 1)
        return kc[i, j, kk]

    vals, rhs = dm.assemble(N.OP_T10_STIFF, coef=kf, load=1.0)
    bnd = np.unique(np.concatenate([m.boundaries[s] for s in C.FACES]))
    mask, x = fixed_mask(dm.rt, m.n_nodes, bnd, np.zeros(len(bnd)))
    pat = dm.pattern
    return dm, BlockSystem(dm.rt, m.n_nodes, 1, pat.row_ptr, pat.col, vals,
                           rhs, x, mask)


def test_batch_results_equal_solo_bitwise(torch):
    """Each system's answer is bitwise the same alone and in a batch."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import pcg
    for mode in (N.SOLVE_FP64, N.SOLVE_MIXED):
        built = [_poisson_system(torch, n, seed=n) for n in (3, 5, 4)]
        systems = [s for _, s in built]
        res_batch = pcg(systems, mode, rtol=1e-10)
        xb = [s.x.clone() for s in systems]
        for s in systems:
            s.x.zero_()
        for i, s in enumerate(systems):
            r = pcg([s], mode, rtol=1e-10)[0]
            assert r.status == 0
            assert r.iterations == res_batch[i].iterations
            assert torch.equal(s.x, xb[i]), f"system {i} differs (mode {mode})"


def test_repeat_is_bitwise_deterministic(torch):
    from cloudfem_b200.fem.tet_poisson import assemble, solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(12, 12, 12)
    A1, b1 = assemble(m, k=C.k_fn, f=C.f_fn)
    A2, b2 = assemble(m, k=C.k_fn, f=C.f_fn)
    assert np.array_equal(A1.data, A2.data) and np.array_equal(b1, b2)
    bc = {s: 0.0 for s in C.FACES}
    u1 = solve_tet_poisson(m, k=C.k_fn, f=C.f_fn, bc=bc)
    u2 = solve_tet_poisson(m, k=C.k_fn, f=C.f_fn, bc=bc)
    assert np.array_equal(u1, u2)


def test_p1_poisson_20cubed_accuracy(torch):
    """P1 20^3 manufactured problem: the discretisation error matches the
    reference's (L2 = 1.89e-3) and both precisions agree to 1e-8."""
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(20, 20, 20)
    bc = {s: 0.0 for s in C.FACES}
    u = solve_tet_poisson(m, k=1.0, f=C.f_sss, bc=bc)
    err = np.sqrt(np.mean((u - C.exact_sss(*m.nodes.T)) ** 2))
    assert abs(err - 1.89e-3) < 0.01e-3, err
    um = solve_tet_poisson(m, k=1.0, f=C.f_sss, bc=bc, precision="mixed",
                           rtol=1e-10)
    assert np.linalg.norm(um - u) / np.linalg.norm(u) <= 1e-8


def test_linear_field_is_exact(torch):
    """Affine exactness at a size where the oracle is slow (P1 and Tet10)."""
    from cloudfem_b200.fem.tet10 import solve_tet10_poisson
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh, box_mesh_tet10
    exact = lambda x, y, z: x + 2.0 * y + 3.0 * z - 1.0  # noqa: E731
    bc = {s: exact for s in C.FACES}
    m = box_mesh(16, 16, 16)
    u = solve_tet_poisson(m, f=0.0, bc=bc)
    assert np.abs(u - exact(*m.nodes.T)).max() < 1e-10
    m = box_mesh_tet10(8, 8, 8)
    u = solve_tet10_poisson(m, f=0.0, bc=bc)
    assert np.abs(u - exact(*m.nodes.T)).max() < 1e-10


def test_singular_system_reports_error(torch):
    """A pure-Neumann elasticity problem has rigid modes: the solve must
    fail loudly (no Dirichlet data), not return garbage."""
    from cloudfem_b200.mesh import box_mesh
    from cloudfem_b200.physics.elastic3d import solve_elasticity_3d
    m = box_mesh(3, 3, 3)
    with pytest.raises(RuntimeError):
        solve_elasticity_3d(m, 1e9, 0.3, bc=None,
                            traction={"xmax": (1e5, 0.0, 0.0)}, max_iter=200)


def test_bad_connectivity_is_rejected(torch):
    from cloudfem_b200.device import DeviceMesh
    from cloudfem_b200.mesh import TetMesh
    m = TetMesh(np.zeros((4, 3)), np.array([[0, 1, 2, 9]]))
    with pytest.raises(ValueError):
        DeviceMesh(m)


def test_pool_trim_keeps_results(torch):
    """Handing the library pool's memory back to the driver between solves
    changes nothing in the next solve."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    m = box_mesh(10, 9, 8)
    bc = {s: 0.0 for s in C.FACES}
    u1 = solve_tet_poisson(m, k=1.0, f=1.0, bc=bc)
    rt = N.runtime()
    assert rt.trim(0) >= 0
    u2 = solve_tet_poisson(m, k=1.0, f=1.0, bc=bc)
    assert np.array_equal(u1, u2)


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("bs", [1, 3])
def test_graph_scheduler_matches_persistent(torch, bs, mode):
    """The two schedulers (one persistent launch; graphs of per-phase
    launches with their own SpMV kernels) solve the same system to the same
    answer, for scalar and 3x3-block rows, in both precisions."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem, DeviceMesh, fixed_mask, pcg
    from cloudfem_b200.mesh import box_mesh_tet10
    if bs == 1:
        dm, sysm = _poisson_system(torch, 7, seed=3)
        mask, x0 = sysm.fixed, sysm.x.clone()
        make = lambda x: BlockSystem(dm.rt, dm.n_nodes, 1, dm.pattern.row_ptr,  # noqa: E731
                                     dm.pattern.col, sysm.vals64, sysm.b, x, mask)
    else:
        m = box_mesh_tet10(12, 3, 3, xlim=(0, 2), ylim=(0, .5), zlim=(0, .5))
        dm = DeviceMesh(m)
        vals, rhs = dm.assemble_elastic(N.OP_T10_ELAST, 210e9, 0.3,
                                        body=(0.0, 0.0, -7.8e4))
        idx = np.concatenate([3 * m.boundaries["xmin"] + c for c in range(3)])
        mask, x0 = fixed_mask(dm.rt, 3 * m.n_nodes, idx, np.zeros(len(idx)))
        make = lambda x: BlockSystem(dm.rt, dm.n_nodes, 3, dm.pattern.row_ptr,  # noqa: E731
                                     dm.pattern.col, vals, rhs, x, mask)
    md = N.SOLVE_FP64 if mode == "fp64" else N.SOLVE_MIXED
    rtol = 1e-12 if mode == "fp64" else 1e-10
    out = {}
    try:
        for sched in (N.SCHED_PERSISTENT, N.SCHED_GRAPH, N.SCHED_GRAPH_POLLED):
            N.check(dm.rt.lib.cfem_ctx_set_scheduler(dm.rt.ctx, sched))
            x = x0.clone()
            r = pcg([make(x)], md, rtol, 20000)[0]
            assert r.status == N.CFEM_OK, r
            out[sched] = x.cpu().numpy()
    finally:
        N.check(dm.rt.lib.cfem_ctx_set_scheduler(dm.rt.ctx, N.SCHED_AUTO))
    a = out[N.SCHED_PERSISTENT]
    tol = 1e-10 if mode == "fp64" else 1e-8
    for sched in (N.SCHED_GRAPH, N.SCHED_GRAPH_POLLED):
        b = out[sched]
        assert np.linalg.norm(a - b) / np.linalg.norm(a) <= tol
    # device-looped and host-polled graphs run the same kernels in order
    assert np.array_equal(out[N.SCHED_GRAPH], out[N.SCHED_GRAPH_POLLED])


def test_plan_repeated_solves_match_one_shot(torch):
    """A solve plan reused for several right-hand sides gives, each time,
    bitwise the answer of a one-shot solve of the same system."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import PcgPlan, pcg
    dm, sysm = _poisson_system(torch, 6, seed=5)
    x0 = sysm.x.clone()
    b0 = sysm.b.clone()
    for sched in (N.SCHED_PERSISTENT, N.SCHED_GRAPH, N.SCHED_GRAPH_POLLED):
        N.check(dm.rt.lib.cfem_ctx_set_scheduler(dm.rt.ctx, sched))
        try:
            plan = PcgPlan([sysm], N.SOLVE_MIXED, 1e-10, 5000)
            for scale in (1.0, -2.5, 0.75):
                sysm.b.copy_(b0 * scale)
                sysm.x.copy_(x0)
                r1 = plan.solve()[0]
                x_plan = sysm.x.clone()
                sysm.x.copy_(x0)
                r2 = pcg([sysm], N.SOLVE_MIXED, 1e-10, 5000)[0]
                assert r1.status == N.CFEM_OK and r2.status == N.CFEM_OK
                assert r1.iterations == r2.iterations
                assert torch.equal(x_plan, sysm.x)
            plan.close()
        finally:
            N.check(dm.rt.lib.cfem_ctx_set_scheduler(dm.rt.ctx, N.SCHED_AUTO))
