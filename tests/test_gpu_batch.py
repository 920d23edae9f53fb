"""Batched assembly and solve (many independent meshes per launch)."""

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


def _problems():
    from cloudfem_b200.batch import HeatProblem
    from cloudfem_b200.mesh import box_mesh, box_mesh_tet10
    rng = np.random.default_rng(3)
    m10a = box_mesh_tet10(3, 3, 3)
    m10b = box_mesh_tet10(4, 3, 2)
    m4 = box_mesh(6, 5, 4)
    bc = {s: 0.0 for s in C.FACES}
    out = []
    for m in (m10a, m10b, m10a, m4, m4, m10b):
        k = np.exp(rng.normal(0.0, 1.0, m.n_elements))
        out.append(HeatProblem(m, k=k, f=1.0, bc=bc))
    out.append(HeatProblem(m10a, k=C.k_fn, f=C.f_fn, bc={"xmin": C.bc_fn}))
    out.append(HeatProblem(m4, k=2.0, f=C.f_fn, bc={"zmax": 1.0, "ymin": 0.0}))
    return out


def test_batched_assembly_equals_single(torch):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.batch import BatchSolver
    probs = _problems()
    solver = BatchSolver()
    batch = solver.prepare(probs)
    batch.assemble()
    for pb, it in zip(probs, batch.items):
        dm = it["dm"]
        op = N.OP_T10_STIFF if dm.npe == 10 else N.OP_P1_STIFF
        k = pb.k
        if isinstance(k, np.ndarray):
            from cloudfem_b200.device import DeviceMesh  # noqa: F401
            where_vals = torch.from_numpy(k).to(dm.rt.device)
            coef = N.Coef(N.ptr(where_vals), 0.0, N.COEF_ELEM, 0)
            vals = torch.empty(dm.pattern.nnz, dtype=torch.float64, device=dm.rt.device)
            lc, keep = dm.coef(pb.f, "qp" if dm.npe == 10 else "centroid")
            rhs = torch.empty(dm.n_nodes, dtype=torch.float64, device=dm.rt.device)
            import ctypes
            N.check(dm.rt.lib.cfem_assemble(
                dm.rt.ctx, dm.pattern.handle, op, N.ptr(dm.nodes), N.ptr(dm.elems),
                ctypes.byref(coef), ctypes.byref(lc), N.ptr(vals), N.ptr(rhs), 0,
                dm.rt.stream()))
        else:
            vals, rhs = dm.assemble(op, coef=pb.k, load=pb.f)
        assert torch.equal(vals, it["vals"])
        assert torch.equal(rhs, it["rhs"])


def test_batched_solve_matches_single_solves(torch):
    from cloudfem_b200.batch import solve_batch
    from cloudfem_b200.fem.tet10 import solve_tet10_poisson
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    probs = _problems()
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-8)):
        us = solve_batch(probs, precision=precision, rtol=1e-12 if precision == "fp64" else 1e-10)
        for pb, u in zip(probs, us):
            k = pb.k
            if isinstance(k, np.ndarray):
                # per-element values as a callable on the element index via
                # centroid lookup is not needed: compare with the same batch
                # machinery in FP64 instead
                continue
            solve = solve_tet10_poisson if pb.mesh.elements.shape[1] == 10 else solve_tet_poisson
            ref = solve(pb.mesh, k=pb.k, f=pb.f, bc=pb.bc)
            err = np.abs(u - ref).max() / np.abs(ref).max()
            assert err <= tol, (precision, err)
    u64 = solve_batch(probs, precision="fp64", rtol=1e-12)
    u32 = solve_batch(probs, precision="mixed", rtol=1e-10)
    for a, b in zip(u64, u32):
        assert np.abs(a - b).max() <= 1e-8 * np.abs(a).max()


def test_batch_result_same_alone_and_in_mix(torch):
    """Each problem's answer alone equals its answer inside the batch (the
    per-system reduction tree does not depend on the other systems)."""
    from cloudfem_b200.batch import solve_batch
    probs = _problems()
    mix = solve_batch(probs, precision="mixed", rtol=1e-10)
    for i in (0, 3, 6):
        alone = solve_batch([probs[i]], precision="mixed", rtol=1e-10)[0]
        assert np.abs(alone - mix[i]).max() <= 1e-9 * np.abs(mix[i]).max()


def test_autotuned_batch_gives_identical_results(tmp_path, monkeypatch):
    """Launch-parameter choices change block shapes and loop bodies, never
    the arithmetic: a batch solved after tuning is bitwise the same."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from cloudfem_b200 import _native as N
    from cloudfem_b200 import autotune
    from cloudfem_b200.batch import BatchSolver, HeatProblem
    from cloudfem_b200.mesh import box_mesh, box_mesh_tet10
    monkeypatch.setenv("CLOUDFEM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    bc = {s: 0.0 for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    rng = np.random.default_rng(2)
    meshes = [box_mesh_tet10(5, 4, 4), box_mesh(9, 8, 7), box_mesh_tet10(3, 3, 3)]
    probs = [HeatProblem(m, k=rng.lognormal(0, 1, len(m.elements)), f=1.0, bc=bc)
             for m in meshes]
    solver = BatchSolver()
    rt = solver.rt
    try:
        N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_GRAPH))
        batch = solver.prepare(probs)
        batch.assemble()
        batch.solve("mixed", rtol=1e-10)
        before = [x.copy() for x in batch.solutions()]
        out = autotune.tune_batch(batch, "mixed", 1e-10, repeat=1)
        assert out["assembly"]["best"]["t10_elements_per_block"] in autotune.T10_WARPS
        assert out["solve"]["best"]["iterations_per_loop_body"] in autotune.GRAPH_ITERS
        batch.assemble()
        batch.solve("mixed", rtol=1e-10)
        for a, b in zip(before, batch.solutions()):
            assert np.array_equal(a, b)
    finally:
        for p, v in ((N.PARAM_T10_WARPS, 4), (N.PARAM_P1_THREADS, 128),
                     (N.PARAM_GRAPH_ITERS, 2)):
            rt.set_param(p, v)
        N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_AUTO))


def test_mixed_matrix_batch_equals_per_system(torch):
    """cfem_mixed_matrix_batch (one launch per block size over many systems)
    writes bitwise the FP32 operators that cfem_mixed_matrix writes one
    system at a time, for scalar and 3x3 systems in one call."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import DeviceMesh, ptr
    from cloudfem_b200.mesh import box_mesh, box_mesh_tet10
    rt = N.runtime()
    systems = []
    for m, op, bs in ((box_mesh(5, 4, 3), N.OP_P1_STIFF, 1),
                      (box_mesh_tet10(3, 2, 2), N.OP_T10_STIFF, 1),
                      (box_mesh(4, 3, 3), N.OP_P1_ELAST, 3)):
        dm = DeviceMesh(m)
        if bs == 1:
            vals, _ = dm.assemble(op, coef=lambda x, y, z: 1.0 + x * y)
        else:
            vals, _ = dm.assemble_elastic(op, 210e9, 0.3)
        systems.append((dm, vals, bs))
    jobs = (N.MixedJob * len(systems))()
    outs = []
    for i, (dm, vals, bs) in enumerate(systems):
        v32 = torch.full((vals.numel(),), float("nan"), dtype=torch.float32, device="cuda")
        outs.append(v32)
        jobs[i] = N.MixedJob(dm.n_nodes, bs, 0, dm.pattern.row_ptr, dm.pattern.col, ptr(vals),
                             ptr(v32))
    N.check(rt.lib.cfem_mixed_matrix_batch(rt.ctx, jobs, len(systems), rt.stream()))
    for (dm, vals, bs), got in zip(systems, outs):
        ref = torch.empty_like(got)
        N.check(rt.lib.cfem_mixed_matrix(rt.ctx, dm.n_nodes, bs, dm.pattern.row_ptr,
                                         dm.pattern.col, ptr(vals), ptr(ref), rt.stream()))
        assert torch.equal(got, ref)
