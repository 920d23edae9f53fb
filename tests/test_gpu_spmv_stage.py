"""SpMV of the graph scheduler with the matrix streamed through
shared-memory windows by 1-D bulk copies (staging 1: scalar rows; 2: also
3x3 blocks) or in the sliced-ELL layout (staging 3: scalar rows, one row
per lane, slices of 32 length-sorted rows; 3x3 block rows over 1, 2 or 4
lanes each, slices of 32, 16 or 8 block rows) against the register path
(staging 0) and a direct FP64 solve:
the same answers, bitwise batch independence, rows longer than a window,
short (P1-like, 4 lanes per row) and long (8 lanes) rows, 3x3 rows that
straddle windows, and CSR arrays that do not start on a 16-byte
boundary."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _hub_matrix(n, hub_degrees, seed):
    """SPD scalar matrix: a chain Laplacian plus hub nodes each coupled to
    `deg` random nodes (rows from a few entries up to far longer than a
    staging window), made strictly diagonally dominant."""
    rng = np.random.default_rng(seed)
    r = list(range(n - 1))
    c = list(range(1, n))
    w = list(-rng.uniform(0.5, 1.5, n - 1))
    hubs = rng.choice(n, size=len(hub_degrees), replace=False)
    for h, deg in zip(hubs, hub_degrees):
        others = rng.choice(np.setdiff1d(np.arange(n), [h]), size=deg, replace=False)
        r += [int(h)] * deg
        c += [int(o) for o in others]
        w += list(-rng.uniform(0.1, 1.0, deg))
    off = sp.coo_matrix((w, (r, c)), shape=(n, n)).tocsr()
    off = off + off.T
    diag = np.asarray(abs(off).sum(axis=1)).ravel() + rng.uniform(0.5, 2.0, n)
    A = (off + sp.diags(diag)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A


def _dense_band(n, half, seed):
    """SPD banded matrix with `2 half + 1` entries per interior row (rows of
    about 29 entries: the 8-lanes-per-row kernel)."""
    rng = np.random.default_rng(seed)
    diags = [-rng.uniform(0.1, 1.0, n - k) for k in range(1, half + 1)]
    off = sp.diags(diags, list(range(1, half + 1)), shape=(n, n))
    off = (off + off.T).tocsr()
    d = np.asarray(abs(off).sum(axis=1)).ravel() + rng.uniform(0.5, 2.0, n)
    A = (off + sp.diags(d)).tocsr()
    A.sort_indices()
    return A


def _offset_copy(torch, arr, dtype, offset):
    """Device copy of arr starting `offset` elements into a larger buffer
    (so the data does not start on a 16-byte boundary when offset > 0)."""
    buf = torch.zeros(arr.size + offset + 4, dtype=dtype, device="cuda")
    buf[offset:offset + arr.size] = torch.as_tensor(arr, dtype=dtype, device="cuda")
    return buf[offset:offset + arr.size]


def _system(torch, rt, A, b, offset):
    from cloudfem_b200.device import BlockSystem
    n = A.shape[0]
    rp = torch.as_tensor(A.indptr.astype(np.int32), device="cuda")
    col = _offset_copy(torch, A.indices.astype(np.int32), torch.int32, offset)
    v64 = _offset_copy(torch, A.data, torch.float64, offset)
    bb = torch.as_tensor(b, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    s = BlockSystem(rt, n, 1, rp, col, v64, bb, x)
    if offset:
        v32 = s.ensure_fp32()
        s.vals32 = _offset_copy(torch, v32.cpu().numpy(), torch.float32, offset)
    return s


def _solve(rt, systems, mode, rtol, stage, sort=1, lanes=4, staged=0):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import pcg
    N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_GRAPH))
    before = rt.get_param(N.PARAM_SPMV_STAGE)
    lanes_before = rt.get_param(N.PARAM_SELL3_LANES)
    staged_before = rt.get_param(N.PARAM_SELL3_STAGED)
    try:
        rt.set_param(N.PARAM_SPMV_STAGE, stage)
        rt.set_param(N.PARAM_SELL_SORT, sort)
        rt.set_param(N.PARAM_SELL3_LANES, lanes)
        rt.set_param(N.PARAM_SELL3_STAGED, staged)
        for s in systems:
            s.x.zero_()
        res = pcg(systems, mode, rtol, 20000)
    finally:
        rt.set_param(N.PARAM_SPMV_STAGE, before)
        rt.set_param(N.PARAM_SELL_SORT, 1)
        rt.set_param(N.PARAM_SELL3_LANES, lanes_before)
        rt.set_param(N.PARAM_SELL3_STAGED, staged_before)
        N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, N.SCHED_AUTO))
    for r in res:
        assert r.status == N.CFEM_OK, r
    return res, [s.x.cpu().numpy() for s in systems]


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_staged_spmv_matches_direct_solve(torch, mode):
    """Hub rows of 200, 400 and 1,500 entries (the last two longer than the
    FP64 window, the last longer than every window) in short-row and
    banded (~29 entries per row) matrices, arrays at 4-, 8- and 12-byte
    offsets: both stagings give the direct solve's answer and agree with
    each other."""
    from cloudfem_b200 import _native as N
    rt = N.runtime()
    md = N.SOLVE_FP64 if mode == "fp64" else N.SOLVE_MIXED
    rtol = 1e-12 if mode == "fp64" else 1e-10
    tol = 1e-9 if mode == "fp64" else 1e-7   # condition number ~1e3
    cases = [(_hub_matrix(3000 + 7 * off, [200, 400, 1500], seed=off), off)
             for off in (0, 1, 3)]
    cases.append((_dense_band(3000, 14, 5) + _hub_matrix(3000, [400, 1500], 6), 1))
    for A, offset in cases:
        b = np.random.default_rng(10 + offset).normal(size=A.shape[0])
        ref = spla.spsolve(A.tocsc(), b)
        sys_ = _system(torch, rt, A, b, offset)
        xs = {}
        for stage, sort in ((0, 1), (1, 1), (3, 1), (3, 0)):
            _, (x,) = _solve(rt, [sys_], md, rtol, stage, sort)
            err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
            assert err <= tol, (offset, stage, sort, err)
            xs[stage] = x
        for stage in (1, 3):
            d = np.linalg.norm(xs[stage] - xs[0]) / np.linalg.norm(xs[0])
            assert d <= tol, (offset, stage, d)


@pytest.mark.parametrize("stage", [1, 3])
@pytest.mark.parametrize("rows", ["long", "short"])
def test_staged_spmv_batch_equals_solo_bitwise(torch, rows, stage):
    """On the graph scheduler with staged (1) or sliced-ELL (3) SpMV, each
    system's answer is bitwise the same alone, in a batch, and on a repeat,
    with 8 lanes per row (mean row above 16 entries) and with 4."""
    from cloudfem_b200 import _native as N
    rt = N.runtime()
    if rows == "long":
        mats = [_dense_band(n, 14, seed=n) for n in (2500, 1800, 4100)]
        mats[0] = mats[0] + _hub_matrix(2500, [600], seed=1)
    else:
        mats = [_hub_matrix(n, degs, seed=n) for n, degs in
                ((2500, [600]), (1800, []), (4100, [50, 900]))]
    systems = [_system(torch, rt, A, np.ones(A.shape[0]), off)
               for A, off in zip(mats, (0, 1, 2))]
    for md in (N.SOLVE_FP64, N.SOLVE_MIXED):
        rb, xb = _solve(rt, systems, md, 1e-10, stage)
        for i, s in enumerate(systems):
            r, (x,) = _solve(rt, [s], md, 1e-10, stage)
            assert r[0].iterations == rb[i].iterations
            assert np.array_equal(x, xb[i]), (md, i)
        _, xr = _solve(rt, systems, md, 1e-10, stage)
        for i in range(len(systems)):
            assert np.array_equal(xr[i], xb[i])


def _elastic_system(torch, nx, ny, nz, seed):
    """Clamped Tet10 beam (3x3 blocks, rows of 10 to 65 blocks) with a
    seeded body load."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem, DeviceMesh, fixed_mask
    from cloudfem_b200.mesh import box_mesh_tet10
    m = box_mesh_tet10(nx, ny, nz, xlim=(0, 2), ylim=(0, .5), zlim=(0, .5))
    dm = DeviceMesh(m)
    g = np.random.default_rng(seed).normal(size=3) * 1e4
    vals, rhs = dm.assemble_elastic(N.OP_T10_ELAST, 210e9, 0.3, body=tuple(g))
    idx = np.concatenate([3 * m.boundaries["xmin"] + c for c in range(3)])
    mask, x = fixed_mask(dm.rt, 3 * m.n_nodes, idx, np.zeros(len(idx)))
    return dm, BlockSystem(dm.rt, dm.n_nodes, 3, dm.pattern.row_ptr, dm.pattern.col,
                           vals, rhs, x, mask)


@pytest.mark.parametrize("stage,lanes,staged", [(2, 4, 0), (3, 1, 0), (3, 2, 0), (3, 4, 0),
                                                (3, 4, 1), (3, 2, 1)])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_staged_3x3_spmv_matches_register_path(torch, mode, stage, lanes, staged):
    """3x3-block systems on the graph scheduler: the staged SpMV (staging
    2: rows that straddle windows, 65-block vertex rows) or the sliced-ELL
    one (staging 3: slices of 32 / lanes block rows, `lanes` lanes per block
    row) and the register path reach the same answer, and the other path
    repeats bitwise; staged = 1 streams the slices through shared memory."""
    from cloudfem_b200 import _native as N
    dm, sysm = _elastic_system(torch, 10, 3, 3, seed=1)
    rt = dm.rt
    md = N.SOLVE_FP64 if mode == "fp64" else N.SOLVE_MIXED
    rtol = 1e-11 if mode == "fp64" else 1e-10
    _, (x0,) = _solve(rt, [sysm], md, rtol, 0)
    r1, (x1,) = _solve(rt, [sysm], md, rtol, stage, lanes=lanes, staged=staged)
    _, (x1b,) = _solve(rt, [sysm], md, rtol, stage, lanes=lanes, staged=staged)
    if stage == 3 and staged:   # the same arithmetic as the register variant
        _, (x1r,) = _solve(rt, [sysm], md, rtol, stage, lanes=lanes)
        assert np.array_equal(x1, x1r)
    d = np.linalg.norm(x1 - x0) / np.linalg.norm(x0)
    assert d <= (1e-8 if mode == "fp64" else 1e-7), d
    assert np.array_equal(x1, x1b)


@pytest.mark.parametrize("stage,lanes,staged", [(2, 4, 0), (3, 2, 0), (3, 4, 0), (3, 4, 1)])
def test_staged_3x3_spmv_batch_equals_solo_bitwise(torch, stage, lanes, staged):
    """Each 3x3 system's answer is bitwise the same alone and in a batch
    with the staged or sliced-ELL SpMV, in both precisions."""
    from cloudfem_b200 import _native as N
    built = [_elastic_system(torch, nx, 3, 3, seed=nx) for nx in (6, 9, 4)]
    rt = built[0][0].rt
    systems = [s for _, s in built]
    for md in (N.SOLVE_FP64, N.SOLVE_MIXED):
        rb, xb = _solve(rt, systems, md, 1e-10, stage, lanes=lanes, staged=staged)
        for i, s in enumerate(systems):
            r, (x,) = _solve(rt, [s], md, 1e-10, stage, lanes=lanes, staged=staged)
            assert r[0].iterations == rb[i].iterations
            assert np.array_equal(x, xb[i]), (md, i)
