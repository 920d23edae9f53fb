"""Solve slots of 3x3 systems in the sliced-ELL layout (the default,
CFEM_PARAM_SLOT_SELL3 = 1) against slots on the entry-major copy (0) and
against a solve alone: the same answers within the solve tolerance, a slot
that takes systems in turn (its two row-order sets alternate) reproducing a
system's answer bitwise, and a system whose layout exceeds the slot's room
refused with the engine still usable."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9     # two FP64 solves to rtol 1e-10 with different sum orders
MIXED_TOL = 1e-8


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _elastic(shape, lims):
    """A maker of fresh clamped Tet10 cantilever systems (x zeroed)."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem, DeviceMesh, fixed_mask, fixed_vector
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics.elastic3d import _assemble
    m = box_mesh_tet10(*shape, xlim=(0, lims[0]), ylim=(0, lims[1]), zlim=(0, lims[2]))
    dm = DeviceMesh(m)
    vals, rhs = _assemble(dm, m, N.OP_T10_ELAST, 210e9, 0.3, None,
                          {"xmax": (0.0, 0.0, -1e6)}, None, 0.0, 0.0, True)
    idx, v = fixed_vector(m, {"xmin": (0.0, 0.0, 0.0)})

    def make():
        mask, x = fixed_mask(dm.rt, 3 * m.n_nodes, idx, v)
        pat = dm.pattern
        return BlockSystem(dm.rt, m.n_nodes, 3, pat.row_ptr, pat.col, vals, rhs, x, mask,
                           keep=(dm,))
    return make


def _engine(rt, sell3, n_slots, mode, max_rows, max_nnzb):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import SlotEngine
    before = rt.get_param(N.PARAM_SLOT_SELL3)
    try:
        rt.set_param(N.PARAM_SLOT_SELL3, sell3)
        return SlotEngine(rt, n_slots, 3, mode, max_rows, max_nnzb)
    finally:
        rt.set_param(N.PARAM_SLOT_SELL3, before)


def _drain(eng, want):
    """Run rounds until `want` systems have finished; {tag: (x, result)}."""
    from cloudfem_b200 import _native as N
    done = {}
    for _ in range(20000):
        if len(done) >= want:
            break
        eng.run(4)
        for system, tag, res in eng.poll():
            assert res.status == N.CFEM_OK, (tag, res)
            done[tag] = (system.x.cpu().numpy().copy(), res)
    assert len(done) >= want
    return done


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("mode_name", ["fp64", "mixed"])
def test_sliced_slots_match_entry_major_slots_and_alone(torch, mode_name):
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import pcg
    mode = N.SOLVE_FP64 if mode_name == "fp64" else N.SOLVE_MIXED
    tol = FP64_TOL if mode_name == "fp64" else MIXED_TOL
    rt = N.runtime()
    beam = _elastic((16, 2, 2), (0.8, 0.1, 0.1))
    cube = _elastic((4, 4, 4), (1.0, 1.0, 1.0))
    alone = {}
    for tag, make in (("beam", beam), ("cube", cube)):
        s = make()
        res = pcg([s], mode, 1e-10)
        assert res[0].status == N.CFEM_OK
        alone[tag] = s.x.cpu().numpy()
    out = {}
    for sell3 in (1, 0):
        eng = _engine(rt, sell3, 2, mode, 2000, 2000 * 30)
        eng.assign(beam(), 1e-10, tag="beam")
        eng.assign(cube(), 1e-10, tag="cube")
        out[sell3] = _drain(eng, 2)
        for tag in ("beam", "cube"):
            assert _rel(out[sell3][tag][0], alone[tag]) <= tol, (sell3, tag)
    for tag in ("beam", "cube"):
        assert _rel(out[1][tag][0], out[0][tag][0]) <= tol, tag


def test_slot_reuse_is_bitwise(torch):
    """One slot takes the cube, then the beam, then the cube again: the
    row-order set in use alternates and the cube's answer is bitwise the
    same both times."""
    from cloudfem_b200 import _native as N
    rt = N.runtime()
    beam = _elastic((16, 2, 2), (0.8, 0.1, 0.1))
    cube = _elastic((4, 4, 4), (1.0, 1.0, 1.0))
    eng = _engine(rt, 1, 1, N.SOLVE_MIXED, 2000, 2000 * 30)
    xs = []
    for i, make in enumerate((cube, beam, cube)):
        eng.assign(make(), 1e-10, tag=i)
        xs.append(_drain(eng, 1)[i])
    assert np.array_equal(xs[0][0], xs[2][0])
    assert xs[0][1].iterations == xs[2][1].iterations


def test_oversized_layout_refused(torch):
    """Rows of 1,000 blocks (one per window of 256 block rows) need about
    three times the room a slot of this capacity keeps (89,920 entries
    against 30,720): assign refuses the system (an invalid argument,
    ValueError as in the reference) and changes nothing; the next system
    solves."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import BlockSystem, pcg
    rt = N.runtime()
    n, cap_nnzb = 2560, 5 * 2560
    rows = []
    for r in range(n):
        if r % 256 == 0:
            cols = np.unique(np.r_[r, np.arange(1, n, 2)[:999]])
        else:
            cols = np.array([r])
        rows.append(cols)
    rp = np.zeros(n + 1, dtype=np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    assert rp[-1] <= cap_nnzb
    ci = np.concatenate(rows).astype(np.int32)
    vals = np.zeros((len(ci), 3, 3))
    vals[ci == np.repeat(np.arange(n), np.diff(rp))] = np.eye(3)
    dev = "cuda"
    bad = BlockSystem(rt, n, 3, torch.as_tensor(rp, device=dev), torch.as_tensor(ci, device=dev),
                      torch.as_tensor(vals.ravel(), device=dev),
                      torch.ones(3 * n, dtype=torch.float64, device=dev),
                      torch.zeros(3 * n, dtype=torch.float64, device=dev))
    eng = _engine(rt, 1, 1, N.SOLVE_FP64, n, cap_nnzb)
    with pytest.raises(ValueError, match="sliced-ELL layout has 89920 blocks"):
        eng.assign(bad, 1e-10, tag="bad")
    assert eng.free == [0]
    cube = _elastic((3, 3, 3), (1.0, 1.0, 1.0))
    eng.assign(cube(), 1e-10, tag="cube")
    x, res = _drain(eng, 1)["cube"]
    s = cube()
    ref = pcg([s], N.SOLVE_FP64, 1e-10)
    assert ref[0].status == N.CFEM_OK
    assert _rel(x, s.x.cpu().numpy()) <= FP64_TOL
