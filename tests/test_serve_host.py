"""Host-side serving policy (no GPU): stream generation and batch admission."""

import numpy as np

from cloudfem_b200 import serve


def test_stream_is_seeded_and_mixed():
    a = serve.make_stream(60, seed=3, dof_range=(1e3, 2e4))
    b = serve.make_stream(60, seed=3, dof_range=(1e3, 2e4))
    assert [r.kind for r in a] == [r.kind for r in b]
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.diff([r.arrival for r in a]) > 0)
    kinds = {r.kind for r in a}
    assert kinds == set(serve.KINDS)
    for r in a:
        assert 200 <= r.dofs <= 2e5


def _slot_class(r):
    return r.size_class()


def test_admission_takes_oldest_into_free_slots():
    """Oldest first; each request needs a free slot of its own class;
    requests of full classes wait while others go ahead."""
    reqs = serve.make_stream(40, seed=1, dof_range=(1e3, 2e4))
    head = reqs[0]
    key = (head.kind, head.size_class())
    free = {key: 1}
    out = serve.admit(list(reqs), lambda k, c: free.get((k, c), 0), 1e15, _slot_class)
    assert out == [head]
    same = [r for r in reqs if (r.kind, r.size_class()) == key]
    free = {key: 3}
    out = serve.admit(list(reqs), lambda k, c: free.get((k, c), 0), 1e15, _slot_class)
    assert out == same[:3]
    # every class open: everything goes, in arrival order
    out = serve.admit(list(reqs), lambda k, c: 64, 1e15, _slot_class)
    assert out == list(reqs)


def test_admission_respects_memory_budget():
    reqs = serve.make_stream(40, seed=2, dof_range=(1e3, 2e4))
    head = reqs[0]
    slots = lambda k, c: 64  # noqa: E731
    assert head not in serve.admit(list(reqs), slots, head.bytes_estimate() - 1, _slot_class)
    out = serve.admit([head], slots, head.bytes_estimate(), _slot_class)
    assert out == [head]
    budget = sum(r.bytes_estimate() for r in reqs[:5])
    out = serve.admit(list(reqs), slots, budget, _slot_class)
    assert sum(r.bytes_estimate() for r in out) <= budget


def test_slot_engine_sizes():
    assert serve.slots_for_class(9) == 64 and serve.slots_for_class(20) == 2
    assert all(2 <= serve.slots_for_class(c) <= 64 for c in range(6, 24))


def test_stream_cap_keeps_the_full_streams_requests():
    """make_stream(max_dofs=...) keeps a subset of the full stream's
    requests, unchanged (same ids, kinds, arrivals, coefficients, meshes)."""
    import numpy as np
    from cloudfem_b200 import serve
    full = {r.id: r for r in serve.make_stream(40, seed=7, dof_range=(1e3, 3e4))}
    kept = serve.make_stream(40, seed=7, dof_range=(1e3, 3e4), max_dofs=5e3)
    assert 0 < len(kept) < len(full)
    for r in kept:
        f = full[r.id]
        assert (r.kind, r.arrival, r.mesh.n_nodes) == (f.kind, f.arrival, f.mesh.n_nodes)
        if r.kind == "t10_elast":
            assert r.E == f.E
        else:
            assert np.array_equal(r.k, f.k)
        assert r.dofs < 4 * 5e3


class _FakeRt:
    def __init__(self, slot_sell3):
        self.slot_sell3 = slot_sell3

    def get_param(self, param):
        from cloudfem_b200 import _native as N
        assert param == N.PARAM_SLOT_SELL3
        return self.slot_sell3


class _FakeEngine:
    def __init__(self, rt, n_slots, bs, max_rows, max_nnzb):
        self.rt, self.n_slots, self.bs = rt, n_slots, bs
        self.max_rows, self.max_nnzb = max_rows, max_nnzb


def test_engine_bytes_cover_the_sliced_slot_room():
    """The budget estimate of a 3x3 engine in the sliced ELL counts the
    room the library keeps per slot (blocks + rows + per window 8 rows of
    96 blocks and 3 blocks of step rounding per row), columns and values,
    and two row-order sets; the entry-major copy counts values only."""
    from cloudfem_b200 import _native as N
    rows, nnzb = 100_000, 3_000_000
    nw = -(-rows // 256)
    room = nnzb + rows + nw * (8 * 96 + 256 * 3)
    vec = 6 * 3 * rows * 4 + 3 * rows * 8
    sliced = serve.engine_bytes(_FakeEngine(_FakeRt(1), 2, 3, rows, nnzb), N.SOLVE_MIXED)
    assert sliced == 2 * (vec + room * (9 * 4 + 4) + 2 * (256 * nw + 16 * (32 * nw + 1)))
    entry = serve.engine_bytes(_FakeEngine(_FakeRt(0), 2, 3, rows, nnzb), N.SOLVE_MIXED)
    assert entry == 2 * (vec + nnzb * 9 * 4)
    assert 1.1 < sliced / entry < 1.4
