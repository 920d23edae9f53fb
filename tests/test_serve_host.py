"""Host-side serving policy (no GPU): stream generation and batch admission."""

import numpy as np

from cloudfem_b200 import serve


def _server(budget, max_batch_dofs=1e9, max_batch=64):
    s = object.__new__(serve.Server)
    s.budget = budget
    s.max_batch_dofs = max_batch_dofs
    s.max_batch = max_batch
    return s


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


def test_batches_take_oldest_and_same_class():
    reqs = serve.make_stream(40, seed=1, dof_range=(1e3, 2e4))
    queue = list(reqs)
    srv = _server(1e12)
    batch, used = srv._take_batch(queue, 1e12)
    assert batch[0] is reqs[0]
    cls = (reqs[0].kind, reqs[0].size_class())
    assert all((r.kind, r.size_class()) == cls for r in batch)
    assert used == sum(r.bytes_estimate() for r in batch)
    assert all(r not in queue for r in batch)


def test_admission_respects_memory_budget():
    reqs = serve.make_stream(40, seed=2, dof_range=(1e3, 2e4))
    head = reqs[0]
    srv = _server(1e12)
    # no room for the oldest request: nothing is admitted
    assert srv._take_batch(list(reqs), head.bytes_estimate() - 1) is None
    # room for exactly the oldest: it goes alone
    batch, used = srv._take_batch(list(reqs), head.bytes_estimate())
    assert batch == [head] and used == head.bytes_estimate()


def test_batch_dof_cap():
    reqs = serve.make_stream(80, seed=4, dof_range=(1e3, 4e3))
    srv = _server(1e12, max_batch_dofs=3 * reqs[0].dofs)
    batch, _ = srv._take_batch(list(reqs), 1e12)
    assert sum(r.dofs for r in batch) <= 3 * reqs[0].dofs


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
