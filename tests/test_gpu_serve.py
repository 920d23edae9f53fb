"""Serving on the GPU: a mixed request stream is solved with continuous
batching, and every result equals the same request solved alone."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


# stated tolerance: mixed-precision solves to rtol 1e-10 agree to 1e-8
MIX_TOL = 1e-8


def test_stream_results_equal_alone(torch):
    """Every request of a mixed stream, served with iteration-level
    continuous batching, is bitwise its answer served alone, and within the
    stated tolerance of a one-shot batched solve of it."""
    from cloudfem_b200 import serve
    reqs = serve.make_stream(24, rate=2000.0, dof_range=(1e3, 3e4), seed=11)
    srv = serve.Server(precision="mixed", rtol=1e-10)
    summary = srv.serve(reqs, realtime=True)
    assert summary["completed"] == len(reqs)
    assert summary["p99_ms"] >= summary["p50_ms"] > 0
    for r in reqs:
        alone, info = srv.solve_alone(r)
        assert info.status == 0 and info.iterations == r.info.iterations
        assert np.array_equal(alone, r.result), (r.id, r.kind)
        once, res = srv.run_batch([r])
        assert res[0].status == 0
        err = np.linalg.norm(r.result - once[0]) / max(np.linalg.norm(once[0]), 1e-300)
        assert err <= MIX_TOL, (r.id, r.kind, err)


def test_request_joins_a_running_solve(torch):
    """A well-conditioned request arriving while an ill-conditioned one of
    the same class is iterating is admitted into a free slot of the same
    engine at the next round, finishes first, and equals its answer alone."""
    from cloudfem_b200 import serve
    from cloudfem_b200.mesh import box_mesh_tet10
    beam = box_mesh_tet10(24, 3, 3, xlim=(0, 2.0), ylim=(0, 0.25), zlim=(0, 0.25))
    cube = box_mesh_tet10(6, 6, 6)
    slow = serve.Request(0, "t10_elast", beam, arrival=0.0)
    fast = serve.Request(1, "t10_elast", cube, arrival=0.003)
    srv = serve.Server(precision="mixed", rtol=1e-10)
    assert srv._slot_class(slow) == srv._slot_class(fast)
    srv.serve([slow, fast], realtime=True)
    assert slow.info.iterations > 3 * fast.info.iterations
    assert fast.t_start < slow.t_done           # admitted mid-solve
    assert fast.t_done < slow.t_done            # and done first
    assert len(srv._engines) == 1               # in the same slot engine
    alone, info = srv.solve_alone(fast)
    assert np.array_equal(alone, fast.result)


def test_heat_request_matches_plain_fp64(torch):
    """A served P1 heat request against the drop-in FP64 path on the same
    mesh and (per-cell, hence callable) conductivity."""
    from cloudfem_b200 import serve
    from cloudfem_b200.fem.tet_poisson import solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    n = 9
    m = box_mesh(n, n, n)
    rng = np.random.default_rng(4)
    kc = rng.lognormal(0.0, 0.5, n ** 3)

    def kf(x, y, z):
        i = np.minimum((np.asarray(x) * n).astype(int), n - 1)
        j = np.minimum((np.asarray(y) * n).astype(int), n - 1)
        k = np.minimum((np.asarray(z) * n).astype(int), n - 1)
        return kc.reshape(n, n, n)[k, j, i]

    r = serve.Request(0, "p1_heat", m, k=np.repeat(kc, 6), f=1.0)
    srv = serve.Server(workers=1)
    srv.serve([r], realtime=False)
    u = solve_tet_poisson(m, k=kf, f=1.0, bc=r.bc)
    assert np.linalg.norm(r.result - u) / np.linalg.norm(u) <= MIX_TOL
