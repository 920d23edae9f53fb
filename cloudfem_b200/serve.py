"""Request serving: continuous batching of heat and elasticity solves.

The reference answers one call at a time on the host (``solve_tet_poisson``,
``solve_tet10_poisson``, ``solve_elasticity_tet10``). Here a server takes a
stream of requests - each a mesh (host arrays, as a client would send them),
its coefficients and boundary data - and keeps the GPU busy with them:

* requests wait in a queue from their arrival time; a free worker takes the
  oldest one together with other queued requests of the same kind and size
  class (powers of two of the DOF count), up to a DOF cap per batch;
* a batch is admitted only while the device memory it is expected to need
  fits in the HBM budget next to the batches in flight (estimates from the
  DOF and nonzero counts); otherwise it waits for memory to free up;
* each worker thread has its own CUDA stream, so batches overlap on the
  device; a batch is one batched assembly and one batched PCG launch
  sequence (``cfem_assemble_batch`` / ``cfem_pcg_solve``);
* meshes stay resident on the device between requests (connectivity,
  pattern, boundary masks), keyed by the mesh object.

Every result is the solve of its own system: batching changes only which
launch it shares, never the arithmetic of another system (per-system
scalars, fixed-order reductions), so a request's answer in the mix equals
its answer alone on the same scheduler, and stays within the solve tolerance
of it otherwise.
"""

import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _native as N
from ._driver import accept, solver_mode
from .batch import BatchSolver, HeatProblem
from .device import BlockSystem, DeviceMesh, fixed_mask, fixed_vector, pcg

KINDS = ("p1_heat", "t10_heat", "t10_elast")


class Request:
    """One solve request.

    kind: "p1_heat" | "t10_heat" (steady -div(k grad T) = f, T = 0 on the
    listed faces) or "t10_elast" (Tet10 elasticity, E scalar, nu, clamped
    faces, surface tractions). k: float or per-element array; arrival:
    seconds from the start of the stream.
    """

    def __init__(self, rid, kind, mesh, arrival=0.0, k=1.0, f=1.0, bc=None,
                 E=210e9, nu=0.3, clamp=("xmin",), traction=None):
        if kind not in KINDS:
            raise ValueError(f"unknown request kind {kind!r}")
        self.id = rid
        self.kind = kind
        self.mesh = mesh
        self.arrival = float(arrival)
        self.k, self.f = k, f
        self.bc = bc if bc is not None else {
            s: 0.0 for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
        self.E, self.nu = E, nu
        self.clamp = tuple(clamp)
        self.traction = traction or {"xmax": (0.0, 0.0, -1e6)}
        self.result = None
        self.info = None
        self.t_start = self.t_done = None

    @property
    def bs(self):
        return 3 if self.kind == "t10_elast" else 1

    @property
    def dofs(self):
        return self.bs * self.mesh.n_nodes

    def nnz_estimate(self):
        npe = np.asarray(self.mesh.elements).shape[1]
        per_row = 27 if npe == 10 else 15
        return self.dofs * per_row * self.bs

    def bytes_estimate(self):
        """Device bytes while in flight: mesh, pattern and contributions,
        FP64 + FP32 values and working copies, solver vectors."""
        m = self.mesh
        npe = np.asarray(m.elements).shape[1]
        n_el = len(m.elements)
        nnz = self.nnz_estimate()
        return int(m.n_nodes * 24 + n_el * npe * 4 + n_el * npe * npe * 24
                   + nnz * (8 + 4 + 16 + 4) + self.dofs * 8 * 12)

    def size_class(self):
        return int(np.log2(max(self.dofs, 1)))

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


class Server:
    def __init__(self, device=None, hbm_budget=150e9, workers=3,
                 precision="mixed", rtol=1e-10, max_batch_dofs=8e6,
                 max_batch=64):
        import torch
        self.rt = N.runtime(device)
        self.torch = torch
        self.budget = float(hbm_budget)
        self.workers = int(workers)
        self.precision = precision
        self.rtol = rtol
        self.max_batch_dofs = float(max_batch_dofs)
        self.max_batch = int(max_batch)
        self.solver = BatchSolver(self.rt.device)
        self._mesh_lock = threading.Lock()
        self._dms = {}

    # -------------------------------------------------------------- batches
    def _device_mesh(self, mesh):
        with self._mesh_lock:
            ent = self._dms.get(id(mesh))
            if ent is None or ent[0] is not mesh:
                dm = DeviceMesh(mesh, self.rt.device)
                dm.pattern  # noqa: B018 - build now
                # other workers' streams use it next
                self.torch.cuda.current_stream(self.rt.device).synchronize()
                ent = (mesh, dm)
                self._dms[id(mesh)] = ent
            return ent[1]

    def _run_heat(self, reqs):
        probs = [HeatProblem(r.mesh, k=r.k, f=r.f, bc=r.bc) for r in reqs]
        with self._mesh_lock:
            for r in reqs:
                self.solver.device_mesh(r.mesh)
            # meshes made here are used by other workers' streams next
            self.torch.cuda.current_stream(self.rt.device).synchronize()
            batch = self.solver.prepare(probs)
        batch.assemble()
        res = batch.solve(self.precision, rtol=self.rtol)
        return batch.solutions(), res

    def _run_elast(self, reqs):
        from .physics.elastic3d import _assemble
        mode, rtol = solver_mode(self.precision, self.rtol)
        systems, keep = [], []
        for r in reqs:
            dm = self._device_mesh(r.mesh)
            vals, rhs = _assemble(dm, r.mesh, N.OP_T10_ELAST, r.E, r.nu, None,
                                  r.traction, None, 0.0, 0.0, tet10=True)
            idx, v = fixed_vector(r.mesh, {c: (0.0, 0.0, 0.0) for c in r.clamp})
            mask, x = fixed_mask(dm.rt, 3 * r.mesh.n_nodes, idx, v)
            pat = dm.pattern
            systems.append(BlockSystem(dm.rt, dm.n_nodes, 3, pat.row_ptr,
                                       pat.col, vals, rhs, x, mask))
            keep.append((vals, rhs, x, mask))
        res = pcg(systems, mode, rtol)
        for i, rr in enumerate(res):
            accept(rr, rtol, f"request {reqs[i].id}")
        return [s.x.cpu().numpy() for s in systems], res

    def run_batch(self, reqs):
        """Solve one batch of same-kind requests on this thread's stream."""
        torch = self.torch
        t0 = time.perf_counter()
        stream = torch.cuda.Stream(device=self.rt.device)
        with torch.cuda.stream(stream):
            if reqs[0].kind == "t10_elast":
                sols, res = self._run_elast(reqs)
            else:
                sols, res = self._run_heat(reqs)
            stream.synchronize()
        dt = time.perf_counter() - t0
        for r in reqs:
            r.batch_s = dt
            r.batch_size = len(reqs)
            r.solve_s = res[0].kernel_ms * 1e-3 if res else 0.0
        return sols, res

    # ---------------------------------------------------------------- loop
    def _take_batch(self, queue, free_bytes):
        """Oldest request plus same-kind, same-size-class followers."""
        head = queue[0]
        if head.bytes_estimate() > free_bytes:
            return None
        batch, dofs, used = [head], head.dofs, head.bytes_estimate()
        cls = (head.kind, head.size_class())
        for r in list(queue)[1:]:
            if len(batch) >= self.max_batch:
                break
            if (r.kind, r.size_class()) != cls:
                continue
            b = r.bytes_estimate()
            if dofs + r.dofs > self.max_batch_dofs or used + b > free_bytes:
                continue
            batch.append(r)
            dofs += r.dofs
            used += b
        for r in batch:
            queue.remove(r)
        return batch, used

    def serve(self, requests, realtime=True):
        """Run a request stream; returns a summary dict. Requests arrive at
        their arrival times (realtime) or all at once."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue = []
        inflight = {}
        in_use = 0.0
        t0 = time.perf_counter()
        pool = ThreadPoolExecutor(max_workers=self.workers)
        errors = []
        try:
            while pending or queue or inflight:
                now = time.perf_counter() - t0
                while pending and (not realtime or pending[0].arrival <= now):
                    queue.append(pending.popleft())
                # collect finished batches
                for fut in [f for f in inflight if f.done()]:
                    reqs, used = inflight.pop(fut)
                    in_use -= used
                    t_done = time.perf_counter() - t0
                    try:
                        sols, res = fut.result()
                    except Exception as exc:  # noqa: BLE001 - reported below
                        errors.append((reqs, exc))
                        continue
                    for r, x, info in zip(reqs, sols, res):
                        r.result, r.info, r.t_done = x, info, t_done
                # admit new batches while workers and memory are free
                while queue and len(inflight) < self.workers:
                    got = self._take_batch(queue, self.budget - in_use)
                    if got is None and not inflight:
                        # larger than the whole budget: run it alone
                        got = ([queue.pop(0)], 0.0)
                    if got is None:
                        break
                    reqs, used = got
                    start = time.perf_counter() - t0
                    for r in reqs:
                        r.t_start = start
                    in_use += used
                    inflight[pool.submit(self.run_batch, reqs)] = (reqs, used)
                if not queue or len(inflight) >= self.workers:
                    time.sleep(0.0005)
                elif realtime and pending and not queue:
                    time.sleep(min(0.0005, max(0.0, pending[0].arrival - now)))
        finally:
            pool.shutdown(wait=True)
        if errors:
            reqs, exc = errors[0]
            raise RuntimeError(f"batch of requests {[r.id for r in reqs]} "
                               f"failed: {exc}") from exc
        return summarize(requests, time.perf_counter() - t0)


def free_dofs(req):
    """DOFs not fixed by Dirichlet data."""
    m = req.mesh
    if req.kind == "t10_elast":
        fixed = set()
        for c in req.clamp:
            fixed.update(np.asarray(m.boundaries[c]).tolist())
        return 3 * (m.n_nodes - len(fixed))
    fixed = set()
    for name in req.bc:
        fixed.update(np.asarray(m.boundaries[name]).tolist())
    return m.n_nodes - len(fixed)


def summarize(requests, wall):
    lat = np.array([r.latency for r in requests if r.latency is not None])
    done = [r for r in requests if r.result is not None]
    dofs = sum(free_dofs(r) for r in done)
    first = min(r.arrival for r in requests)
    last = max(r.t_done for r in done) if done else first
    span = max(last - first, 1e-9)
    return {
        "requests": len(requests), "completed": len(done),
        "solved_dofs": int(dofs), "span_s": span, "wall_s": wall,
        "dof_per_s": dofs / span,
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None,
        "max_ms": float(lat.max() * 1e3) if lat.size else None,
        "by_kind": {k: {"requests": sum(1 for r in done if r.kind == k),
                        "solved_dofs": int(sum(free_dofs(r) for r in done if r.kind == k)),
                        "batches": len({id(getattr(r, "t_start", None)) and (r.t_start, r.t_done)
                                        for r in done if r.kind == k}),
                        "worker_s": float(sum(getattr(r, "batch_s", 0.0) / max(getattr(r, "batch_size", 1), 1)
                                              for r in done if r.kind == k)),
                        "solve_device_s": float(sum(getattr(r, "solve_s", 0.0) / max(getattr(r, "batch_size", 1), 1)
                                                    for r in done if r.kind == k)),
                        "iterations_max": int(max([r.info.iterations for r in done
                                                   if r.kind == k and r.info is not None] or [0]))}
                    for k in KINDS},
    }


# ------------------------------------------------------------ request mix
def _cells_for(kind, dofs, aspect):
    """Box cells (nx, ny, nz), nx = aspect * ny, for about `dofs` DOFs."""
    # nodes per cell: P1 1, Tet10 8; elasticity 3 DOFs per node
    per_cell = {"p1_heat": 1.0, "t10_heat": 8.0, "t10_elast": 24.0}[kind]
    cells = max(dofs / per_cell, 8.0)
    ny = max(1, int(round((cells / aspect) ** (1.0 / 3.0))))
    nx = max(1, int(round(aspect * ny)))
    return nx, ny, ny


def make_stream(n_requests, rate=200.0, mix=(0.60, 0.25, 0.15),
                dof_range=(1e3, 2e6), aspect_range=(1.0, 4.0), sigma=0.5,
                seed=0, mesh_cache=None, max_dofs=None):
    """Seeded request stream: Poisson arrivals, kind mix, log-uniform DOF
    counts, random box aspect ratios, lognormal coefficients (per hex cell
    for heat, one E per elasticity request). Meshes with the same cells are
    shared (a client resubmitting one geometry). max_dofs: keep only the
    requests drawn with at most that many DOFs; every random draw is still
    made, so the kept requests are exactly those of the full stream (and
    no mesh is built for the others)."""
    from .mesh import box_mesh, box_mesh_tet10
    rng = np.random.default_rng(seed)
    cache = {} if mesh_cache is None else mesh_cache
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        kind = KINDS[int(rng.choice(3, p=np.asarray(mix) / np.sum(mix)))]
        dofs = float(np.exp(rng.uniform(np.log(dof_range[0]), np.log(dof_range[1]))))
        aspect = float(rng.uniform(*aspect_range))
        nx, ny, nz = _cells_for(kind, dofs, aspect)
        if kind == "t10_elast":
            coef = float(210e9 * rng.lognormal(0.0, sigma))
        else:
            coef = rng.lognormal(0.0, sigma, nx * ny * nz)
        if max_dofs is not None and dofs > max_dofs:
            continue
        key = (kind != "p1_heat", nx, ny, nz)
        if key not in cache:
            lim = dict(xlim=(0.0, nx / max(ny, 1)), ylim=(0.0, 1.0), zlim=(0.0, 1.0))
            cache[key] = (box_mesh_tet10 if key[0] else box_mesh)(nx, ny, nz, **lim)
        mesh = cache[key]
        if kind == "t10_elast":
            out.append(Request(i, kind, mesh, t, E=coef, nu=0.3))
        else:
            out.append(Request(i, kind, mesh, t, k=np.repeat(coef, 6), f=1.0))
    return out
