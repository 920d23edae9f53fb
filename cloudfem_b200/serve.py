"""Request serving: iteration-level continuous batching of heat and
elasticity solves.

The reference answers one call at a time on the host (``solve_tet_poisson``,
``solve_tet10_poisson``, ``solve_elasticity_tet10``). Here a server takes a
stream of requests - each a mesh (host arrays, as a client would send them),
its coefficients and boundary data - and keeps the GPU busy with them:

* requests wait in a queue from their arrival time; each (kind, size class)
  - size classes are powers of two of the DOF count - has a slot engine
  (``device.SlotEngine`` over ``cfem_pcg_slots_*``): a fixed set of solve
  slots of that class's capacity whose systems iterate together in rounds
  of 16 CG iterations on the engine's own stream;
* between rounds the server admits the oldest waiting requests into free
  slots (their matrices assembled and their solver state initialised while
  the other slots keep their iterates), as long as the device memory they
  are expected to need fits in the HBM budget next to everything in flight
  (estimates from the DOF and nonzero counts); a request that finishes
  frees its slot at once, whatever the others are doing;
* the engines' rounds are queued on their own streams before any of them
  is polled, so different classes overlap on the device;
* meshes stay resident on the device between requests (connectivity,
  pattern, boundary masks), keyed by the mesh object.

Every result is the solve of its own system: a slot's iterates depend only
on its own system (per-system scalars, fixed-order reductions), so a
request's answer in the mix is bitwise its answer alone on the same engine
class, and within the solve tolerance of any other solve of it.
"""

import threading
import time
from collections import deque

import numpy as np

from . import _native as N
from ._driver import accept, solver_mode
from .batch import BatchSolver, HeatProblem
from .device import BlockSystem, DeviceMesh, SlotEngine, fixed_mask, fixed_vector, pcg

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
        # the estimates depend on the mesh and kind only: computed once (the
        # serving loop asks for them at every admission point)
        if getattr(self, "_nnz_est", None) is None:
            npe = np.asarray(self.mesh.elements).shape[1]
            per_row = 27 if npe == 10 else 15
            self._nnz_est = self.dofs * per_row * self.bs
        return self._nnz_est

    def bytes_estimate(self):
        """Device bytes while in flight: mesh, pattern and contributions,
        FP64 + FP32 values and working copies, solver vectors."""
        if getattr(self, "_bytes_est", None) is None:
            m = self.mesh
            npe = np.asarray(m.elements).shape[1]
            n_el = len(m.elements)
            nnz = self.nnz_estimate()
            self._bytes_est = int(m.n_nodes * 24 + n_el * npe * 4 + n_el * npe * npe * 24
                                  + nnz * (8 + 4 + 16 + 4) + self.dofs * 8 * 12)
        return self._bytes_est

    def size_class(self):
        return int(np.log2(max(self.dofs, 1)))

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


class Server:
    """A serving loop on one GPU.

    hbm_budget: device bytes the server may have in flight (engines and
    requests); precision / rtol: the solves' mode ("mixed" or "fp64") and
    relative residual;
    rounds: rounds of 16 iterations between admission points. workers,
    max_batch_dofs and max_batch only shape ``run_batch`` (one batched
    assembly and solve of a list of requests, the non-streaming path).
    """

    def __init__(self, device=None, hbm_budget=150e9, workers=3,
                 precision="mixed", rtol=1e-10, max_batch_dofs=8e6,
                 max_batch=64, rounds=1):
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
        self.rounds = int(rounds)
        solver_mode(precision, rtol)   # validates
        self._prec = {k: precision for k in KINDS}
        self._engines = {}
        self._engine_bytes = 0.0

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
        res = batch.solve(self._prec[reqs[0].kind], rtol=self.rtol)
        return batch.solutions(), res

    def _run_elast(self, reqs):
        from .physics.elastic3d import _assemble
        mode, rtol = solver_mode(self._prec["t10_elast"], self.rtol)
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

    # ---------------------------------------------------------- slot engines
    def _engine(self, kind, cls):
        """The slot engine of a (kind, size class), created on first use."""
        key = (kind, cls)
        eng = self._engines.get(key)
        if eng is None:
            bs = 3 if kind == "t10_elast" else 1
            max_rows = -(-(2 ** (cls + 1)) // bs)
            per_row = SLOT_ROW_BLOCKS[kind]
            mode = solver_mode(self._prec[kind], self.rtol)[0]
            eng = SlotEngine(self.rt, slots_for_class(cls), bs, mode,
                             max_rows, max_rows * per_row)
            self._engines[key] = eng
            self._engine_bytes += engine_bytes(eng, mode)
        return eng

    def _system(self, r):
        """Assemble request r on the device; returns its BlockSystem (the
        arrays it needs are kept alive by the system's `keep`)."""
        if r.kind == "t10_elast":
            from .physics.elastic3d import _assemble
            dm = self._device_mesh(r.mesh)
            vals, rhs = _assemble(dm, r.mesh, N.OP_T10_ELAST, r.E, r.nu, None,
                                  r.traction, None, 0.0, 0.0, tet10=True)
            idx, v = fixed_vector(r.mesh, {c: (0.0, 0.0, 0.0) for c in r.clamp})
            mask, x = fixed_mask(dm.rt, 3 * r.mesh.n_nodes, idx, v)
            pat = dm.pattern
            return BlockSystem(dm.rt, dm.n_nodes, 3, pat.row_ptr, pat.col, vals,
                               rhs, x, mask, keep=(dm,))
        with self._mesh_lock:
            self.solver.device_mesh(r.mesh)
            batch = self.solver.prepare([HeatProblem(r.mesh, k=r.k, f=r.f, bc=r.bc)])
        batch.assemble()
        it = batch.items[0]
        dm, pat = it["dm"], it["dm"].pattern
        return BlockSystem(self.rt, dm.n_nodes, 1, pat.row_ptr, pat.col, it["vals"],
                           it["rhs"], it["x"], it["mask"], keep=(dm, batch))

    def serve(self, requests, realtime=True):
        """Run a request stream; returns a summary dict. Requests arrive at
        their arrival times (realtime) or all at once."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue = []
        in_use = 0.0
        t0 = time.perf_counter()
        errors = []
        inflight = set()
        changed = True   # arrivals or freed slots since the last admission
        while pending or queue or inflight or any(e.busy for e in self._engines.values()):
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.popleft())
                changed = True
            # admit the oldest waiting requests into free slots (only when an
            # arrival or a finished request changed the picture)
            budget = self.budget - self._engine_bytes - in_use
            chosen = admit(queue, self._free_slots, budget, self._slot_class) if changed else []
            changed = False
            if not chosen and queue and not inflight and \
                    not any(e.busy for e in self._engines.values()):
                chosen = [queue[0]]   # larger than the whole budget: alone
            for r in chosen:
                eng = self._engine(r.kind, self._slot_class(r))
                r.t_start = time.perf_counter() - t0
                eng.assign(self._system(r), self.rtol, tag=r)
                in_use += r.bytes_estimate()
                queue.remove(r)
            # engines whose round has run: collect their finished requests
            # and queue the next round at once; an engine still running is
            # left alone (no engine waits for another)
            idle = True
            for e in list(self._engines.values()):
                if e in inflight:
                    if not e.ready():
                        idle = False
                        continue
                    inflight.discard(e)
                    for system, r, res in e.poll():
                        changed = True
                        r.t_done = time.perf_counter() - t0
                        in_use -= r.bytes_estimate()
                        r.info = res
                        try:
                            accept(res, self.rtol, f"request {r.id}")
                        except RuntimeError as exc:
                            errors.append((r, exc))
                            continue
                        r.result = system.x.cpu().numpy()
                if e.busy:
                    e.run(self.rounds)
                    inflight.add(e)
                    idle = False
            if idle and not queue and pending and realtime:
                time.sleep(min(0.0005, max(0.0, pending[0].arrival - now)))
        if errors:
            r, exc = errors[0]
            raise RuntimeError(f"request {r.id} failed: {exc}") from exc
        return summarize(requests, time.perf_counter() - t0)

    def _slot_class(self, r):
        """The engine class of a request: its size class, or the next one up
        when it would not fit (rows or stored blocks) the class's slots."""
        cached = getattr(r, "_slot_cls", None)
        if cached is not None:
            return cached
        cls = r.size_class()
        bs = r.bs
        rows = r.mesh.n_nodes
        if rows > -(-(2 ** (cls + 1)) // bs) or r.nnz_estimate() // (bs * bs) > \
                -(-(2 ** (cls + 1)) // bs) * SLOT_ROW_BLOCKS[r.kind]:
            cls += 1
        r._slot_cls = cls
        return cls

    def _free_slots(self, kind, cls):
        eng = self._engines.get((kind, cls))
        return slots_for_class(cls) if eng is None else len(eng.free)

    def solve_alone(self, r):
        """The answer a request gets with nothing else in flight (a new
        server of the same settings, the same slot engine class)."""
        import copy
        q = copy.copy(r)
        q.result = q.info = q.t_start = q.t_done = None
        q.arrival = 0.0
        srv = Server(self.rt.device, self.budget, self.workers, self.precision,
                     self.rtol, rounds=self.rounds)
        srv.serve([q], realtime=False)
        return q.result, q.info


# Stored blocks per row a slot is sized for: P1 rows hold at most 15 entries
# on box meshes, Tet10 rows 27-28 on average (vertex rows up to 65).
SLOT_ROW_BLOCKS = {"p1_heat": 16, "t10_heat": 30, "t10_elast": 30}


def slots_for_class(cls):
    """Slots of an engine whose systems hold up to 2^(cls+1) DOFs: about 4 M
    DOFs of capacity per engine (measured faster on the mixed stream than
    2 M: fewer requests wait for a slot), between 2 and 64 slots."""
    return int(min(64, max(2, (1 << 22) >> (cls + 1))))


def engine_bytes(eng, mode):
    """Device bytes a slot engine holds: solver vectors, Jacobi inverse,
    partial sums and the padded working copies of every slot."""
    ts = 4 if mode == N.SOLVE_MIXED else 8
    bs2 = eng.bs * eng.bs
    nd = eng.max_rows * eng.bs
    vec = 6 * nd * ts + nd * 8
    if eng.bs == 1:
        ne = eng.max_nnzb + 3 * eng.max_rows + 8
        copies = ne * (4 + 8 + (4 if mode == N.SOLVE_MIXED else 0))
    elif eng.rt.get_param(N.PARAM_SLOT_SELL3) == 1:
        # sliced ELL: room for block rows of up to 96 blocks (slices of 8
        # block rows on 4 lanes, windows of 256 rows), two row-order sets
        nw = -(-eng.max_rows // 256)
        cap = eng.max_nnzb + eng.max_rows + nw * (8 * 96 + 256 * 3)
        copies = cap * (bs2 * ts + 4) + 2 * (256 * nw + 16 * (32 * nw + 1))
    else:
        copies = eng.max_nnzb * bs2 * ts
    return eng.n_slots * (vec + copies)


def admit(queue, free_slots, budget, slot_class):
    """Requests of `queue` (oldest first) to put into solve slots now: each
    needs a free slot of its (kind, slot class) - free_slots(kind, cls)
    counts them - and its memory estimate within what is left of `budget`.
    A request that does not fit waits; younger requests of other classes
    may still go ahead of it."""
    taken = {}
    out = []
    left = float(budget)
    for r in queue:
        key = (r.kind, slot_class(r))
        free = free_slots(*key) - taken.get(key, 0)
        b = r.bytes_estimate()
        if free <= 0 or b > left:
            continue
        taken[key] = taken.get(key, 0) + 1
        left -= b
        out.append(r)
    return out


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
                        "in_flight_s": float(sum(r.t_done - r.t_start for r in done
                                                 if r.kind == k and r.t_start is not None)),
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
