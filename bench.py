"""Benchmark of the assembly -> CSR -> solve hot path on B200.

Default workload: 512 independent Tet10 steady-heat unit cubes, subdivision
n ~ U{4..24} (seed 0; 14.4 M Tet10 elements, 17.7 M free DOFs in total),
lognormal(0, 1) conductivity per hex cell, unit source, T = 0 on all faces.
One step = batched element matrices + CSR reduction of every mesh (one
launch per pass) + one batched mixed-precision PCG (FP32 CG, FP64 residual,
update and convergence test) to 1e-8 relative residual, meshes and patterns
resident. Beside it, in the same line: the plain FP64 GPU path (one
assembly + FP64 solve call per mesh over all 512 meshes, same tolerance),
the ratio of the two, the same batched launches in FP64, and the largest
error of the mixed answers against an FP64 solve.

Other workloads (--workload): the Tet10 elasticity beam 80 x 10 x 10
(213,003 DOFs; FP64 by default), a transient P1 heat march on a 128^3 box,
a serving stream of mixed requests, and the Tet10 A-V eddy-current phasor
and transient solves.

value  : solved (free) DOF/s with the meshes already resident in HBM.
e2e    : the same through the public API (solve_batch with host
         coefficient arrays in and nodal solutions out, copies inside the
         timed region).
--impl reference : the CPU oracle (a NumPy/SciPy restatement of the
         reference: vectorised assembly, the reference's Dirichlet step and
         SuperLU) on a bounded sample of the workload, on the host cores.

Multi-GPU: the path solves independent systems, so --gpus N runs N
replicas (one process per GPU) and reports the aggregate DOF/s.
"""

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("solved DOF/s at 1e-8 rel err vs FP64 plain GPU path; "
          "p50/p99 latency")
E, NU = 210e9, 0.3
BC = {"xmin": (0.0, 0.0, 0.0)}
TRACTION = {"xmax": (0.0, 0.0, -1e6)}
BEAM = dict(xlim=(0.0, 2.0), ylim=(0.0, 0.25), zlim=(0.0, 0.25))
FULL = (80, 10, 10)
CPU_SAMPLE = (48, 6, 6)   # about 12 s of one SuperLU solve on 16 host cores
RTOL = 1e-10
L2_FLUSH_BYTES = 256 << 20


SPMV_STAGE = None   # --spmv-stage: None keeps the library default
SELL_SORT = None    # --sell-sort: None keeps the library default
SELL3_LANES = None  # --sell3-lanes: None keeps the library default
SELL3_STAGED = None  # --sell3-staged: None keeps the library default
SLOT_SELL3 = None   # --slot-sell3: None keeps the library default


def _set_scheduler(rt, name):
    """Solver scheduler of the run (auto unless asked; polled graphs make
    every solver launch visible to per-launch profilers), and the scalar
    SpMV staging when asked."""
    from cloudfem_b200 import _native as N
    code = {"auto": N.SCHED_AUTO, "persistent": N.SCHED_PERSISTENT,
            "graph": N.SCHED_GRAPH, "polled": N.SCHED_GRAPH_POLLED}[name]
    N.check(rt.lib.cfem_ctx_set_scheduler(rt.ctx, code))
    if SPMV_STAGE is not None:
        rt.set_param(N.PARAM_SPMV_STAGE, SPMV_STAGE)
    if SELL_SORT is not None:
        rt.set_param(N.PARAM_SELL_SORT, SELL_SORT)
    if SELL3_LANES is not None:
        rt.set_param(N.PARAM_SELL3_LANES, SELL3_LANES)
    if SELL3_STAGED is not None:
        rt.set_param(N.PARAM_SELL3_STAGED, SELL3_STAGED)
    if SLOT_SELL3 is not None:
        rt.set_param(N.PARAM_SLOT_SELL3, SLOT_SELL3)


def _block_spmv_kernel(rt, precision):
    """(name, profile summary) of the 3x3 SpMV-phase kernel the context's
    staging selects."""
    from cloudfem_b200 import _native as N
    stage = rt.get_param(N.PARAM_SPMV_STAGE)
    if stage in (3, 4):
        lanes = rt.get_param(N.PARAM_SELL3_LANES)
        staged = rt.get_param(N.PARAM_SELL3_STAGED)
        if staged == 1 or (staged == 2 and precision == "mixed"):
            return (f"k_gxl3s (PCG SpMV phase, sliced ELL, {lanes} lanes per block row, "
                    "slices bulk-copied through shared memory)",
                    "k_gxl3_tet10_elasticity_80x10x10")
        return (f"k_gxl3 (PCG SpMV phase, sliced ELL, {lanes} lanes per block row: "
                "q = A p, p update, p.q)", "k_gxl3_tet10_elasticity_80x10x10")
    if stage == 2:
        return ("k_gxs3 (PCG SpMV phase, blocks bulk-staged through shared memory)", None)
    return ("k_gx (PCG SpMV phase, register path: q = A p, p update, p.q)",
            "k_gx_tet10_elasticity_80x10x10")


def _scalar_spmv_kernel(rt, precision):
    """Name of the scalar SpMV-phase kernel the context's staging selects."""
    from cloudfem_b200 import _native as N
    stage = rt.get_param(N.PARAM_SPMV_STAGE)
    if stage == 4:   # auto: sliced ELL in FP64, staged windows in FP32
        stage = 3 if precision == "fp64" else 1
    return {0: "k_gx (register path)", 3: "k_gxl (sliced ELL, one row per lane)"}.get(
        stage, "k_gxs (matrix bulk-staged through shared memory)")


def _barrier(world):
    """Every rank at the same point with its GPU idle: before and after each
    timed region (on one process only the device synchronisation)."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def _max_over_ranks(world, values):
    """The slowest rank's figures (MAX over ranks, element by element); every
    rank must call it, in the same order. On one process the values as
    floats."""
    vals = [float(v) for v in values]
    if world <= 1:
        return vals
    import torch
    import torch.distributed as dist
    dev = (torch.device("cuda", torch.cuda.current_device())
           if dist.get_backend() == "nccl" else torch.device("cpu"))
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
             "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(self.NAMES, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _beam(shape):
    from cloudfem_b200.mesh import box_mesh_tet10
    return box_mesh_tet10(*shape, **BEAM)


def _free_dofs(mesh):
    return 3 * mesh.n_nodes - 3 * len(mesh.boundaries["xmin"])


def pcg_bytes(n_nodes, nnzb, iters, updates, precision="mixed"):
    """Algorithmic HBM bytes of one solve launch (3x3 blocks, s = 4 B for
    the mixed path's FP32 vectors and matrix, 8 B for the FP64 path).

    Phase A per iteration: blocks + column index (9 s + 4 B / block), row
    pointers, read z and p, write p and q (4 x 3 s B / node).
    Phase B: read p, q, r (9 s), block-Jacobi inverse (9 s), fixed mask
    (3 B), x (24 B), write x (24 B), r, z (6 s) per node.
    Phase R (true residual; plus INIT once): FP64 blocks + index
    (76 B / block), row pointers, read x, b (48 B), fixed mask (3 B), write
    r, z (6 s).
    """
    sz = 4 if precision == "mixed" else 8
    a = nnzb * (9 * sz + 4) + 4 * (n_nodes + 1) + 12 * sz * n_nodes
    b = (24 * sz + 51) * n_nodes
    r = nnzb * 76 + 4 * (n_nodes + 1) + (51 + 6 * sz) * n_nodes
    return iters * (a + b) + (updates + 1) * r


def spmv_bytes(n_nodes, nnzb, sz):
    """Algorithmic bytes of one SpMV-phase launch (3x3 blocks, s-byte
    values): blocks + column index, row pointers, read z and p, write p and
    q."""
    return nnzb * (9 * sz + 4) + 4 * (n_nodes + 1) + 12 * sz * n_nodes


def _profiled_traffic(name, precision):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    key = f"dram_bytes_per_launch_{precision}:"
    with open(path) as f:
        for line in f:
            if line.strip().startswith(key):
                return int(line.split(":")[1].strip().split()[0])
    return None


def _device_step(dm, mesh, precision):
    """Pattern + assembly + loads + masking + solve on resident inputs."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200._driver import last_solve_info, solve_block
    from cloudfem_b200.device import fixed_vector
    from cloudfem_b200.physics.elastic3d import _assemble
    dm._pattern = None                      # rebuild the CSR structure
    vals, rhs = _assemble(dm, mesh, N.OP_T10_ELAST, E, NU, None, TRACTION,
                          None, 0.0, 0.0, tet10=True)
    idx, v = fixed_vector(mesh, BC)
    x = solve_block(dm, 3, vals, rhs, idx, v, precision, RTOL,
                    what="bench solve")
    return x, last_solve_info()[0]


def run_ours(args, rank, world, local_rank):
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import DeviceMesh
    from cloudfem_b200.physics.elastic_tet10 import solve_elasticity_tet10

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    _set_scheduler(rt, args.scheduler)
    mesh = _beam(FULL)
    free = _free_dofs(mesh)
    dm = DeviceMesh(mesh, local_rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    # FP64 plain reference solution (accuracy gate) and one solve in the
    # other precision, reported beside the timed one.
    _device_step(dm, mesh, "fp64")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x64, info64 = _device_step(dm, mesh, "fp64")
    torch.cuda.synchronize()
    fp64_s = time.perf_counter() - t0
    u64 = x64.clone()
    t0 = time.perf_counter()
    xm, infom = _device_step(dm, mesh, "mixed")
    torch.cuda.synchronize()
    mixed_s = time.perf_counter() - t0
    mixed_err = float(torch.linalg.norm(xm - u64) / torch.linalg.norm(u64))

    for _ in range(args.warmup):
        _device_step(dm, mesh, args.precision)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing (value)
    times, infos = [], []
    l0 = rt.launches()
    barrier()
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)                # evict L2 between steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            x, info = _device_step(dm, mesh, args.precision)
            e1.record()
            infos.append(info)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    barrier()
    launches = rt.launches() - l0
    err = float(torch.linalg.norm(x - u64) / torch.linalg.norm(u64))

    # ---- end-to-end through the public API (host inputs and outputs)
    for _ in range(1):
        solve_elasticity_tet10(mesh, E, NU, bc=BC, traction=TRACTION,
                               precision=args.precision, rtol=RTOL)
    e2e_times = []
    barrier()
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solve_elasticity_tet10(mesh, E, NU, bc=BC, traction=TRACTION,
                               precision=args.precision, rtol=RTOL)
        torch.cuda.synchronize()
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    barrier()

    ms, e2e_ms = _max_over_ranks(world, [np.sum(times), np.sum(e2e_times)])
    if rank != 0:
        return None

    pat = dm.pattern
    last = infos[-1]
    bytes_solve = pcg_bytes(mesh.n_nodes, pat.nnz, last.iterations,
                            last.residual_updates, args.precision)
    sz = 4 if args.precision == "mixed" else 8
    bytes_spmv = spmv_bytes(mesh.n_nodes, pat.nnz, sz)
    spmv_ms = float(np.mean([i.spmv_ms for i in infos if i.spmv_samples])) \
        if any(i.spmv_samples for i in infos) else None
    peak, peak_kind = _peaks()
    if spmv_ms:
        achieved = bytes_spmv / (spmv_ms * 1e-3) / 1e9
    else:
        achieved = bytes_solve / (last.kernel_ms * 1e-3) / 1e9
    kname, kprof = _block_spmv_kernel(rt, args.precision)
    traffic = (_profiled_traffic(kprof, "fp32" if args.precision == "mixed" else "fp64")
               if kprof else None)
    h2d = mesh.nodes.size * 8 + mesh.elements.size * 4
    d2h = 3 * mesh.n_nodes * 8
    value = world * free * args.steps / (ms * 1e-3)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "DOF/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 PCG + f64 residual/update" if args.precision == "mixed"
                 else "f64",
        "data": "synthetic (structured Kuhn Tet10 beam, no dataset)",
        "config": {
            "workload": "tet10_elasticity_beam_80x10x10",
            "elements": int(mesh.n_elements), "nodes": int(mesh.n_nodes),
            "dofs": int(3 * mesh.n_nodes), "free_dofs": int(free),
            "precision": args.precision, "rtol": RTOL,
            "iterations": last.iterations,
            "residual_updates": last.residual_updates,
            "rel_err_vs_fp64_plain": err,
            "fp64_plain": {"iterations": info64.iterations,
                           "dof_per_s": free / fp64_s,
                           "kernel_ms": info64.kernel_ms},
            "mixed": {"iterations": infom.iterations,
                      "residual_updates": infom.residual_updates,
                      "dof_per_s": free / mixed_s,
                      "kernel_ms": infom.kernel_ms,
                      "rel_err_vs_fp64_plain": mixed_err},
            "l2": "256 MiB buffer written between timed steps",
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": world * free * args.steps / (e2e_ms * 1e-3),
                "unit": "DOF/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {
            "kernel": kname,
            "bound": "hbm", "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "bytes_per_launch": bytes_spmv,
            "launch_ms": spmv_ms,
            "traffic": traffic,
            "solve": {"bytes": bytes_solve, "kernel_ms": last.kernel_ms,
                      "achieved_gbs": bytes_solve / (last.kernel_ms * 1e-3) / 1e9},
        },
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    return out


def cpu_baseline(shape=CPU_SAMPLE):
    """The oracle (NumPy + SuperLU) on a bounded sample of the workload."""
    from oracle import cfem_oracle as O
    m = O.box_mesh_tet10(*shape, **BEAM)
    free = 3 * m.n_nodes - 3 * len(m.boundaries["xmin"])
    t0 = time.perf_counter()
    O.solve_elasticity_tet10(m, E, NU, bc=BC, traction=TRACTION)
    dt = time.perf_counter() - t0
    return {"value": free / dt, "unit": "DOF/s", "cores": os.cpu_count(),
            "kind": "port", "seconds": dt,
            "sample": f"Tet10 beam {shape[0]}x{shape[1]}x{shape[2]} cells "
                      f"({free} free DOFs), one solve, {dt:.1f} s"}


# ---------------------------------------------------- batched Tet10 heat meshes
BATCH_MESHES = 512
BATCH_SEED = 0


def batch_draw(count=BATCH_MESHES, seed=BATCH_SEED):
    """Seeded batch: n ~ U{4..24}, lognormal(0, 1) conductivity per hex cell."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(4, 25, size=count)
    ks = [rng.lognormal(0.0, 1.0, int(n) ** 3) for n in ns]
    return ns, ks


def batch_cell_fn(n, kc):
    """The per-cell conductivity as the reference's callable API sees it:
    k(x, y, z) = K[i, j, k] of the hex cell containing the point (Keast
    points are interior, so the lookup is exact)."""
    kc3 = kc.reshape(n, n, n)          # cell order k, j, i (box_mesh)

    def k(x, y, z):
        i = np.minimum((np.asarray(x) * n).astype(int), n - 1)
        j = np.minimum((np.asarray(y) * n).astype(int), n - 1)
        kk = np.minimum((np.asarray(z) * n).astype(int), n - 1)
        return kc3[kk, j, i]
    return k


def batch_problems(ns, ks):
    from cloudfem_b200.batch import HeatProblem
    from cloudfem_b200.mesh import box_mesh_tet10
    meshes = {int(n): box_mesh_tet10(int(n), int(n), int(n)) for n in set(ns)}
    bc = {s: 0.0 for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    # 6 Kuhn tets per cell, cells in k, j, i order: element e is in cell e // 6
    return [HeatProblem(meshes[int(n)], k=np.repeat(kc, 6), f=1.0, bc=bc)
            for n, kc in zip(ns, ks)]


def run_batched_heat(args, rank, world, local_rank):
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200.batch import BatchSolver, solve_batch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    _set_scheduler(rt, args.scheduler)
    ns, ks = batch_draw(args.meshes)
    problems = batch_problems(ns, ks)
    solver = BatchSolver(local_rank)
    batch = solver.prepare(problems)
    free = batch.free_dofs
    if args.one_pass:
        # one assembly and one mixed solve, nothing else: the launch
        # sequence a per-launch profiler should see (no timing, no line)
        batch.assemble()
        res = batch.solve("mixed", rtol=1e-8)
        torch.cuda.synchronize()
        print(f"one pass: {len(res)} systems, {free} free DOFs, "
              f"{max(r.iterations for r in res)} iterations at most", file=sys.stderr)
        return None
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    # the configuration's tolerance: CG with FP64 refinement to 1e-8 relative
    # residual (the answer then agrees with FP64 to about 6e-9, within the
    # 1e-8 accuracy bar); the plain FP64 path is timed to the same tolerance
    rtol = 1e-8

    def step(precision, tol=rtol):
        batch.assemble()
        return batch.solve(precision, rtol=tol)

    # FP64 answer of the same batch (accuracy gate, tighter tolerance)
    step("fp64", 1e-12)
    x64 = [it["x"].clone() for it in batch.items]
    # plain FP64 GPU path: one problem per assembly + solve call (what a
    # caller of the drop-in solve gets, mesh and pattern resident), over
    # every mesh of the batch, to the same tolerance
    solve_batch(problems[:2], precision="fp64", rtol=rtol, solver=solver)
    torch.cuda.synchronize()
    _barrier(world)
    t0 = time.perf_counter()
    for pb in problems:
        solve_batch([pb], precision="fp64", rtol=rtol, solver=solver)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    # the same batched launches in FP64: separates batching from precision
    step("fp64")
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    flush.fill_(1.0)
    e0.record()
    step("fp64")
    e1.record()
    e1.synchronize()
    fp64_batched_ms = e0.elapsed_time(e1)
    plain_s, fp64_batched_ms = _max_over_ranks(world, [plain_s, fp64_batched_ms])

    # autotuner: element-kernel block shape and solve-loop body length
    from cloudfem_b200 import autotune
    tuned = autotune.tune_batch(batch, args.precision, rtol, repeat=2)
    for _ in range(args.warmup):
        step(args.precision)
    torch.cuda.synchronize()
    times, launches0 = [], rt.launches()
    _barrier(world)
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res = step(args.precision)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    _barrier(world)
    launches = rt.launches() - launches0
    err = max(float(torch.linalg.norm(it["x"] - x) / torch.linalg.norm(x))
              for it, x in zip(batch.items, x64))
    iters = [r.iterations for r in res]
    # SpMV roofline: k_gx over every system of the batch (scalar CSR: values
    # and column indices, row pointers, gathered p read once, q written)
    sz = 4 if args.precision == "mixed" else 8
    nnz_all = sum(it["dm"].pattern.nnz for it in batch.items)
    n_all = sum(it["dm"].n_nodes for it in batch.items)
    spmv_b = nnz_all * (sz + 4) + 4 * (n_all + len(batch.items)) + 2 * sz * n_all
    spmv_ms = float(np.mean([r.spmv_ms for r in res[:1] if r.spmv_samples] or [0.0]))
    peak, peak_kind = _peaks()

    # end to end: host coefficient arrays in, solutions out (meshes and
    # their patterns stay resident in the solver, as in a serving process)
    e2e = []
    _barrier(world)
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solve_batch(problems, precision=args.precision, rtol=rtol, solver=solver)
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    _barrier(world)
    ms, e2e_ms = _max_over_ranks(world, [np.sum(times), np.sum(e2e)])
    if rank != 0:
        return None
    h2d = sum(pb.k.nbytes for pb in problems)
    d2h = sum(it["dm"].n_nodes * 8 for it in batch.items)
    value = world * free * args.steps / (ms * 1e-3)
    plain_rate = world * free / plain_s
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "DOF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 PCG + f64 residual/update" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded unit-cube Tet10 meshes, lognormal k per cell)",
        "config": {
            "workload": f"batched_tet10_heat_{len(problems)}_meshes_n4to24",
            "meshes": len(problems), "free_dofs": int(free),
            "precision": args.precision, "rtol": rtol,
            "iterations_max": int(max(iters)), "iterations_mean": float(np.mean(iters)),
            "rel_err_vs_fp64_max": err,
            "autotune": {k: v["best"] for k, v in tuned.items()},
            "plain_fp64_per_mesh": {
                "meshes": len(problems), "dof_per_s": plain_rate,
                "seconds": plain_s,
                "what": "one assembly + FP64 solve call per mesh, all meshes, "
                        "same tolerance, meshes resident"},
            "vs_plain_fp64": value / plain_rate,
            "fp64_batched": {"dof_per_s": world * free / (fp64_batched_ms * 1e-3),
                             "ms": fp64_batched_ms,
                             "what": "the same batched launches with the FP64 solver"},
            "l2": "256 MiB buffer written between timed steps",
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": world * free * args.steps / (e2e_ms * 1e-3), "unit": "DOF/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": "meshes and patterns resident; coefficients and solutions cross"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if spmv_ms > 0:
        ach = spmv_b / (spmv_ms * 1e-3) / 1e9
        out["roofline"] = {
            "kernel": _scalar_spmv_kernel(rt, args.precision) + " (batched PCG SpMV phase over all systems: q = A p, p.q)",
            "bound": "hbm", "achieved": ach, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": ach / peak, "bytes_per_launch": int(spmv_b),
            "launch_ms": spmv_ms,
            "traffic": (_profiled_traffic("k_gxs_batched_tet10_heat", "fp32")
                        if args.precision == "mixed" else
                        _profiled_traffic("k_gxl_batched_tet10_heat_fp64", "fp64")),
        }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_batched_heat(ns, ks)
    return out


def cpu_baseline_batched_heat(ns, ks, cap_n=7, count=24):
    """Oracle (NumPy assembly + the reference's Dirichlet step and SuperLU,
    explicit zeros kept) on the first `count` draws with n <= cap_n, one
    solve each; plus a power law t(n) = a n^b fitted to those per-mesh times
    and summed over every mesh of the draw, an extrapolated estimate of the
    whole workload on the host (labelled as such)."""
    from oracle import cfem_oracle as O
    bc = {s: 0.0 for s in O.FACE_NAMES}
    picked = [(int(n), kc) for n, kc in zip(ns, ks) if n <= cap_n][:count]
    free, per_n = 0, []
    t0 = time.perf_counter()
    for n, kc in picked:
        t1 = time.perf_counter()
        m = O.box_mesh_tet10(n, n, n)
        O.solve_tet10_poisson(m, k=batch_cell_fn(n, kc), f=1.0, bc=bc)
        per_n.append((n, time.perf_counter() - t1))
        free += (2 * n - 1) ** 3
    dt = time.perf_counter() - t0
    out = {"value": free / dt, "unit": "DOF/s", "cores": os.cpu_count(),
           "kind": "port", "seconds": dt,
           "sample": f"{len(picked)} of the seeded meshes with n <= {cap_n} "
                     f"({free} free DOFs), one solve each"}
    nn = np.array([p[0] for p in per_n], dtype=float)
    tt = np.array([p[1] for p in per_n])
    if len(set(nn.tolist())) >= 2:
        b, loga = np.polyfit(np.log(nn), np.log(tt), 1)
        t_all = float(np.sum(np.exp(loga) * np.asarray(ns, dtype=float) ** b))
        free_all = float(np.sum((2 * np.asarray(ns, dtype=float) - 1) ** 3))
        out["extrapolated_full_workload"] = {
            "dof_per_s": free_all / t_all, "seconds": t_all,
            "fit": f"t(n) = {np.exp(loga):.3e} n^{b:.2f} s over n = "
                   f"{int(nn.min())}..{int(nn.max())}",
            "note": "extrapolated, not measured: the sample's power law summed "
                    f"over all {len(ns)} meshes (n up to {int(max(ns))})"}
    return out


# ------------------------------------------------ transient P1 heat, 128^3 box
TRANSIENT_N = 128
TRANSIENT_STEPS = 200
TRANSIENT_PARAMS = dict(k=45.0, rho_cp=3.6e6, t0=20.0, h=25.0, t_inf=20.0,
                 q0=1e7, sigma=0.1, dt=1.0)
TRANSIENT_FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


def transient_source(x, y, z):
    """Gaussian heat source of peak q0 at the box centre."""
    p = TRANSIENT_PARAMS
    r2 = (np.asarray(x) - 0.5) ** 2 + (np.asarray(y) - 0.5) ** 2 + (np.asarray(z) - 0.5) ** 2
    return p["q0"] * np.exp(-r2 / (2.0 * p["sigma"] ** 2))


def transient_robin():
    return {f: (TRANSIENT_PARAMS["h"], TRANSIENT_PARAMS["t_inf"]) for f in TRANSIENT_FACES}


def _transient_device_march(dm, mesh, precision, n_steps, rtol):
    """Pattern + K, C, F and Robin terms + theta march on resident inputs;
    returns the final field on the device and the per-step solve records."""
    from cloudfem_b200 import _native as N
    from cloudfem_b200._driver import last_solve_info, theta_march
    from cloudfem_b200.fem.tet_heat import _terms, add_into
    p = TRANSIENT_PARAMS
    dm._pattern = None
    K, F = dm.assemble(N.OP_P1_STIFF, coef=p["k"], load=transient_source)
    K_add, F_add, _ = _terms(dm, mesh, None, transient_robin())
    K = add_into(dm, K, K_add)
    F = F + F_add
    C, _ = dm.assemble(N.OP_P1_MASS, coef=p["rho_cp"])
    empty = np.zeros(0, dtype=np.int64)
    _, T = theta_march(dm, K, C, F, empty, np.zeros(0), n_steps * p["dt"],
                       n_steps, p["t0"], 0.5, precision, rtol,
                       keep_history=False)
    return T, last_solve_info()


def run_transient_heat(args, rank, world, local_rank):
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200.device import DeviceMesh
    from cloudfem_b200.fem.tet_heat import transient_heat_tet
    from cloudfem_b200.mesh import box_mesh

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    _set_scheduler(rt, args.scheduler)
    n = args.transient_n
    n_steps = args.transient_steps
    mesh = box_mesh(n, n, n)
    dm = DeviceMesh(mesh, local_rank)
    free = mesh.n_nodes                       # Robin everywhere: no fixed DOF
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    rtol = args.transient_rtol or (1e-10 if args.precision == "mixed" else 1e-12)

    # accuracy gate: the first 20 steps in both precisions
    gate = min(20, n_steps)
    T64, _ = _transient_device_march(dm, mesh, "fp64", gate, 1e-12)
    T64 = T64.clone()
    Tm, _ = _transient_device_march(dm, mesh, args.precision, gate, rtol)
    gate_err = float(torch.linalg.norm(Tm - T64) / torch.linalg.norm(T64))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _transient_device_march(dm, mesh, "fp64", gate, 1e-12)
    torch.cuda.synchronize()
    fp64_s = time.perf_counter() - t0

    for _ in range(args.warmup):
        _transient_device_march(dm, mesh, args.precision, min(10, n_steps), rtol)
    torch.cuda.synchronize()
    times, l0 = [], rt.launches()
    _barrier(world)
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            T, infos = _transient_device_march(dm, mesh, args.precision, n_steps, rtol)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    _barrier(world)
    launches = rt.launches() - l0
    its = [r.iterations for r in infos]
    spmv = [r.spmv_ms for r in infos if r.spmv_samples]

    # end to end through the public API: host mesh in, host history out
    e2e = []
    _barrier(world)
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        transient_heat_tet(mesh, k=TRANSIENT_PARAMS["k"], rho_cp=TRANSIENT_PARAMS["rho_cp"],
                           f=transient_source, robin=transient_robin(),
                           t_end=n_steps * TRANSIENT_PARAMS["dt"], dt=TRANSIENT_PARAMS["dt"],
                           T0=TRANSIENT_PARAMS["t0"], method="cn",
                           precision=args.precision, rtol=rtol)
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    _barrier(world)
    ms, e2e_mean = _max_over_ranks(world, [np.sum(times), np.mean(e2e)])
    if rank != 0:
        return None
    dof_steps = free * n_steps
    pat = dm.pattern
    sz = 4 if args.precision == "mixed" else 8
    spmv_b = pat.nnz * (sz + 4) + 4 * (mesh.n_nodes + 1) + 2 * sz * mesh.n_nodes
    peak, peak_kind = _peaks()
    out = {
        "metric": METRIC,
        "value": world * dof_steps * args.steps / (ms * 1e-3),
        "unit": "DOF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 PCG + f64 residual/update" if args.precision == "mixed" else "f64",
        "data": "synthetic (structured Kuhn P1 box, analytic Gaussian source)",
        "config": {
            "workload": f"transient_p1_heat_cn_box_{n}cubed_{n_steps}_steps",
            "nodes": int(mesh.n_nodes), "elements": int(len(mesh.elements)),
            "nnz": int(pat.nnz), "time_steps": n_steps, "free_dofs": int(free),
            "precision": args.precision, "rtol_per_step": rtol,
            "cg_iterations_per_step_mean": float(np.mean(its)),
            "cg_iterations_per_step_max": int(max(its)),
            "rel_err_vs_fp64_after_20_steps": gate_err,
            "fp64_plain_20_steps": {"dof_per_s": free * gate / fp64_s},
            "l2": "256 MiB buffer written between timed steps",
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": world * dof_steps / (e2e_mean * 1e-3),
                "unit": "DOF/s",
                "h2d_bytes_per_step": int(mesh.nodes.nbytes + mesh.elements.nbytes),
                "d2h_bytes_per_step": int((n_steps + 1) * mesh.n_nodes * 8),
                "note": "transient_heat_tet: host mesh in, full host history out"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if spmv:
        ach = spmv_b / (float(np.mean(spmv)) * 1e-3) / 1e9
        out["roofline"] = {
            "kernel": _scalar_spmv_kernel(rt, args.precision) + " (scalar PCG SpMV phase: q = A p, p.q)",
            "bound": "hbm", "achieved": ach, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": ach / peak, "bytes_per_launch": int(spmv_b),
            "launch_ms": float(np.mean(spmv)),
            # DRAM bytes per launch from the committed ncu summary (FP32 staged
            # kernel, captured at 112^3 and scaled by nonzeros)
            "traffic": (_profiled_traffic("k_gxs_transient_p1_heat_128cubed", "fp32")
                        if args.precision == "mixed" else None),
        }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_transient_heat()
    return out


def cpu_baseline_transient_heat(n=32, n_steps=20):
    """Oracle (NumPy assembly + SciPy LU, factorised once) on a small box."""
    from oracle import cfem_oracle as O
    p = TRANSIENT_PARAMS
    t0 = time.perf_counter()
    m = O.box_mesh(n, n, n)
    O.transient_heat_p1(m, k=p["k"], rho_cp=p["rho_cp"], f=transient_source,
                        robin=transient_robin(), t_end=n_steps * p["dt"], dt=p["dt"],
                        T0=p["t0"], method="cn")
    dt = time.perf_counter() - t0
    free = (n + 1) ** 3
    return {"value": free * n_steps / dt, "unit": "DOF/s", "cores": os.cpu_count(),
            "kind": "port", "seconds": dt,
            "sample": f"box {n}^3 ({free} nodes), {n_steps} CN steps incl. assembly"}


# ------------------------------------------------ Tet10 A-V eddy currents
AV_N = 10
AV_SIGMA, AV_FREQ = 1.0e6, 1000.0


def av_js(x, y, z):
    """Complex source current density of the phasor A-V workload."""
    s = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    return np.array([(1.0 + 2.0j) * 1e9 * s, 0.5e9 * s * (1.0 + x), 0.3j * 1e9 * y * z])


def _av_kw():
    return dict(nu=1.0 / (4e-7 * np.pi), sigma=AV_SIGMA, omega=2.0 * np.pi * AV_FREQ,
                J_s=av_js, boundary=["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"])


def cpu_baseline_av(nb=8):
    """Oracle (NumPy + SuperLU) phasor A-V solve on a box of nb^3 cells."""
    from oracle import cfem_oracle as O
    mo = O.box_mesh_tet10(nb, nb, nb)
    t0 = time.perf_counter()
    O.solve_eddy_current_tet10(mo, **_av_kw())
    dt = time.perf_counter() - t0
    fb = len(np.unique(np.concatenate([mo.boundaries[f] for f in _av_kw()["boundary"]])))
    ub = 3 * (mo.n_nodes - fb)
    return {"value": ub / dt, "unit": "DOF/s", "cores": os.cpu_count(),
            "kind": "port", "seconds": dt,
            "sample": f"box {nb}^3 (~{ub} A unknowns), SuperLU"}


def run_av(args, rank, world, local_rank):
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics import em3d_tet10 as em

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    n = args.av_n
    mesh = box_mesh_tet10(n, n, n)
    for _ in range(args.warmup):
        em.solve_eddy_current_tet10(mesh, **_av_kw())
    walls, kms, l0 = [], [], rt.launches()
    _barrier(world)
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            a, v = em.solve_eddy_current_tet10(mesh, **_av_kw())
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
            kms.append(em.last_solve_info()["kernel_ms"])
    _barrier(world)
    launches = rt.launches() - l0
    info = em.last_solve_info()
    ms, wall_mean = _max_over_ranks(world, [np.mean(kms), np.mean(walls)])
    if rank != 0:
        return None
    fixed = len(np.unique(np.concatenate([mesh.boundaries[f] for f in _av_kw()["boundary"]])))
    n_v = int(np.count_nonzero(v))     # V unknowns: conductor nodes but the pinned one
    unknowns = 3 * (mesh.n_nodes - fixed) + n_v
    out = {
        "metric": METRIC, "value": world * unknowns / (ms * 1e-3), "unit": "DOF/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic (Tet10 box, manufactured source current)",
        "config": {"workload": f"phasor_av_tet10_box_{n}cubed", "unknowns": int(unknowns),
                   "cocg_iterations": info["iterations"], "relres": info["relres"],
                   "sigma": AV_SIGMA, "freq_hz": AV_FREQ,
                   "note": "value: COCG on the device-resident eliminated system; "
                           "e2e: the public call (device blocks, host block "
                           "combination and elimination, device COCG)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * unknowns / wall_mean, "unit": "DOF/s",
                "h2d_bytes_per_step": int(mesh.nodes.nbytes + mesh.elements.nbytes),
                "d2h_bytes_per_step": int(16 * (3 * mesh.n_nodes + mesh.n_nodes))},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_av()
    return out


AVT_STEPS = 50


def _avt_kw(steps=AVT_STEPS):
    return dict(nu=1.0 / (4e-7 * np.pi), sigma=AV_SIGMA, t_end=steps * 1e-4, dt=1e-4,
                method="cn", J_s=lambda x, y, z: np.real(av_js(x, y, z)),
                time_scale=lambda t: np.sin(2 * np.pi * 500.0 * t),
                boundary=["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"])


def cpu_baseline_avt(nb=8, steps=AVT_STEPS):
    """Oracle transient A-V march (one LU, then the steps) on nb^3 cells."""
    from oracle import cfem_oracle as O
    kw = _avt_kw(steps)
    mo = O.box_mesh_tet10(nb, nb, nb)
    t0 = time.perf_counter()
    O.transient_eddy_current_tet10(mo, **kw)
    dt = time.perf_counter() - t0
    fb = len(np.unique(np.concatenate([mo.boundaries[f] for f in kw["boundary"]])))
    ub = 3 * (mo.n_nodes - fb)
    return {"value": ub * steps / dt, "unit": "DOF/s", "cores": os.cpu_count(),
            "kind": "port", "seconds": dt,
            "sample": f"box {nb}^3, {steps} CN steps, one LU"}


def run_avt(args, rank, world, local_rank):
    """Transient A-V eddy currents: conducting Tet10 box, sinusoidal source,
    Crank-Nicolson, one device PCG solve per step (a conductor in gauge-
    regularised air is a parity case; with Jacobi it needs thousands of
    iterations per step at this size)."""
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics import em3d_tet10 as em

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    n, steps = args.av_n, AVT_STEPS
    kw = _avt_kw(steps)
    mesh = box_mesh_tet10(n, n, n)
    for _ in range(args.warmup):
        em.transient_eddy_current_tet10(mesh, precision=args.precision, rtol=1e-10, **kw)
    walls, l0 = [], rt.launches()
    _barrier(world)
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = em.transient_eddy_current_tet10(mesh, precision=args.precision, rtol=1e-10, **kw)
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
    _barrier(world)
    launches = rt.launches() - l0
    (wall,) = _max_over_ranks(world, [np.mean(walls)])
    if rank != 0:
        return None
    fixed = len(np.unique(np.concatenate([mesh.boundaries[f] for f in kw["boundary"]])))
    unknowns = 3 * (mesh.n_nodes - fixed)
    out = {
        "metric": METRIC, "value": world * unknowns * steps / wall, "unit": "DOF/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32 PCG + f64 residual/update",
        "data": "synthetic (conducting Tet10 box, sinusoidal source current)",
        "config": {"workload": f"transient_av_tet10_box_{n}cubed_{steps}_cn_steps",
                   "a_unknowns": int(unknowns), "time_steps": steps,
                   "note": "value and e2e: the public call, A-block DOF-steps per second "
                           "(device blocks, A and V solves and Joule power; fields copied "
                           "back once at the end)",
                   "P_last": float(r["P"][-1]), "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * unknowns * steps / wall, "unit": "DOF/s",
                "h2d_bytes_per_step": int(mesh.nodes.nbytes + mesh.elements.nbytes),
                "d2h_bytes_per_step": int(((steps + 1) + 4 * mesh.n_nodes) * 8)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_avt(steps=steps)
    return out


# ---------------------------------------------------- serving a request stream
SERVE_REQUESTS = 200


def _cell_coef(mesh, k_elem):
    """A per-element coefficient of a box mesh (6 tets per hex cell, cells
    in k, j, i order, unit cell width 1 / ny as the request stream builds
    them) as the callable(x, y, z) the reference's API takes: the value of
    the hex cell holding the point (centroids and Keast points are interior,
    so the lookup is exact)."""
    corners = np.asarray(mesh.nodes)[np.unique(np.asarray(mesh.elements)[:, :4])]
    nx, ny, nz = (len(np.unique(np.round(corners[:, d], 9))) - 1 for d in range(3))
    lo = corners.min(axis=0)
    hi = corners.max(axis=0)
    kc = np.asarray(k_elem, dtype=float)[::6].reshape(nz, ny, nx)

    def k(x, y, z):
        i = np.clip(((np.asarray(x) - lo[0]) / (hi[0] - lo[0]) * nx).astype(int), 0, nx - 1)
        j = np.clip(((np.asarray(y) - lo[1]) / (hi[1] - lo[1]) * ny).astype(int), 0, ny - 1)
        kk = np.clip(((np.asarray(z) - lo[2]) / (hi[2] - lo[2]) * nz).astype(int), 0, nz - 1)
        return kc[kk, j, i]
    return k


def cpu_baseline_serving(count=12, cap_dofs=6e3, seed=7):
    """Oracle (NumPy + SuperLU, the reference's one-request-at-a-time path)
    on the first `count` requests of the seeded stream drawn with at most
    `cap_dofs` DOFs; DOF/s over their free DOFs. The cap keeps SuperLU
    within memory: the reference's Dirichlet step stores the cleared
    columns as explicit zeros (a dense free x fixed block), which at 25 k
    P1 DOFs already exhausts its workspace here."""
    from cloudfem_b200 import serve
    from oracle import cfem_oracle as O
    stream = serve.make_stream(SERVE_REQUESTS, rate=200.0, seed=seed, max_dofs=cap_dofs)
    picked = stream[:count]
    free, kinds, t0 = 0, {}, time.perf_counter()
    for r in picked:
        m = O.Mesh(r.mesh.nodes, r.mesh.elements, r.mesh.boundaries)
        if r.kind == "t10_elast":
            O.solve_elasticity_tet10(m, r.E, r.nu, bc={c: (0.0, 0.0, 0.0) for c in r.clamp},
                                     traction=r.traction)
        else:
            solve = O.solve_p1_poisson if r.kind == "p1_heat" else O.solve_tet10_poisson
            solve(m, k=_cell_coef(r.mesh, r.k), f=r.f, bc=r.bc)
        free += serve.free_dofs(r)
        kinds[r.kind] = kinds.get(r.kind, 0) + 1
    dt = time.perf_counter() - t0
    mix = ", ".join(f"{v} {k}" for k, v in sorted(kinds.items()))
    return {"value": free / dt, "unit": "DOF/s", "cores": os.cpu_count(),
            "kind": "port", "seconds": dt,
            "sample": f"the first {len(picked)} requests of the seeded stream drawn with at most "
                      f"{int(cap_dofs)} DOFs ({mix}; {free} free DOFs), one solve each"}


def run_serving(args, rank, world, local_rank):
    import torch

    from cloudfem_b200 import _native as N
    from cloudfem_b200 import serve

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rt = N.runtime(local_rank)
    _set_scheduler(rt, args.scheduler)
    cache = {}
    stream = serve.make_stream(args.serve_requests, rate=200.0, seed=7,
                               mesh_cache=cache)

    def fresh():
        for r in stream:
            r.result = r.info = r.t_start = r.t_done = None
        return stream

    # warm-up on a short stream of small requests (kernels, pools)
    warm = serve.make_stream(30, rate=2000.0, dof_range=(1e3, 2e4), seed=1)
    serve.Server(local_rank, precision=args.precision, rtol=args.serve_rtol).serve(warm, realtime=False)

    # end to end: a new server, every mesh arrives with its request (H2D,
    # pattern build, assembly, solve, D2H per request)
    torch.cuda.synchronize()
    e2e = serve.Server(local_rank, precision=args.precision, rtol=args.serve_rtol).serve(fresh())
    # resident: the same stream again on that server's warm device meshes
    srv = serve.Server(local_rank, precision=args.precision, rtol=args.serve_rtol)
    srv.serve(fresh(), realtime=False)
    runs = []
    for _ in range(args.warmup):
        srv.serve(fresh())
    l0 = rt.launches()
    _barrier(world)
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            runs.append(srv.serve(fresh()))
    _barrier(world)
    launches = rt.launches() - l0
    mixed_sol = {r.id: r.result for r in stream}
    # give the resident server's device meshes (up to the HBM budget) back
    # before the comparison paths build their own
    workers = srv.workers
    del srv
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    rt.trim()

    # plain FP64 GPU path: one request at a time, unbatched, FP64, to the
    # same tolerance, on the first requests of the stream; accuracy of the
    # served answers against a tight FP64 solve of each
    plain = serve.Server(local_rank, workers=1, precision="fp64", rtol=args.serve_rtol)
    sub = [r for r in fresh()[: min(40, len(stream))]]
    for r in sub[:2]:
        plain.run_batch([r])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_dofs = 0
    for r in sub:
        plain.run_batch([r])
        plain_dofs += serve.free_dofs(r)
    plain_s = time.perf_counter() - t0
    tight = serve.Server(local_rank, workers=1, precision="fp64", rtol=1e-12)
    errs = []
    for r in sub:
        sol, _ = tight.run_batch([r])
        x = mixed_sol[r.id]
        errs.append(float(np.linalg.norm(x - sol[0]) / max(np.linalg.norm(sol[0]), 1e-300)))
    best = max(runs, key=lambda d: d["dof_per_s"])
    med = sorted(runs, key=lambda d: d["dof_per_s"])[len(runs) // 2]
    # the slowest replica's throughputs (MAX of the negated rates)
    neg = _max_over_ranks(world, [-med["dof_per_s"], -e2e["dof_per_s"]])
    med_dps, e2e_dps = -neg[0], -neg[1]
    if rank != 0:
        return None
    out = {
        "metric": METRIC, "value": world * med_dps, "unit": "DOF/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean([d["span_s"] for d in runs])) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 PCG + f64 residual/update" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded Poisson request stream of box meshes)",
        "config": {
            "workload": f"serving_stream_{len(stream)}_requests_lambda200",
            "mix": "60% P1 heat / 25% Tet10 heat / 15% Tet10 elasticity",
            "dof_range": [1e3, 2e6], "hbm_budget_gb": 150, "workers": workers,
            "rtol": args.serve_rtol,
            "requests": len(stream), "solved_dofs": med["solved_dofs"],
            "p50_ms": med["p50_ms"], "p99_ms": med["p99_ms"], "max_ms": med["max_ms"],
            "by_kind": med["by_kind"],
            "best_run_dof_per_s": best["dof_per_s"],
            "plain_fp64_unbatched": {"requests": len(sub),
                                     "dof_per_s": plain_dofs / plain_s},
            "rel_err_vs_fp64_plain_max": max(errs),
            "resident": "device meshes kept from an earlier pass of the stream",
            "l2": "inputs larger than L2 (batch matrices)",
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": world * e2e_dps, "unit": "DOF/s",
                "p50_ms": e2e["p50_ms"], "p99_ms": e2e["p99_ms"],
                # nodes in FP64 and connectivity as the int32 the device
                # copy holds (the host converts before the copy)
                "h2d_bytes_per_step": int(sum(r.mesh.nodes.nbytes + 4 * np.asarray(r.mesh.elements).size
                                              for r in stream)),
                "d2h_bytes_per_step": int(sum(r.dofs * 8 for r in stream)),
                "note": "new server: every mesh crosses with its request"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_serving()
    return out


def run_reference(args, rank):
    if rank != 0:
        return None
    per = []
    if args.workload == "batched-heat":
        draw = batch_draw()
    for i in range(args.warmup + args.steps):
        if args.workload == "batched-heat":
            c = cpu_baseline_batched_heat(*draw)
        elif args.workload == "transient-heat":
            c = cpu_baseline_transient_heat()
        elif args.workload == "serving":
            c = cpu_baseline_serving()
        elif args.workload == "av-phasor":
            c = cpu_baseline_av()
        elif args.workload == "av-transient":
            c = cpu_baseline_avt()
        else:
            c = cpu_baseline()
        if i >= args.warmup:
            per.append(c)
    value = float(np.mean([c["value"] for c in per]))
    c = per[-1]
    c["value"] = value
    return {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "DOF/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": float(np.mean([c["seconds"] for c in per])) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if args.workload == "av-phasor" else "f64", "data": "synthetic",
        "config": {"workload": {"batched-heat": "batched_tet10_heat_512_meshes_n4to24",
                                "transient-heat": f"transient_p1_heat_cn_box_{TRANSIENT_N}cubed_{TRANSIENT_STEPS}_steps",
                                "serving": f"serving_stream_{SERVE_REQUESTS}_requests_lambda200",
                                "av-phasor": f"phasor_av_tet10_box_{AV_N}cubed",
                                "av-transient": f"transient_av_tet10_box_{AV_N}cubed_{AVT_STEPS}_cn_steps",
                                }.get(args.workload, "tet10_elasticity_beam_80x10x10"),
                   "sample": c["sample"]},
        "cpu_baseline": c,
        "e2e": {"value": value, "unit": "DOF/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["mixed", "fp64"],
                    help="default: fp64 for the elasticity beam and the A-V transient, "
                         "mixed otherwise")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--one-pass", action="store_true",
                    help="batched-heat: one assembly and one mixed solve of the batch and "
                         "exit without a line (for per-launch profilers)")
    ap.add_argument("--workload", default="batched-heat",
                    choices=["elasticity", "batched-heat", "transient-heat", "serving",
                             "av-phasor", "av-transient"],
                    help="batched-heat: 512 seeded Tet10 heat meshes, mixed "
                         "precision against the plain FP64 path (default); "
                         "elasticity: Tet10 elasticity beam 80x10x10; "
                         "transient-heat: P1 heat, 128^3 box, 200 Crank-Nicolson "
                         "steps; serving: stream of 200 mixed requests; "
                         "av-phasor / av-transient: Tet10 A-V eddy currents, 10^3 box")
    ap.add_argument("--av-n", type=int, default=AV_N,
                    help="av-phasor / av-transient: cells per box edge")
    ap.add_argument("--serve-rtol", type=float, default=1e-8,
                    help="serving: relative residual each request is solved to")
    ap.add_argument("--serve-requests", type=int, default=SERVE_REQUESTS,
                    help="serving: requests in the stream")
    ap.add_argument("--scheduler", default="auto",
                    choices=["auto", "persistent", "graph", "polled"],
                    help="solver scheduler (polled: host-polled graph replays, "
                         "for per-launch profiling)")
    ap.add_argument("--transient-n", type=int, default=TRANSIENT_N,
                    help="transient-heat: cells per box edge")
    ap.add_argument("--transient-rtol", type=float, default=None,
                    help="transient-heat: relative residual per time step (default 1e-10 "
                         "mixed, 1e-12 FP64)")
    ap.add_argument("--transient-steps", type=int, default=TRANSIENT_STEPS,
                    help="transient-heat: time steps per bench step")
    ap.add_argument("--meshes", type=int, default=BATCH_MESHES,
                    help="batched-heat: number of meshes of the seeded draw (a smaller "
                         "batch of the same kind, e.g. for profiling)")
    ap.add_argument("--spmv-stage", type=int, default=None, choices=[0, 1, 2, 3, 4],
                    help="SpMV: 1 scalar rows bulk-staged through shared memory, 3x3 "
                         "blocks in registers; 2 both staged; 0 both in registers; 3 "
                         "scalar and 3x3 rows in the sliced-ELL layout (one row per "
                         "lane); 4 per precision and block size (library default)")
    ap.add_argument("--sell-sort", type=int, default=None, choices=[0, 1],
                    help="sliced-ELL SpMV: 1 sort each 256-row window by row length, "
                         "0 keep rows in order (default: the library's)")
    ap.add_argument("--sell3-lanes", type=int, default=None, choices=[1, 2, 4],
                    help="sliced-ELL SpMV of 3x3 blocks: lanes per block row (default: "
                         "the library's)")
    ap.add_argument("--sell3-staged", type=int, default=None, choices=[0, 1, 2],
                    help="sliced-ELL SpMV of 3x3 blocks: 1 streams slices through shared "
                         "memory with bulk copies, 0 loads them into registers, 2 streams "
                         "FP32 slices only (default: the library's)")
    ap.add_argument("--slot-sell3", type=int, default=None, choices=[0, 1],
                    help="serving: 3x3 solve slots in the sliced-ELL layout (1) or the "
                         "entry-major copy (0) (default: the library's)")
    args = ap.parse_args()
    global SPMV_STAGE, SELL_SORT, SELL3_LANES, SELL3_STAGED, SLOT_SELL3
    SLOT_SELL3 = args.slot_sell3
    SPMV_STAGE = args.spmv_stage
    SELL_SORT = args.sell_sort
    SELL3_LANES = args.sell3_lanes
    SELL3_STAGED = args.sell3_staged
    if args.precision is None:
        args.precision = "fp64" if args.workload in ("elasticity", "av-transient") else "mixed"
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl",
                                    timeout=datetime.timedelta(seconds=300))
        if args.workload == "batched-heat":
            out = run_batched_heat(args, rank, world, local_rank)
        elif args.workload == "transient-heat":
            out = run_transient_heat(args, rank, world, local_rank)
        elif args.workload == "serving":
            out = run_serving(args, rank, world, local_rank)
        elif args.workload == "av-phasor":
            out = run_av(args, rank, world, local_rank)
        elif args.workload == "av-transient":
            out = run_avt(args, rank, world, local_rank)
        else:
            out = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
