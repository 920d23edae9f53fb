"""Batched assembly and solution of many independent scalar heat problems.

The reference solves one mesh per call (``cloudfem/fem/tet10.py:168-178``,
``cloudfem/fem/tet_poisson.py:113-122``). Here a list of problems - each a
mesh, a conductivity k, a source f and a Dirichlet dict - is assembled by
one batched element / reduction launch per pass (``cfem_assemble_batch``)
and solved by one batched PCG (``cfem_pcg_solve``: every system advances in
the same kernels; each keeps its own scalars and convergence test).

Meshes are device-resident and shared: problems that use the same mesh
object reuse its connectivity, pattern and boundary mask (meshes are treated
as immutable while cached; ``BatchSolver.clear()`` drops the cache).
"""

import numpy as np

from . import _native as N
from ._driver import accept, solver_mode
from .device import BlockSystem, DeviceMesh, evaluate, fixed_scalar
from .device import pcg, ptr

OPS = {4: N.OP_P1_STIFF, 10: N.OP_T10_STIFF}


class HeatProblem:
    """-div(k grad u) = f on `mesh` with Dirichlet data `bc`.

    k, f: float, callable(x, y, z), or an array with one value per element
    (sampled where the reference samples: centroids for Tet4, each Keast
    point of the element for Tet10 - a per-element array means the value is
    constant over the element).
    """

    def __init__(self, mesh, k=1.0, f=0.0, bc=None):
        self.mesh = mesh
        self.k = k
        self.f = f
        self.bc = bc or {}


class BatchSolver:
    def __init__(self, device=None):
        self.rt = N.runtime(device)
        self._meshes = {}
        self._fixed = {}

    def clear(self):
        self._meshes.clear()
        self._fixed.clear()

    def device_mesh(self, mesh):
        key = id(mesh)
        ent = self._meshes.get(key)
        if ent is None or ent[0] is not mesh:
            dm = DeviceMesh(mesh, self.rt.device)
            dm.pattern  # noqa: B018 - build now
            self._meshes[key] = (mesh, dm)
            return dm
        return ent[1]

    def _coef(self, dm, spec):
        import torch
        if isinstance(spec, np.ndarray):
            a = np.ascontiguousarray(spec, dtype=float)
            if a.shape != (dm.n_elems,):
                raise ValueError(f"per-element array needs {dm.n_elems} values, "
                                 f"got {a.shape}")
            t = torch.from_numpy(a).to(self.rt.device, non_blocking=True)
            return N.Coef(ptr(t), 0.0, N.COEF_ELEM, 0), t
        if not callable(spec):
            return N.Coef(None, float(spec), N.COEF_CONST, 0), None
        if dm.npe == 10:
            vals, mode = evaluate(spec, dm.sample_points("qp")), N.COEF_QP
        else:
            vals, mode = evaluate(spec, dm.sample_points("centroid")), N.COEF_ELEM
        if np.isscalar(vals):
            return N.Coef(None, float(vals), N.COEF_CONST, 0), None
        t = torch.from_numpy(np.ascontiguousarray(vals, dtype=float)).to(
            self.rt.device, non_blocking=True)
        return N.Coef(ptr(t), 0.0, mode, 0), t

    def _dirichlet(self, dm, mesh, bc):
        """Device mask and initial guess holding the Dirichlet values, cached
        per mesh for constant-valued bc dicts; (mask, x0, free count)."""
        import torch
        key = None
        if all(not callable(v) for v in (bc or {}).values()):
            key = (id(mesh), tuple(sorted((k, float(v)) for k, v in (bc or {}).items())))
            hit = self._fixed.get(key)
            if hit is not None and hit[0] is mesh:
                return hit[1:]
        idx, v = fixed_scalar(mesh, bc)
        mask = np.zeros(dm.n_nodes, dtype=np.uint8)
        mask[idx] = 1
        x0 = np.zeros(dm.n_nodes)
        x0[idx] = v
        out = (torch.from_numpy(mask).to(self.rt.device, non_blocking=True),
               torch.from_numpy(x0).to(self.rt.device, non_blocking=True),
               int(dm.n_nodes - len(idx)))
        if key is not None:
            self._fixed[key] = (mesh,) + out
        return out

    def prepare(self, problems):
        """Device inputs of every problem; returns a Batch. Per-element
        coefficient arrays cross in one pinned copy; matrix values, loads and
        solutions live in one allocation each."""
        import torch
        dev = self.rt.device
        dms = [self.device_mesh(pb.mesh) for pb in problems]
        packed = []
        for i, (pb, dm) in enumerate(zip(problems, dms)):
            for which in ("k", "f"):
                spec = getattr(pb, which)
                if isinstance(spec, np.ndarray):
                    a = np.ascontiguousarray(spec, dtype=float)
                    if a.shape != (dm.n_elems,):
                        raise ValueError(f"per-element array needs {dm.n_elems} "
                                         f"values, got {a.shape}")
                    packed.append((i, which, a))
        keep = []
        dev_arrays = {}
        total = sum(a.size for _, _, a in packed)
        if total:
            host = torch.empty(total, dtype=torch.float64, pin_memory=True)
            hv = host.numpy()
            off, offs = 0, []
            for _, _, a in packed:
                hv[off:off + a.size] = a
                offs.append(off)
                off += a.size
            dbuf = host.to(dev, non_blocking=True)
            keep += [host, dbuf]
            for (i, which, a), o in zip(packed, offs):
                dev_arrays[(i, which)] = dbuf[o:o + a.size]
        nnz = [dm.pattern.nnz for dm in dms]
        nn = [dm.n_nodes for dm in dms]
        vals_all = torch.empty(max(sum(nnz), 1), dtype=torch.float64, device=dev)
        rhs_all = torch.empty(max(sum(nn), 1), dtype=torch.float64, device=dev)
        fixed = [self._dirichlet(dm, pb.mesh, pb.bc) for pb, dm in zip(problems, dms)]
        x0_all = torch.cat([f[1] for f in fixed]) if fixed else rhs_all[:0]
        x_all = x0_all.clone()
        items = []
        ov = on = 0
        for i, (pb, dm) in enumerate(zip(problems, dms)):
            coefs = []
            for which in ("k", "f"):
                t = dev_arrays.get((i, which))
                if t is not None:
                    coefs.append(N.Coef(ptr(t), 0.0, N.COEF_ELEM, 0))
                else:
                    c, t2 = self._coef(dm, getattr(pb, which))
                    keep.append(t2)
                    coefs.append(c)
            mask, x0, free = fixed[i]
            items.append({
                "dm": dm, "coef": coefs[0], "load": coefs[1],
                "vals": vals_all[ov:ov + nnz[i]], "rhs": rhs_all[on:on + nn[i]],
                "mask": mask, "x0": x0_all[on:on + nn[i]], "x": x_all[on:on + nn[i]],
                "free": free,
            })
            ov += nnz[i]
            on += nn[i]
        batch = Batch(self, items, keep)
        batch.x_all, batch.x0_all = x_all, x0_all
        return batch


class Batch:
    def __init__(self, solver, items, keep):
        self.solver = solver
        self.rt = solver.rt
        self.items = items
        self.keep = keep
        self.results = []

    @property
    def free_dofs(self):
        return sum(it["free"] for it in self.items)

    def assemble(self):
        """One cfem_assemble_batch call per element type."""
        for npe, op in OPS.items():
            sel = [it for it in self.items if it["dm"].npe == npe]
            if not sel:
                continue
            jobs = (N.AssemblyJob * len(sel))()
            for i, it in enumerate(sel):
                dm = it["dm"]
                jobs[i] = N.AssemblyJob(dm.pattern.handle, ptr(dm.nodes),
                                        ptr(dm.elems), it["coef"], it["load"],
                                        ptr(it["vals"]), ptr(it["rhs"]))
            N.check(self.rt.lib.cfem_assemble_batch(
                self.rt.ctx, op, jobs, len(sel), self.rt.stream()))

    def _mixed_operators(self):
        """FP32 difference-form operators of every problem from the current
        FP64 values, in one launch (cfem_mixed_matrix_batch); the FP32
        arrays are kept between solves."""
        import torch
        jobs = (N.MixedJob * len(self.items))()
        for i, it in enumerate(self.items):
            if it.get("vals32") is None:
                it["vals32"] = torch.empty(it["vals"].numel(), dtype=torch.float32,
                                           device=it["vals"].device)
            pat = it["dm"].pattern
            jobs[i] = N.MixedJob(it["dm"].n_nodes, 1, 0, pat.row_ptr, pat.col,
                                 ptr(it["vals"]), ptr(it["vals32"]))
        N.check(self.rt.lib.cfem_mixed_matrix_batch(self.rt.ctx, jobs, len(self.items),
                                                    self.rt.stream()))

    def solve(self, precision="mixed", rtol=None, max_iter=None, fresh=True):
        """One batched PCG over every problem; returns SolveResult list."""
        mode, rtol = solver_mode(precision, rtol)
        if mode == N.SOLVE_MIXED:
            self._mixed_operators()
        systems = []
        x_all = getattr(self, "x_all", None)
        if fresh and x_all is not None:
            x_all.copy_(self.x0_all)
        for it in self.items:
            if fresh and x_all is None:
                it["x"].copy_(it["x0"])
            dm = it["dm"]
            pat = dm.pattern
            sysm = BlockSystem(self.rt, dm.n_nodes, 1, pat.row_ptr, pat.col,
                               it["vals"], it["rhs"], it["x"], it["mask"],
                               vals32=it.get("vals32") if mode == N.SOLVE_MIXED else None)
            it["system"] = sysm
            systems.append(sysm)
        self.results = pcg(systems, mode, rtol, max_iter)
        for i, r in enumerate(self.results):
            accept(r, rtol, f"batched solve of problem {i}")
        return self.results

    def solutions(self):
        """Host copies of every problem's solution (one device-to-host copy)."""
        x_all = getattr(self, "x_all", None)
        if x_all is None:
            return [it["x"].cpu().numpy() for it in self.items]
        h = x_all.cpu().numpy()
        out, o = [], 0
        for it in self.items:
            n = it["dm"].n_nodes
            out.append(h[o:o + n].copy())
            o += n
        return out


def solve_batch(problems, precision="mixed", rtol=None, max_iter=None,
                solver=None):
    """Assemble and solve a list of HeatProblem; returns nodal solutions."""
    solver = solver or BatchSolver()
    batch = solver.prepare(problems)
    batch.assemble()
    batch.solve(precision, rtol, max_iter)
    return batch.solutions()
