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

    def prepare(self, problems):
        """Device inputs of every problem; returns a Batch."""
        import torch
        dev = self.rt.device
        items, keep = [], []
        for pb in problems:
            dm = self.device_mesh(pb.mesh)
            kc, t1 = self._coef(dm, pb.k)
            fc, t2 = self._coef(dm, pb.f)
            keep += [t1, t2]
            idx, v = fixed_scalar(pb.mesh, pb.bc)
            mask = np.zeros(dm.n_nodes, dtype=np.uint8)
            mask[idx] = 1
            x0 = np.zeros(dm.n_nodes)
            x0[idx] = v
            item = {
                "dm": dm, "coef": kc, "load": fc,
                "vals": torch.empty(dm.pattern.nnz, dtype=torch.float64, device=dev),
                "rhs": torch.empty(dm.n_nodes, dtype=torch.float64, device=dev),
                "mask": torch.from_numpy(mask).to(dev, non_blocking=True),
                "x0": torch.from_numpy(x0).to(dev, non_blocking=True),
                "free": int(dm.n_nodes - len(idx)),
            }
            item["x"] = item["x0"].clone()
            items.append(item)
        return Batch(self, items, keep)


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

    def solve(self, precision="mixed", rtol=None, max_iter=None, fresh=True):
        """One batched PCG over every problem; returns SolveResult list."""
        mode, rtol = solver_mode(precision, rtol)
        systems = []
        for it in self.items:
            if fresh:
                it["x"].copy_(it["x0"])
            dm = it["dm"]
            pat = dm.pattern
            sysm = BlockSystem(self.rt, dm.n_nodes, 1, pat.row_ptr, pat.col,
                               it["vals"], it["rhs"], it["x"], it["mask"])
            it["system"] = sysm
            systems.append(sysm)
        self.results = pcg(systems, mode, rtol, max_iter)
        for i, r in enumerate(self.results):
            accept(r, rtol, f"batched solve of problem {i}")
        return self.results

    def solutions(self):
        return [it["x"].cpu().numpy() for it in self.items]


def solve_batch(problems, precision="mixed", rtol=None, max_iter=None,
                solver=None):
    """Assemble and solve a list of HeatProblem; returns nodal solutions."""
    solver = solver or BatchSolver()
    batch = solver.prepare(problems)
    batch.assemble()
    batch.solve(precision, rtol, max_iter)
    return batch.solutions()
