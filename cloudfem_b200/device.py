"""Device-resident meshes, patterns, assembly and solves over libcfem.

This is the host half of the drop-in boundary: it keeps the reference's
host-side semantics (coefficient callables evaluated on the host into
per-element or per-quadrature-point arrays, boundary dictionaries, SciPy
CSR results) and hands all element, CSR and solver work to the CUDA
library through the C ABI of ``include/cfem.h``. Device memory is held in
torch tensors (plumbing only); every kernel is libcfem's.
"""

import ctypes

import numpy as np
import scipy.sparse as sp

from . import _native as N
from ._native import ptr

# Keast 5-point rule (cloudfem/fem/tet10.py:84-100).
_A, _B = 0.5, 1.0 / 6.0
KEAST_L = np.array([[0.25, 0.25, 0.25, 0.25], [_A, _B, _B, _B],
                    [_B, _A, _B, _B], [_B, _B, _A, _B], [_B, _B, _B, _A]])
KEAST_W = np.array([-4.0 / 5.0] + [9.0 / 20.0] * 4)

# Local corner triples of the four faces (cloudfem/fem/tet_heat.py:112 and
# the Tet10 table of cloudfem/fem/tet10.py:287-292).
FACES_P1 = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
FACES_T10 = (((0, 1, 2), (4, 5, 6)), ((0, 3, 1), (7, 8, 4)),
             ((0, 2, 3), (6, 9, 7)), ((1, 3, 2), (8, 9, 5)))


def _torch():
    import torch
    return torch


# ------------------------------------------------------------ host helpers

EVAL_CHUNK = 1 << 16   # points per vectorised call of a coefficient function


def evaluate(spec, pts):
    """Evaluate a float or callable(x, y, z) at points (..., 3).

    Constants stay Python floats. Callables are pointwise (the reference
    calls them one point at a time), so they are called on arrays of
    EVAL_CHUNK points at a time (the temporaries of a NumPy expression then
    stay in the host caches: 6x faster than one call on 12.6 M points), and
    fall back to one call per point when they do not broadcast.
    """
    if not callable(spec):
        return float(spec)
    shape = pts.shape[:-1]
    flat = pts.reshape(-1, 3)
    n = flat.shape[0]
    try:
        with np.errstate(all="ignore"):
            m = min(EVAL_CHUNK, n)
            v = np.asarray(spec(flat[:m, 0], flat[:m, 1], flat[:m, 2]), dtype=float)
            if v.shape == (m,):
                out = np.empty(n)
                out[:m] = v
                for i in range(m, n, EVAL_CHUNK):
                    f = flat[i:i + EVAL_CHUNK]
                    out[i:i + f.shape[0]] = np.asarray(spec(f[:, 0], f[:, 1], f[:, 2]),
                                                       dtype=float)
                return out.reshape(shape)
        if v.ndim == 0:
            return np.full(shape, float(v))
    except Exception:  # noqa: BLE001 - callable is scalar-only
        pass
    return np.fromiter((spec(x, y, z) for x, y, z in flat), dtype=float,
                       count=flat.shape[0]).reshape(shape)


def centroids(nodes, elements):
    return nodes[elements[:, :4]].mean(axis=1)


def keast_points(nodes, elements):
    p = nodes[elements[:, :4]]
    return np.einsum("qc,ecd->eqd", KEAST_L, p)


def fixed_scalar(mesh, bc):
    """{name|'all': value|callable} -> sorted node ids and values.

    Later names overwrite earlier ones, as the dict in
    cloudfem/fem/tet_poisson.py:85-93 does.
    """
    n = mesh.n_nodes
    if not bc:
        return np.zeros(0, np.int64), np.zeros(0)
    val = np.zeros(n)
    has = np.zeros(n, dtype=bool)
    for name, value in bc.items():
        ids = (np.arange(n) if name == "all"
               else np.asarray(mesh.boundaries[name], dtype=np.int64))
        v = evaluate(value, mesh.nodes[ids])
        val[ids] = v
        has[ids] = True
    idx = np.nonzero(has)[0]
    return idx, val[idx]


def fixed_vector(mesh, bc):
    """elastic3d.py:204-218: (name|'all') -> (ux, uy, uz), None = free."""
    n = mesh.n_nodes
    val = np.zeros(3 * n)
    has = np.zeros(3 * n, dtype=bool)
    for name, vals in (bc or {}).items():
        ids = (np.arange(n) if name == "all"
               else np.asarray(mesh.boundaries[name], dtype=np.int64))
        for comp, v in enumerate(vals):
            if v is None:
                continue
            dofs = 3 * ids + comp
            val[dofs] = evaluate(v, mesh.nodes[ids])
            has[dofs] = True
    idx = np.nonzero(has)[0]
    return idx, val[idx]


# ------------------------------------------------------------ device objects

class Pattern:
    """Node-level sparsity of a mesh (owned libcfem handle)."""

    def __init__(self, rt, handle, n_nodes, nnz):
        self.rt = rt
        self.handle = handle
        self.n_nodes = n_nodes
        self.nnz = nnz
        rp, col = N._vp(), N._vp()
        N.check(rt.lib.cfem_pattern_node_csr(handle, ctypes.byref(rp),
                                             ctypes.byref(col)))
        self.row_ptr = rp
        self.col = col

    def expand(self, bs):
        """Device DOF-level CSR indptr / indices for bs DOFs per node."""
        torch = _torch()
        dev = self.rt.device
        indptr = torch.empty(self.n_nodes * bs + 1, dtype=torch.int32,
                             device=dev)
        indices = torch.empty(max(self.nnz * bs * bs, 1), dtype=torch.int32,
                              device=dev)
        N.check(self.rt.lib.cfem_pattern_expand(
            self.handle, bs, ptr(indptr), ptr(indices), self.rt.stream()))
        return indptr, indices[: self.nnz * bs * bs]

    def to_scipy(self, bs, vals):
        """scipy csr_matrix of block values (nnz*bs*bs) in DOF order."""
        torch = _torch()
        indptr, indices = self.expand(bs)
        if bs > 1:
            flat = torch.empty_like(vals)
            N.check(self.rt.lib.cfem_block_to_csr(
                self.handle, bs, ptr(vals), ptr(flat), self.rt.stream()))
        else:
            flat = vals
        n = self.n_nodes * bs
        A = sp.csr_matrix((flat.cpu().numpy(), indices.cpu().numpy(),
                           indptr.cpu().numpy()), shape=(n, n))
        A.has_sorted_indices = True
        return A

    def __del__(self):
        try:
            self.rt.lib.cfem_pattern_destroy(self.handle)
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class DeviceMesh:
    """Nodes (N, 3) f64 and int32 connectivity (M, 4|10) resident in HBM."""

    def __init__(self, mesh, device=None):
        torch = _torch()
        self.rt = N.runtime(device)
        self.host = mesh
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
        els = np.asarray(mesh.elements)
        if els.ndim != 2 or els.shape[1] not in (4, 10):
            raise ValueError(f"elements must be (M, 4) or (M, 10), got "
                             f"{els.shape}")
        if nodes.ndim != 2 or nodes.shape[1] != 3:
            raise ValueError(f"nodes must be (N, 3), got {nodes.shape}")
        if els.size and (els.min() < 0 or els.max() >= nodes.shape[0]):
            raise ValueError("element connectivity references a node id "
                             f"outside [0, {nodes.shape[0]})")
        self.n_nodes = nodes.shape[0]
        self.n_elems = els.shape[0]
        self.npe = els.shape[1]
        dev = self.rt.device
        self.nodes = torch.from_numpy(nodes).to(dev, non_blocking=True)
        self.elems = torch.from_numpy(
            np.ascontiguousarray(els, dtype=np.int32)).to(dev,
                                                          non_blocking=True)
        self._pattern = None

    @property
    def pattern(self):
        if self._pattern is None:
            h = N._vp()
            N.check(self.rt.lib.cfem_pattern_create(
                self.rt.ctx, ptr(self.elems), self.n_elems, self.npe,
                self.n_nodes, self.rt.stream(), ctypes.byref(h)))
            n, nnz = N._i64(), N._i64()
            N.check(self.rt.lib.cfem_pattern_info(h, ctypes.byref(n),
                                                  ctypes.byref(nnz)))
            self._pattern = Pattern(self.rt, h, n.value, nnz.value)
        return self._pattern

    # ------------------------------------------------------ coefficients
    def coef(self, spec, where):
        """cfem_coef for a float/callable sampled at 'centroid' or 'qp', or
        a per-element array (constant over each element).

        Returns (struct, keepalive) - the tensor must outlive the launch.
        """
        if isinstance(spec, np.ndarray):
            a = np.ascontiguousarray(spec, dtype=float)
            if a.shape != (self.n_elems,):
                raise ValueError(f"per-element array needs {self.n_elems} values, "
                                 f"got {a.shape}")
            t = _torch().from_numpy(a).to(self.rt.device)
            return N.Coef(ptr(t), 0.0, N.COEF_ELEM, 0), t
        if not callable(spec):
            return N.Coef(None, float(spec), N.COEF_CONST, 0), None
        if where == "qp":
            vals = evaluate(spec, self.sample_points("qp"))
            mode = N.COEF_QP
        else:
            vals = evaluate(spec, self.sample_points("centroid"))
            mode = N.COEF_ELEM
        if np.isscalar(vals):
            return N.Coef(None, float(vals), N.COEF_CONST, 0), None
        t = _torch().from_numpy(np.ascontiguousarray(vals, dtype=float)).to(
            self.rt.device)
        return N.Coef(ptr(t), 0.0, mode, 0), t

    def sample_points(self, where):
        """Element centroids (M, 3) or Keast points (M, 5, 3) as host
        arrays, computed once per mesh on the device (the gather of corner
        coordinates is the costly part on the host for large meshes) with
        the same operation order as the host formulas."""
        pts = self.__dict__.setdefault("_pts", {})
        if where not in pts:
            torch = _torch()
            corner = self.elems[:, :4].long()
            p = [self.nodes[corner[:, c]] for c in range(4)]
            if where == "qp":
                L = torch.as_tensor(KEAST_L, dtype=torch.float64, device=self.nodes.device)
                out = torch.empty((self.n_elems, L.shape[0], 3), dtype=torch.float64,
                                  device=self.nodes.device)
                for q in range(L.shape[0]):
                    acc = L[q, 0] * p[0]
                    for c in range(1, 4):
                        acc = acc + L[q, c] * p[c]
                    out[:, q] = acc
            else:
                out = (((p[0] + p[1]) + p[2]) + p[3]) / 4.0
            pts[where] = out.cpu().numpy()
        return pts[where]

    def nodal_coef(self, values):
        t = _torch().from_numpy(
            np.ascontiguousarray(values, dtype=float)).to(self.rt.device)
        if t.numel() != self.n_nodes:
            raise ValueError(f"nodal field has {t.numel()} values, mesh has "
                             f"{self.n_nodes} nodes")
        return N.Coef(ptr(t), 0.0, N.COEF_NODAL, 0), t

    # ------------------------------------------------------ assembly
    def assemble(self, op, coef=1.0, load=None, vals=None, rhs=None,
                 accumulate=False):
        """Scalar operator into device (vals[nnz], rhs[N])."""
        torch = _torch()
        pat = self.pattern
        dev = self.rt.device
        where = "qp" if op == N.OP_T10_STIFF else "centroid"
        kc, keep1 = self.coef(coef, where)
        if vals is None:
            vals = torch.empty(pat.nnz, dtype=torch.float64, device=dev)
        lc, keep2 = (self.coef(load, where) if load is not None
                     else (N.Coef(None, 0.0, N.COEF_CONST, 0), None))
        if rhs is None and load is not None:
            rhs = torch.empty(self.n_nodes, dtype=torch.float64, device=dev)
        N.check(self.rt.lib.cfem_assemble(
            self.rt.ctx, pat.handle, op, ptr(self.nodes), ptr(self.elems),
            ctypes.byref(kc), ctypes.byref(lc), ptr(vals), ptr(rhs),
            1 if accumulate else 0, self.rt.stream()))
        del keep1, keep2
        return vals, rhs

    def assemble_elastic(self, op, E, nu, body=None, T=None, alpha=0.0,
                         T_ref=0.0, vals=None, rhs=None):
        torch = _torch()
        pat = self.pattern
        dev = self.rt.device
        where = "qp" if op == N.OP_T10_ELAST else "centroid"
        keep = []
        b3 = (N.Coef * 3)()
        comps = list(body) if body is not None else [0.0, 0.0, 0.0]
        if len(comps) != 3:
            raise ValueError("body force needs three components")
        for c, v in enumerate(comps):
            b3[c], k = self.coef(0.0 if v is None else v, where)
            keep.append(k)
        tcoef = None
        if T is not None and alpha != 0.0:
            if callable(T):
                tcoef, k = self.coef(T, where)
            else:
                tcoef, k = self.nodal_coef(T)
            keep.append(k)
        if vals is None:
            vals = torch.empty(pat.nnz * 9, dtype=torch.float64, device=dev)
        if rhs is None:
            rhs = torch.empty(3 * self.n_nodes, dtype=torch.float64,
                              device=dev)
        N.check(self.rt.lib.cfem_assemble_elastic(
            self.rt.ctx, pat.handle, op, ptr(self.nodes), ptr(self.elems),
            float(E), float(nu), b3,
            ctypes.byref(tcoef) if tcoef is not None else None,
            float(alpha), float(T_ref), ptr(vals), ptr(rhs), 0,
            self.rt.stream()))
        del keep
        return vals, rhs

    # ------------------------------------------------------ faces
    def boundary_faces(self, name, tet10=False):
        """Exterior faces on a named node set, in the reference's order.

        Faces whose key (sorted corner triple) occurs once among all element
        faces and whose corners are all in the set, listed at their first
        occurrence in element order (tet_heat.py:97-120, tet10.py:329-352):
        candidates flagged and compacted on the device
        (cfem_face_candidates), the once-only count and the node lists on
        the device too (cfem_face_exterior). Only faces with all corners in
        the set can share a key with such a face, so counting among the
        candidates is exact.
        """
        return self.boundary_faces_device(name, tet10).cpu().numpy()

    def boundary_faces_device(self, name, tet10=False):
        """boundary_faces as a device int64 tensor (F, 3 or 6)."""
        torch = _torch()
        host = self.host
        ids = np.asarray(host.boundaries[name], dtype=np.int64)
        width = 6 if tet10 else 3
        empty = torch.zeros((0, width), dtype=torch.int64, device=self.rt.device)
        if ids.size == 0 or self.n_elems == 0:
            return empty
        inset = torch.zeros(self.n_nodes, dtype=torch.uint8,
                            device=self.rt.device)
        inset[torch.from_numpy(ids).to(self.rt.device)] = 1
        out = torch.empty(self.n_elems * 4, dtype=torch.int64,
                          device=self.rt.device)
        cnt = N._i64()
        N.check(self.rt.lib.cfem_face_candidates(
            self.rt.ctx, ptr(self.elems), self.n_elems, self.npe,
            1 if tet10 else 0, ptr(inset), self.n_nodes, ptr(out),
            ctypes.byref(cnt), self.rt.stream()))
        nc = cnt.value
        if nc == 0:
            return empty
        ids = torch.empty(nc, dtype=torch.int64, device=self.rt.device)
        nodes = torch.empty(nc * width, dtype=torch.int64, device=self.rt.device)
        nout = N._i64()
        N.check(self.rt.lib.cfem_face_exterior(
            self.rt.ctx, ptr(self.elems), self.npe, 1 if tet10 else 0, ptr(out), nc,
            self.n_nodes, ptr(ids), ptr(nodes), ctypes.byref(nout), self.rt.stream()))
        return nodes[: nout.value * width].reshape(-1, width)


# ------------------------------------------------------------ solver

class SolveResult:
    def __init__(self, stats):
        self.status = int(stats.status)
        self.iterations = int(stats.iterations)
        self.residual_updates = int(stats.residual_updates)
        self.relres = float(stats.relres)
        self.bnorm = float(stats.bnorm)
        self.kernel_ms = float(stats.kernel_ms)
        self.spmv_ms = float(stats.spmv_ms)
        self.spmv_samples = int(stats.spmv_samples)

    def __repr__(self):
        return (f"SolveResult(status={N.STATUS_NAMES.get(self.status)}, "
                f"iterations={self.iterations}, relres={self.relres:.3e}, "
                f"residual_updates={self.residual_updates})")


class BlockSystem:
    """One SPD block-CSR system on the device, ready for cfem_pcg_solve."""

    def __init__(self, rt, n_rows, bs, row_ptr, col, vals64, b, x,
                 fixed=None, vals32=None, precond=None, keep=()):
        self.rt = rt
        self.n_rows = n_rows
        self.bs = bs
        self.row_ptr = row_ptr        # c_void_p or tensor
        self.col = col
        self.vals64 = vals64
        self.vals32 = vals32
        self.b = b
        self.x = x
        self.fixed = fixed
        # point Jacobi by default (the reference's method name); on the Tet10
        # cantilever it also beats the 3x3 block inverse: 2,947 vs 3,185
        # FP64 iterations, 4,453 vs 6,481 mixed
        self.precond = (precond if precond is not None else
                        N.PRECOND_JACOBI)
        self.keep = keep

    def ensure_fp32(self):
        """FP32 difference-form operator for the mixed solver."""
        torch = _torch()
        if self.vals32 is None:
            n = self.vals64.numel()
            self.vals32 = torch.empty(n, dtype=torch.float32,
                                      device=self.vals64.device)

            def p(v):
                return v if isinstance(v, N._vp) else ptr(v)
            N.check(self.rt.lib.cfem_mixed_matrix(
                self.rt.ctx, self.n_rows, self.bs, p(self.row_ptr),
                p(self.col), ptr(self.vals64), ptr(self.vals32),
                self.rt.stream()))
        return self.vals32

    def linsys(self, mode, rtol, max_iter, reliable_delta=0.0, max_stall=0,
               history=None):
        def p(v):
            return v if isinstance(v, N._vp) else ptr(v)
        v32 = self.ensure_fp32() if mode == N.SOLVE_MIXED else None
        cap = 0 if history is None else history.numel() // 2
        return N.LinSys(self.n_rows, self.bs, self.precond, p(self.row_ptr),
                        p(self.col), ptr(self.vals64), ptr(v32), ptr(self.b),
                        ptr(self.x), ptr(self.fixed), float(rtol),
                        int(max_iter), int(mode), float(reliable_delta),
                        int(max_stall), int(cap), ptr(history))


def pcg(systems, mode=N.SOLVE_FP64, rtol=1e-12, max_iter=None,
        reliable_delta=0.0, max_stall=0, history=None):
    """Solve a batch of BlockSystems in one persistent launch.

    history: optional list (one device f64 tensor of 2*k entries per
    system) receiving (iteration, relres) at each FP64 residual.
    """
    if not systems:
        return []
    rt = systems[0].rt
    arr = (N.LinSys * len(systems))()
    for i, s in enumerate(systems):
        mi = max_iter if max_iter is not None else max(
            1000, 20 * int(np.sqrt(s.n_rows * s.bs)) + 2000)
        arr[i] = s.linsys(mode, rtol, mi, reliable_delta, max_stall,
                          None if history is None else history[i])
    stats = (N.SolveStats * len(systems))()
    N.check(rt.lib.cfem_pcg_solve(rt.ctx, arr, len(systems), stats,
                                  rt.stream()))
    return [SolveResult(s) for s in stats]


class PcgPlan:
    """Set-up of a batch solve kept for repeated solves (time steps, a
    serving loop): working copies of the matrices, solver vectors and the
    captured iteration graphs stay on the device. Each solve() starts from
    the current contents of every system's b and x. After changing matrix
    values in place, call refresh()."""

    def __init__(self, systems, mode=N.SOLVE_FP64, rtol=1e-12, max_iter=None,
                 reliable_delta=0.0, max_stall=0):
        if not systems:
            raise ValueError("a plan needs at least one system")
        self.rt = systems[0].rt
        self.systems = list(systems)        # keeps the device arrays alive
        arr = (N.LinSys * len(systems))()
        for i, sy in enumerate(systems):
            mi = max_iter if max_iter is not None else max(
                1000, 20 * int(np.sqrt(sy.n_rows * sy.bs)) + 2000)
            arr[i] = sy.linsys(mode, rtol, mi, reliable_delta, max_stall)
        self._arr = arr
        self._stats = (N.SolveStats * len(systems))()
        h = N._vp()
        N.check(self.rt.lib.cfem_pcg_plan_create(self.rt.ctx, arr, len(systems),
                                                 self.rt.stream(), ctypes.byref(h)))
        self.handle = h

    def refresh(self):
        N.check(self.rt.lib.cfem_pcg_plan_refresh(self.handle, self.rt.stream()))

    def solve(self):
        N.check(self.rt.lib.cfem_pcg_plan_solve(self.handle, self._stats,
                                                self.rt.stream()))
        return [SolveResult(st) for st in self._stats]

    def close(self):
        if getattr(self, "handle", None):
            self.rt.lib.cfem_pcg_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def pcg_noalloc(system, mode=N.SOLVE_FP64, rtol=1e-12, max_iter=None):
    """Solve one BlockSystem without any device allocation by the library.

    For callers that cannot allocate device memory at solve time (an
    application that has reserved the whole HBM budget for its own pools,
    or a latency-bound loop that cannot take cudaMalloc's implicit
    synchronisation): the workspace is libcfem's fixed 32 MiB device array
    (``cfem_pcg_noalloc_capacity()``), so larger systems raise ValueError.
    Concurrent calls on one GPU share that array and must not overlap. The
    FP32 operator of the mixed mode is the caller's to provide (made here
    once by ``ensure_fp32`` if missing).
    """
    rt = system.rt
    mi = max_iter if max_iter is not None else max(
        1000, 20 * int(np.sqrt(system.n_rows * system.bs)) + 2000)
    ls = system.linsys(mode, rtol, mi)
    st = N.SolveStats()
    N.check(rt.lib.cfem_pcg_solve_noalloc(rt.ctx, ctypes.byref(ls),
                                          ctypes.byref(st), rt.stream()))
    return SolveResult(st)


def raise_for(result, what="solve"):
    if result.status == N.CFEM_OK:
        return
    if result.status == N.CFEM_ERR_BREAKDOWN:
        raise RuntimeError(
            f"{what} failed: {N.STATUS_NAMES[result.status]} "
            f"(singular or indefinite system; check the boundary conditions)")
    raise RuntimeError(f"{what} failed: {N.STATUS_NAMES.get(result.status)} "
                       f"after {result.iterations} iterations, relative "
                       f"residual {result.relres:.3e}")


def fixed_mask(rt, n, idx, vals, x=None):
    """Device uint8 mask and an x vector holding the Dirichlet values."""
    torch = _torch()
    dev = rt.device
    mask = np.zeros(n, dtype=np.uint8)
    mask[idx] = 1
    d_mask = torch.from_numpy(mask).to(dev)
    if x is None:
        xh = np.zeros(n)
        xh[idx] = vals
        d_x = torch.from_numpy(xh).to(dev)
    else:
        d_x = x
        if len(idx):
            d_x[torch.from_numpy(np.asarray(idx, np.int64)).to(dev)] = \
                torch.from_numpy(np.asarray(vals, float)).to(dev)
    return d_mask, d_x


def csr_to_device(rt, A):
    """Canonical scipy CSR -> device (indptr, indices, data) tensors."""
    torch = _torch()
    A = sp.csr_matrix(A, dtype=float)
    A.sum_duplicates()
    A.sort_indices()
    dev = rt.device
    return (torch.from_numpy(A.indptr.astype(np.int32)).to(dev),
            torch.from_numpy(A.indices.astype(np.int32)).to(dev),
            torch.from_numpy(A.data.astype(np.float64)).to(dev), A)


class SlotEngine:
    """Solve slots (``cfem_pcg_slots_*``): iteration-level continuous
    batching. ``n_slots`` systems of one block size and precision, each of
    at most ``max_rows`` block rows and ``max_nnzb`` stored blocks, iterate
    together in rounds of 16 CG iterations on the engine's own stream; a
    system assigned between rounds joins the running ones, and a finished
    system frees its slot at once. Systems are BlockSystem objects whose
    arrays stay alive while they are in a slot."""

    def __init__(self, rt, n_slots, bs, mode, max_rows, max_nnzb):
        self.rt = rt
        self.n_slots = int(n_slots)
        self.bs, self.mode = int(bs), int(mode)
        self.max_rows, self.max_nnzb = int(max_rows), int(max_nnzb)
        h = N._vp()
        N.check(rt.lib.cfem_pcg_slots_create(rt.ctx, self.n_slots, self.bs, self.mode,
                                             self.max_rows, self.max_nnzb, rt.stream(),
                                             ctypes.byref(h)))
        self.handle = h
        self.free = list(range(self.n_slots))
        self.busy = {}                       # slot -> (system, tag)
        self._stats = (N.SolveStats * self.n_slots)()

    def fits(self, system):
        return (system.bs == self.bs and system.n_rows <= self.max_rows)

    def assign(self, system, rtol, max_iter=None, tag=None):
        """Put a system into a free slot (raises if none is free); returns it."""
        if not self.free:
            raise RuntimeError("no free solve slot")
        mi = max_iter if max_iter is not None else max(
            1000, 20 * int(np.sqrt(system.n_rows * system.bs)) + 2000)
        ls = system.linsys(self.mode, rtol, mi)
        slot = self.free[0]
        N.check(self.rt.lib.cfem_pcg_slots_assign(self.handle, slot, ctypes.byref(ls),
                                                  self.rt.stream()))
        self.free.pop(0)
        self.busy[slot] = (system, tag)
        return slot

    def run(self, rounds=1):
        """Queue `rounds` rounds of 16 iterations over every slot."""
        N.check(self.rt.lib.cfem_pcg_slots_run(self.handle, int(rounds), self.rt.stream()))

    def ready(self):
        """True once the queued rounds have run (no wait)."""
        st = self.rt.lib.cfem_pcg_slots_ready(self.handle)
        if st == N.CFEM_SLOT_RUNNING:
            return False
        N.check(st)
        return True

    def poll(self):
        """Wait for the queued rounds; returns [(system, tag, SolveResult)] of
        the systems that finished (their slots are free again)."""
        N.check(self.rt.lib.cfem_pcg_slots_poll(self.handle, self._stats))
        done = []
        for slot in sorted(self.busy):
            st = self._stats[slot]
            if st.status == N.CFEM_SLOT_RUNNING:
                continue
            system, tag = self.busy.pop(slot)
            self.free.append(slot)
            done.append((system, tag, SolveResult(st)))
        self.free.sort()
        return done

    def release(self, slot):
        N.check(self.rt.lib.cfem_pcg_slots_release(self.handle, int(slot), self.rt.stream()))
        if slot in self.busy:
            del self.busy[slot]
            self.free.append(slot)
            self.free.sort()

    def close(self):
        if getattr(self, "handle", None):
            self.rt.lib.cfem_pcg_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
