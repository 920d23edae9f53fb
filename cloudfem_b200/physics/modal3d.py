"""Natural frequencies of P1 tetrahedral solids with the solves on the GPU.

Drop-in for cloudfem/physics/modal3d.py:

* ``assemble_mass_3d`` (:40-75): consistent mass rho V / 20 (1 + delta_ij)
  per component, or the row-sum lumped diagonal rho V / 4; the element
  matrices are the P1 capacity kernel's, reduced into the node pattern on
  the device and returned with the reference's CSR structure (entries
  between the same component of two nodes only);
* ``solve_modes_3d`` (:100-156): the lowest eigenpairs of K phi = w^2 M phi
  on the free DOFs by shift-invert Lanczos (SciPy's ARPACK driver, as the
  reference), where every application of (K - sigma M)^-1 is one FP64
  Jacobi-PCG solve on the device (a solve plan on the node block pattern,
  constrained DOFs masked) in place of the reference's sparse LU, and the
  products with M are device SpMVs. K and M stay on the device.
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .. import _native as N
from .._driver import accept, solver_mode
from ..device import BlockSystem, DeviceMesh, PcgPlan, fixed_mask, ptr
from .elastic3d import _assemble

__all__ = ["assemble_mass_3d", "solve_modes_3d"]


def _mass_values(dm, rho, lumped):
    """Node-level mass values (consistent) or nodal lumped masses (device)."""
    import torch
    if not lumped:
        vals, _ = dm.assemble(N.OP_P1_MASS, coef=float(rho))
        return vals
    # row sums of the consistent matrix are rho V / 4 per node of each
    # element; summed on the host in the reference's element order
    vols = dm.host.element_volumes()
    diag = np.zeros(dm.n_nodes)
    np.add.at(diag, np.asarray(dm.host.elements).ravel(),
              np.repeat(rho * vols / 4.0, 4))
    return torch.from_numpy(diag).to(dm.rt.device)


def _diag_positions(dm):
    """Device indices of the diagonal entries of the node pattern."""
    import torch
    rp, ci = dm.pattern.expand(1)
    rp = rp.cpu().numpy().astype(np.int64)
    ci = ci.cpu().numpy().astype(np.int64)
    row_of = np.repeat(np.arange(dm.n_nodes), np.diff(rp))
    return torch.from_numpy(np.nonzero(ci == row_of)[0]).to(dm.rt.device)


def _componentwise_csr(dm, vals):
    """(3N, 3N) CSR with entry (3i+c, 3j+c) = m_ij for each component c."""
    indptr, indices = dm.pattern.expand(1)
    ip = indptr.cpu().numpy().astype(np.int64)
    ix = indices.cpu().numpy().astype(np.int64)
    v = vals.cpu().numpy()
    n = dm.n_nodes
    lens = np.diff(ip)
    out_ptr = np.concatenate([[0], np.cumsum(np.repeat(lens, 3))])
    row_of = np.repeat(np.arange(n), lens)
    rank = np.arange(len(ix)) - ip[row_of]
    out_idx = np.empty(3 * len(ix), dtype=np.int64)
    out_val = np.empty(3 * len(ix))
    for c in range(3):
        pos = out_ptr[3 * row_of + c] + rank
        out_idx[pos] = 3 * ix + c
        out_val[pos] = v
    A = sp.csr_matrix((out_val, out_idx.astype(np.int32), out_ptr.astype(np.int32)),
                      shape=(3 * n, 3 * n))
    A.has_sorted_indices = True
    return A


def assemble_mass_3d(mesh, rho, lumped=False):
    """Mass matrix (3N, 3N) csr, DOF order ux0, uy0, uz0, ux1, ..."""
    dm = DeviceMesh(mesh)
    vals = _mass_values(dm, rho, lumped)
    if lumped:
        return sp.diags(np.repeat(vals.cpu().numpy(), 3), format="csr")
    return _componentwise_csr(dm, vals)


def _fixed_dofs(mesh, bc):
    """Constrained DOFs of a bc dict (a component not None is fixed;
    modal3d.py:78-97)."""
    fixed = set()
    for name, vals in bc.items():
        ids = np.arange(mesh.n_nodes) if name == "all" else np.asarray(mesh.boundaries[name])
        for comp, v in enumerate(vals):
            if v is not None:
                fixed.update((3 * np.asarray(ids, dtype=np.int64) + comp).tolist())
    return np.array(sorted(fixed), dtype=int)


class _ModalOperators:
    """Device K and M (node block pattern), the shifted operator K - sigma M
    with a solve plan, and products with M, all on the free DOFs."""

    def __init__(self, mesh, E, nu, rho, lumped, fixed, sigma_fn):
        import torch
        self.dm = dm = DeviceMesh(mesh)
        rt = dm.rt
        K, _ = _assemble(dm, mesh, N.OP_P1_ELAST, E, nu, None, None, None, 0.0, 0.0, False)
        m = _mass_values(dm, rho, lumped)
        pat = dm.pattern
        n3 = 3 * dm.n_nodes
        # M as 3x3 blocks (m_ij I) on the node pattern: lumped masses on the
        # diagonal entries only
        Mb = torch.zeros(pat.nnz, 3, 3, dtype=torch.float64, device=rt.device)
        if lumped:
            diag = self._diag_positions()
            for c in range(3):
                Mb[diag, c, c] = m
        else:
            for c in range(3):
                Mb[:, c, c] = m
        self.M = Mb.reshape(-1)
        Kd = torch.diagonal(K.view(-1, 3, 3), dim1=1, dim2=2)
        Md = torch.diagonal(Mb, dim1=1, dim2=2)
        diag = self._diag_positions()
        free = np.ones(n3, dtype=bool)
        free[fixed] = False
        fmask = torch.from_numpy(free.reshape(-1, 3)).to(rt.device)
        kd = Kd[diag][fmask]
        md = Md[diag][fmask]
        self.sigma = sigma_fn(float(kd.mean()) / float(md.mean()))
        self.A = (K - self.sigma * self.M).contiguous()
        self.n3 = n3
        self.free = np.nonzero(free)[0]
        self.mask, self.x = fixed_mask(rt, n3, fixed, np.zeros(len(fixed)))
        self.b = torch.zeros(n3, dtype=torch.float64, device=rt.device)
        self.y = torch.zeros(n3, dtype=torch.float64, device=rt.device)
        mode, self.rtol = solver_mode("fp64", 1e-13)
        sysA = BlockSystem(rt, dm.n_nodes, 3, pat.row_ptr, pat.col, self.A, self.b,
                           self.x, self.mask)
        self.plan = PcgPlan([sysA], mode, self.rtol)
        self.solves = 0

    def _diag_positions(self):
        return _diag_positions(self.dm)

    def _full(self, v):
        import torch
        full = np.zeros(self.n3)
        full[self.free] = v
        return torch.from_numpy(full).to(self.dm.rt.device)

    def solve(self, v):
        """(K - sigma M)^-1 v on the free DOFs: one device PCG solve."""
        self.b.copy_(self._full(v))
        self.x.zero_()
        res = self.plan.solve()
        accept(res[0], self.rtol, "shift-invert solve")
        self.solves += 1
        return self.x.cpu().numpy()[self.free]

    def mass(self, v):
        """M v on the free DOFs (device SpMV)."""
        rt, pat = self.dm.rt, self.dm.pattern
        x = self._full(v)
        N.check(rt.lib.cfem_spmv(rt.ctx, self.dm.n_nodes, 3, pat.row_ptr, pat.col,
                                 ptr(self.M), 1.0, ptr(x), 0.0, ptr(self.y), rt.stream()))
        return self.y.cpu().numpy()[self.free]

    def close(self):
        self.plan.close()


def solve_modes_3d(mesh, E, nu, rho, bc=None, n_modes=6, lumped=False):
    """Lowest n_modes natural frequencies [Hz] and M-orthonormal mode shapes
    (3N, n_modes), zero at constrained DOFs (modal3d.py:100-156)."""
    n3 = 3 * mesh.n_nodes
    fixed = _fixed_dofs(mesh, bc) if bc else np.zeros(0, dtype=int)
    n_free = n3 - len(fixed)
    if not 0 < n_modes < n_free:
        raise ValueError(f"n_modes={n_modes} must be in [1, {n_free})")
    # the reference's shift: just below zero on the Rayleigh scale of the
    # free diagonals, so K - sigma M stays definite for free-free bodies
    ops = _ModalOperators(mesh, E, nu, rho, lumped, fixed, lambda scale: -1e-8 * scale)
    try:
        shape = (n_free, n_free)
        OPinv = spla.LinearOperator(shape, matvec=ops.solve, dtype=float)
        Mop = spla.LinearOperator(shape, matvec=ops.mass, dtype=float)
        Aop = spla.LinearOperator(shape, matvec=lambda v: v, dtype=float)  # shape only
        ncv = min(n_free, max(2 * n_modes + 2, 24))
        vals, vecs = spla.eigsh(Aop, M=Mop, k=n_modes, sigma=ops.sigma, which="LM",
                                mode="normal", OPinv=OPinv, tol=1e-10, maxiter=10000,
                                ncv=ncv)
        order = np.argsort(vals)
        vals, vecs = vals[order], vecs[:, order]
        for j in range(n_modes):
            vecs[:, j] /= np.sqrt(vecs[:, j] @ ops.mass(vecs[:, j]))
    finally:
        ops.close()
    modes = np.zeros((n3, n_modes))
    modes[ops.free, :] = vecs
    return np.sqrt(np.clip(vals, 0.0, None)) / (2.0 * np.pi), modes
