"""Generate the configuration-scale golden fixtures by running the reference.

Usage (from the repository root)::

    python tests/golden/make_config_golden.py /path/to/CloudFEM

The reference (zhangkalin627-svg/CloudFEM) is imported unchanged from the
given checkout and run on the benchmark configurations of ``cases.py`` at
sizes it finishes in minutes on the host cores:

* C1 exactly: P1 20^3 steady heat (pre-BC stiffness, load, solution);
* C3 subset: seeded Tet10 unit cubes with n in ``C3_GOLDEN_NS`` and
  lognormal per-cell conductivity (solutions);
* C4 at n = 32: P1 Crank-Nicolson march, 20 steps (fields after steps 1
  and 20);
* C2 at quarter resolution (40 x 5 x 5 Tet10 cantilever): the reference's
  SuperLU solution, plus the same system's solution after iterative
  refinement with residuals accumulated in extended precision
  (``np.longdouble``), which the CUDA path's error is measured against
  because this beam's condition number puts the plain SuperLU answer's own
  error near 1e-11.

Output: ``config_fixtures.npz`` next to this script. Nothing at test time
reads the reference itself.
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases as C  # noqa: E402


def refine_ext(A, b, x, solve, steps=4):
    """x <- x + solve(b - A x) with the residual summed in long double."""
    A = A.tocsr()
    Al = A.astype(np.longdouble)
    bl = np.asarray(b, dtype=np.longdouble)
    x = np.asarray(x, dtype=float).copy()
    hist = []
    for _ in range(steps):
        r = bl - Al @ x.astype(np.longdouble)
        hist.append(float(np.linalg.norm(r.astype(float)) / np.linalg.norm(b)))
        x = x + solve(r.astype(float))
    return x, hist


def main(ref_path):
    sys.path.insert(0, ref_path)
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    from cloudfem.fem import tet10 as t10
    from cloudfem.fem import tet_heat as th
    from cloudfem.fem import tet_poisson as tp
    from cloudfem.mesh.tet10_mesh import box_mesh_tet10
    from cloudfem.mesh.tet_mesh import box_mesh
    from cloudfem.physics import elastic3d as e3
    from cloudfem.physics import elastic_tet10 as e10

    out = {}
    t_start = time.time()

    def put(name, arr):
        out[name] = np.asarray(arr)

    def put_csr(name, A):
        A = A.tocsr()
        put(name + "__indptr", A.indptr.astype(np.int32))
        put(name + "__indices", A.indices.astype(np.int32))
        put(name + "__data", A.data)
        put(name + "__shape", np.array(A.shape, dtype=np.int64))

    def log(msg):
        print(f"[{time.time() - t_start:7.1f} s] {msg}", flush=True)

    allfaces = {s: 0.0 for s in C.FACES}

    # C1 exactly
    m = box_mesh(C.C1_N, C.C1_N, C.C1_N)
    A, b = tp.assemble(m, k=1.0, f=C.f_sss)
    put_csr("c1_K", A)
    put("c1_F", b)
    put("c1_u", tp.solve_tet_poisson(m, k=1.0, f=C.f_sss, bc=allfaces))
    log("C1 done")

    # C3 seeded subset
    ks = C.c3_draw(C.C3_GOLDEN_NS)
    for n, kc in zip(C.C3_GOLDEN_NS, ks):
        mt = box_mesh_tet10(n, n, n)
        kf = C.c3_cell_fn(n, kc)
        if n == C.C3_GOLDEN_NS[0]:
            A, b = t10.assemble_tet10(mt, k=kf, f=1.0)
            put_csr(f"c3_n{n}_K", A)
            put(f"c3_n{n}_F", b)
        put(f"c3_n{n}_u", t10.solve_tet10_poisson(mt, k=kf, f=1.0, bc=allfaces))
        log(f"C3 n={n} done")

    # C4 at n = 32, 20 CN steps
    p = C.C4
    m4 = box_mesh(C.C4_N, C.C4_N, C.C4_N)
    times, hist = th.transient_heat_tet(
        m4, k=p["k"], rho_cp=p["rho_cp"], f=C.c4_source, robin=C.c4_robin(),
        t_end=C.C4_STEPS * p["dt"], dt=p["dt"], T0=p["t0"], method="cn")
    put("c4_times", times)
    put("c4_T1", hist[1])
    put("c4_Tend", hist[-1])
    log("C4 done")

    # C2 at quarter resolution
    nx, ny, nz, xl, yl, zl = C.C2Q_BOX
    mb = box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    ux, uy, uz = e10.solve_elasticity_tet10(mb, C.C2_E, C.C2_NU, bc=C.C2_BC,
                                            traction=C.C2_TRACTION)
    put("c2q_sol", np.stack([ux, uy, uz]))
    log("C2 quarter (reference solve) done")
    # the same reduced system, refined with extended-precision residuals
    A, b = e10.assemble_elasticity_tet10(mb, C.C2_E, C.C2_NU,
                                         traction=C.C2_TRACTION)
    fixed = np.sort(np.concatenate([3 * np.asarray(mb.boundaries["xmin"]) + c
                                    for c in range(3)]))
    free = np.setdiff1d(np.arange(A.shape[0]), fixed)
    Af = A.tocsr()[free][:, free].tocsc()
    bf = b[free]
    lu = spla.splu(Af)
    x0 = lu.solve(bf)
    xr, hist = refine_ext(Af, bf, x0, lu.solve)
    u = np.zeros(A.shape[0])
    u[free] = xr
    put("c2q_sol_refined", np.stack([u[0::3], u[1::3], u[2::3]]))
    put("c2q_refine_relres", np.array(hist))
    put("c2q_refine_change", np.array(np.linalg.norm(xr - x0) / np.linalg.norm(xr)))
    # condition number of the Jacobi-scaled reduced system (the solver's
    # preconditioned operator): the tests state errors beside kappa * eps
    dh = 1.0 / np.sqrt(Af.diagonal())
    As = (sp.diags(dh) @ Af @ sp.diags(dh)).tocsc()
    lmax = spla.eigsh(As, k=1, which="LA", return_eigenvectors=False)[0]
    lmin = spla.eigsh(As, k=1, sigma=0.0, which="LM", return_eigenvectors=False)[0]
    put("c2q_kappa", np.array(lmax / lmin))
    log(f"C2 quarter: Jacobi-scaled condition number {lmax / lmin:.3e}")
    log(f"C2 quarter refinement: residuals {hist}, "
        f"change {np.linalg.norm(xr - x0) / np.linalg.norm(xr):.2e}")
    del e3

    path = os.path.join(HERE, "config_fixtures.npz")
    np.savez_compressed(path, **out)
    size = os.path.getsize(path)
    log(f"wrote {path}: {len(out)} arrays, {size / 1024:.0f} KiB")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_config_golden.py <path of the CloudFEM checkout>")
    main(sys.argv[1])
