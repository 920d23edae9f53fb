"""The CUDA path against the reference on the benchmark configurations.

Tolerances of the plain FP64 path (stated here, checked below):

* integer structure (indptr, indices) bit-exact;
* matrix and load values entry-wise within 1e-12 of themselves (an entry
  that cancels to near zero is held to 64 ulps of its row's largest entry,
  the rounding of its own sum; ``conftest.assert_csr_entrywise``);
* solutions within 1e-12 relative (max-norm) of the reference's answer, on
  the configurations whose conditioning allows it (C1, C3, C4). The Tet10
  cantilever's does not: its Jacobi-scaled condition number is ~6e6, its
  plain SuperLU answer moves by 8e-12 under iterative refinement, and a
  1-ulp perturbation of the matrix entries moves its exact solution by
  ~7e-12. There the CUDA answer is measured against the refined solution
  and held to kappa * eps, with both errors printed.

Mixed precision (FP32 CG with FP64 refinement) is held to 1e-8 of the FP64
path, the benchmark's accuracy bar.

References: ``tests/golden/config_fixtures.npz`` (the reference itself, run
by ``make_config_golden.py``) and, for meshes the reference is too slow on,
the oracle with the reference's explicit Dirichlet zeros dropped before
SuperLU (the answer is the same to round-off; the zeros only cost time).
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import cases as C
from conftest import assert_csr_entrywise, assert_entrywise, golden_csr, rel_err

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-12
MIXED_TOL = 1e-8
ALL0 = {s: 0.0 for s in C.FACES}


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _oracle_solve(A, b, mesh, bc):
    """The reference's elimination and SuperLU solve, explicit zeros dropped."""
    from oracle import cfem_oracle as O
    Abc, bbc = O.apply_dirichlet(A, b, mesh, bc)
    Abc = Abc.tocsr()
    Abc.eliminate_zeros()
    return np.asarray(spla.spsolve(Abc.tocsc(), bbc)).ravel()


def test_c1_p1_poisson_20cubed(torch, config_golden):
    """C1 exactly: box_mesh(20, 20, 20), k = 1, f = 3 pi^2 sin sin sin."""
    from cloudfem_b200.fem.tet_poisson import assemble, solve_tet_poisson
    from cloudfem_b200.mesh import box_mesh
    g = config_golden
    m = box_mesh(C.C1_N, C.C1_N, C.C1_N)
    A, b = assemble(m, k=1.0, f=C.f_sss)
    worst, at_floor = assert_csr_entrywise(A, golden_csr(g, "c1_K"), 1e-12, "C1 K")
    assert_entrywise(b, g["c1_F"], 1e-12, "C1 load")
    u = solve_tet_poisson(m, k=1.0, f=C.f_sss, bc=ALL0)
    err = rel_err(u, g["c1_u"])
    print(f"C1: K entry-wise {worst:.2e} ({at_floor} entries at the cancellation "
          f"floor), solution {err:.2e} vs the reference")
    assert err <= SOL_TOL, err


def _c3_problems(ns, ks):
    from cloudfem_b200.batch import HeatProblem
    from cloudfem_b200.mesh import box_mesh_tet10
    meshes = {int(n): box_mesh_tet10(int(n), int(n), int(n)) for n in set(ns)}
    # Kuhn box: 6 tets per hex cell, cells in (k, j, i) order, so element e
    # lies in cell e // 6 and the per-cell draw repeats 6 times
    return [HeatProblem(meshes[int(n)], k=np.repeat(kc, 6), f=1.0, bc=ALL0)
            for n, kc in zip(ns, ks)]


def test_c3_subset_batched_against_reference(torch, config_golden):
    """Seeded C3 meshes (n 4..8, lognormal per-cell k) in one batched FP64
    solve with per-element k arrays, against the reference's solutions; the
    n = 4 matrix and load entry-wise against the reference's."""
    from cloudfem_b200.batch import BatchSolver, solve_batch
    from cloudfem_b200.fem.tet10 import assemble_tet10
    g = config_golden
    ns = C.C3_GOLDEN_NS
    ks = C.c3_draw(ns)
    probs = _c3_problems(ns, ks)
    n0 = ns[0]
    A, b = assemble_tet10(probs[0].mesh, k=C.c3_cell_fn(n0, ks[0]), f=1.0)
    assert_csr_entrywise(A, golden_csr(g, f"c3_n{n0}_K"), 1e-12, "C3 n=4 K")
    assert_entrywise(b, g[f"c3_n{n0}_F"], 1e-12, "C3 n=4 load")
    solver = BatchSolver()
    batch = solver.prepare(probs)
    batch.assemble()
    # the batched per-element assembly agrees with the callable one of the
    # drop-in (k sampled at the Keast points)
    vals = batch.items[0]["vals"].cpu().numpy()
    assert_entrywise(vals, A.data, 1e-12, "C3 n=4 batched values")
    us = solve_batch(probs, precision="fp64", solver=solver)
    errs = [rel_err(u, g[f"c3_n{n}_u"]) for n, u in zip(ns, us)]
    print("C3 subset vs reference:", ", ".join(f"n={n}: {e:.2e}" for n, e in zip(ns, errs)))
    assert max(errs) <= SOL_TOL, errs
    um = solve_batch(probs, precision="mixed", rtol=1e-8, solver=solver)
    mixed = [rel_err(a, b) for a, b in zip(um, us)]
    print("C3 subset mixed (rtol 1e-8) vs FP64:", ", ".join(f"{e:.2e}" for e in mixed))
    assert max(mixed) <= MIXED_TOL, mixed


def test_c3_draw_batched_against_oracle(torch):
    """A seeded C3 draw with n up to 12 (the largest the oracle's SuperLU
    solves in seconds), batched FP64 and mixed, against the oracle."""
    from cloudfem_b200.batch import solve_batch
    from oracle import cfem_oracle as O
    rng = np.random.default_rng(C.C3_SEED + 1)
    ns = [int(n) for n in rng.integers(4, 13, size=6)] + [12]
    ks = [rng.lognormal(0.0, 1.0, n ** 3) for n in ns]
    probs = _c3_problems(ns, ks)
    us = solve_batch(probs, precision="fp64")
    um = solve_batch(probs, precision="mixed", rtol=1e-8)
    errs, mixed = [], []
    for n, kc, u, v in zip(ns, ks, us, um):
        mo = O.box_mesh_tet10(n, n, n)
        A, b = O.assemble_tet10(mo, k=C.c3_cell_fn(n, kc), f=1.0)
        ref = _oracle_solve(A, b, mo, ALL0)
        errs.append(rel_err(u, ref))
        mixed.append(rel_err(v, u))
    print("C3 draw vs oracle:", ", ".join(f"n={n}: {e:.2e}" for n, e in zip(ns, errs)))
    print("C3 draw mixed vs FP64:", ", ".join(f"{e:.2e}" for e in mixed))
    assert max(errs) <= SOL_TOL, errs
    assert max(mixed) <= MIXED_TOL, mixed


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c4_transient_n32(torch, config_golden, precision):
    """C4's operator at n = 32: Crank-Nicolson, Robin on all faces, Gaussian
    source, 20 steps, against the reference's march (one LU, 20 solves)."""
    from cloudfem_b200.fem.tet_heat import transient_heat_tet
    from cloudfem_b200.mesh import box_mesh
    g = config_golden
    p = C.C4
    m = box_mesh(C.C4_N, C.C4_N, C.C4_N)
    kw = {} if precision == "fp64" else dict(precision="mixed", rtol=1e-10)
    times, hist = transient_heat_tet(
        m, k=p["k"], rho_cp=p["rho_cp"], f=C.c4_source, robin=C.c4_robin(),
        t_end=C.C4_STEPS * p["dt"], dt=p["dt"], T0=p["t0"], method="cn", **kw)
    np.testing.assert_array_equal(times, g["c4_times"])
    e1 = rel_err(hist[1], g["c4_T1"])
    e20 = rel_err(hist[-1], g["c4_Tend"])
    print(f"C4 n=32 {precision}: step 1 {e1:.2e}, step 20 {e20:.2e}")
    tol = SOL_TOL if precision == "fp64" else MIXED_TOL
    assert e1 <= tol and e20 <= tol, (e1, e20)


def test_c2_quarter_beam(torch, config_golden):
    """C2 at quarter resolution (40 x 5 x 5 Tet10 cantilever, 29,403 DOFs).
    The pre-BC matrix is held entry-wise to the oracle at 1e-12. The
    solution cannot be held to 1e-12: the Jacobi-scaled condition number is
    about 6e6, and a random 1-ulp perturbation of the matrix entries alone
    moves this beam's exact solution by ~7e-12 (any two assemblies that sum
    in different orders differ by that much), while the reference's own
    SuperLU answer is 7.8e-12 from the refined solution. So, as prescribed
    for ill-conditioned cases, the FP64 answer is measured against the
    refined solution of the reference's system and printed beside kappa *
    eps, which bounds it."""
    from cloudfem_b200.mesh import box_mesh_tet10
    from cloudfem_b200.physics.elastic_tet10 import (assemble_elasticity_tet10,
                                                     solve_elasticity_tet10)
    from oracle import cfem_oracle as O
    g = config_golden
    nx, ny, nz, xl, yl, zl = C.C2Q_BOX
    m = box_mesh_tet10(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)
    A, b = assemble_elasticity_tet10(m, C.C2_E, C.C2_NU, traction=C.C2_TRACTION)
    mo = O.box_mesh_tet10(nx, ny, nz, xl, yl, zl)
    Ao, bo = O.assemble_elasticity_tet10(mo, C.C2_E, C.C2_NU, traction=C.C2_TRACTION)
    worst, _ = assert_csr_entrywise(A, Ao, 1e-12, "C2 quarter K")
    assert_entrywise(b, bo, 1e-12, "C2 quarter load")
    sol = np.stack(solve_elasticity_tet10(m, C.C2_E, C.C2_NU, bc=C.C2_BC,
                                          traction=C.C2_TRACTION))
    refined = g["c2q_sol_refined"]
    ours = rel_err(sol, refined)
    theirs = rel_err(g["c2q_sol"], refined)
    bound = float(g["c2q_kappa"]) * np.finfo(float).eps
    print(f"C2 quarter: K entry-wise {worst:.2e}; solution vs refined: ours "
          f"{ours:.2e}, reference SuperLU {theirs:.2e}; kappa * eps {bound:.2e}")
    assert ours <= bound, (ours, bound)
    solm = np.stack(solve_elasticity_tet10(m, C.C2_E, C.C2_NU, bc=C.C2_BC,
                                           traction=C.C2_TRACTION,
                                           precision="mixed", rtol=1e-10))
    assert rel_err(solm, sol) <= MIXED_TOL
