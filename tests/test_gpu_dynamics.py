"""Modal analysis and Newmark dynamics (modal3d / dynamics3d) on the device
against the reference's own outputs (tests/golden/ref_fixtures.npz, made by
make_golden.py on a P1 steel beam clamped at x = 0, 8 x 2 x 2 cells).

Tolerances (checked below):

* mass matrices: structure bit-exact, values entry-wise within 1e-12;
* frequencies within 1e-10 relative (ARPACK at tol 1e-10 in both codes;
  the shift-invert solves are FP64 PCG at rtol 1e-13 here, LU there);
* mode shapes up to sign: the M-weighted Gram matrix of the two bases is
  orthogonal to 1e-9 and, for modes whose frequency is isolated, its
  diagonal is +-1 to 1e-9 (eigenvector error scales with 1 / gap);
* Newmark histories within 1e-9 of the reference's largest value (20
  steps, each an FP64 PCG solve of K + a4 C + a1 M where the reference
  reuses one LU); the modal superposition history within 1e-9 too.

Measured on a B200: frequencies 4e-13 / 6e-13 (consistent / lumped mass),
Gram orthogonality 2e-15, direct histories 1.6e-12 (U), 1.2e-11 (final
acceleration, average acceleration rule), modal superposition 3.6e-12.
"""

import numpy as np
import pytest

import cases as C
from conftest import assert_csr_entrywise, golden_csr, rel_err

pytestmark = pytest.mark.gpu

FREQ_TOL = 1e-10
MODE_TOL = 1e-9
HIST_TOL = 1e-9


@pytest.fixture(scope="module")
def beam():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from cloudfem_b200.mesh import box_mesh
    nx, ny, nz, xl, yl, zl = C.DYN_BOX
    return box_mesh(nx, ny, nz, xlim=xl, ylim=yl, zlim=zl)


@pytest.mark.parametrize("lumped", [False, True])
def test_mass_matrix(beam, golden, lumped):
    from cloudfem_b200.physics.modal3d import assemble_mass_3d
    M = assemble_mass_3d(beam, C.DYN_RHO, lumped=lumped)
    worst, _ = assert_csr_entrywise(M, golden_csr(golden, "dyn_Ml" if lumped else "dyn_M"),
                                    1e-12, "mass")
    print(f"mass (lumped={lumped}): entry-wise {worst:.2e}")


@pytest.mark.parametrize("lumped", [False, True])
def test_modes_against_reference(beam, golden, lumped):
    from cloudfem_b200.physics.modal3d import assemble_mass_3d, solve_modes_3d
    sfx = "_l" if lumped else ""
    fr, modes = solve_modes_3d(beam, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC, n_modes=6,
                               lumped=lumped)
    ref_f, ref_m = golden["dyn_freqs" + sfx], golden["dyn_modes" + sfx]
    ferr = float(np.max(np.abs(fr - ref_f) / ref_f))
    M = assemble_mass_3d(beam, C.DYN_RHO, lumped=lumped)
    G = modes.T @ (M @ ref_m)
    orth = float(np.abs(G.T @ G - np.eye(6)).max())
    gap = np.full(6, np.inf)
    for j in range(6):
        others = np.delete(ref_f, j)
        gap[j] = np.min(np.abs(others - ref_f[j])) / ref_f[j]
    iso = gap > 1e-2
    diag = float(np.max(np.abs(np.abs(np.diag(G))[iso] - 1.0), initial=0.0))
    print(f"modes (lumped={lumped}): freqs {fr} Hz, rel err {ferr:.2e}; Gram orthogonality "
          f"{orth:.2e}; isolated modes {int(iso.sum())}, |diag| - 1 {diag:.2e}")
    assert ferr <= FREQ_TOL, ferr
    assert orth <= MODE_TOL, orth
    assert diag <= MODE_TOL, diag
    fixed = np.asarray(beam.boundaries["xmin"])
    assert not modes[3 * fixed].any()


@pytest.mark.parametrize("tag,kw", [("avg", dict(method="average")),
                                    ("lin", dict(method="linear", rayleigh=(5.0, 1e-6)))])
def test_transient_against_reference(beam, golden, tag, kw):
    from cloudfem_b200.physics.dynamics3d import transient_3d
    times, U, V, A = transient_3d(beam, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC,
                                  t_end=C.DYN_T_END, dt=C.DYN_DT, load=C.dyn_load(beam), **kw)
    np.testing.assert_array_equal(times, golden[f"dyn_{tag}_times"])
    eu = rel_err(U[:, ::7], golden[f"dyn_{tag}_U"])
    ev = rel_err(V[-1], golden[f"dyn_{tag}_V"])
    ea = rel_err(A[-1], golden[f"dyn_{tag}_A"])
    print(f"transient {tag}: U {eu:.2e}, V(end) {ev:.2e}, A(end) {ea:.2e}")
    assert max(eu, ev, ea) <= HIST_TOL, (eu, ev, ea)
    fixed = np.asarray(beam.boundaries["xmin"])
    assert not U[:, 3 * fixed].any()


def test_modal_superposition_against_reference(beam, golden):
    from cloudfem_b200.physics.dynamics3d import modal_superposition_3d
    times, U, V, A = modal_superposition_3d(
        beam, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc=C.DYN_BC, t_end=C.DYN_T_END, dt=C.DYN_DT,
        load=C.dyn_load(beam), n_modes=6, rayleigh=(5.0, 1e-6))
    # the modal history is invariant under the sign of each mode
    err = rel_err(U[:, ::7], golden["dyn_ms_U"])
    print(f"modal superposition: U {err:.2e}")
    assert err <= HIST_TOL, err


def test_newmark_integrate_sdof(golden):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from cloudfem_b200.physics.dynamics3d import newmark_integrate
    times, U, V, A = newmark_integrate(np.array([[2.0]]), np.array([[0.3]]),
                                       np.array([[50.0]]), lambda t: np.array([np.sin(3 * t)]),
                                       2.0, 0.05, u0=1.0, v0=0.0)
    eu = rel_err(U.ravel(), golden["dyn_sdof_U"])
    ea = rel_err(A.ravel(), golden["dyn_sdof_A"])
    print(f"single-DOF Newmark: U {eu:.2e}, A {ea:.2e}")
    assert eu <= 1e-12 and ea <= 1e-12, (eu, ea)


def test_transient_rejects_nonzero_bc(beam):
    from cloudfem_b200.physics.dynamics3d import transient_3d
    with pytest.raises(ValueError, match="homogeneous"):
        transient_3d(beam, C.DYN_E, C.DYN_NU, C.DYN_RHO, bc={"xmin": (0.0, 1e-3, 0.0)},
                     t_end=C.DYN_T_END, dt=C.DYN_DT)
