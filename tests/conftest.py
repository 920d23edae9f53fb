import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "ref_fixtures.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def config_golden():
    """Reference outputs on the benchmark configurations (make_config_golden.py)."""
    path = os.path.join(ROOT, "tests", "golden", "config_fixtures.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def golden_csr(golden, name):
    import scipy.sparse as sp
    shape = tuple(int(v) for v in golden[name + "__shape"])
    return sp.csr_matrix((golden[name + "__data"],
                          golden[name + "__indices"],
                          golden[name + "__indptr"]), shape=shape)


def _drop_zeros(A, tol):
    """Remove entries with |v| <= tol * max|v| (exact zeros included).

    The reference's Dirichlet step stores its cleared columns as explicit
    zeros, and on Kuhn meshes some P1 couplings cancel to exactly 0.0 in the
    reference's LAPACK arithmetic but to ~1e-17 in any other order of
    operations, so post-BC structures are compared without (near-)zeros.
    """
    A = A.tocsr().copy()
    scale = float(np.abs(A.data).max(initial=0.0))
    A.data[np.abs(A.data) <= tol * scale] = 0.0
    A.eliminate_zeros()
    return A


def assert_csr_equal(A, B, rtol=1e-12, eliminate=False):
    """Bit-exact structure and values within rtol of the largest entry."""
    A = A.tocsr().copy()
    B = B.tocsr().copy()
    if eliminate:
        A = _drop_zeros(A, 1e-13)
        B = _drop_zeros(B, 1e-13)
    assert A.shape == B.shape
    np.testing.assert_array_equal(np.asarray(A.indptr, np.int64),
                                  np.asarray(B.indptr, np.int64))
    np.testing.assert_array_equal(np.asarray(A.indices, np.int64),
                                  np.asarray(B.indices, np.int64))
    scale = max(float(np.abs(B.data).max(initial=0.0)), 1e-300)
    err = float(np.abs(A.data - B.data).max(initial=0.0)) / scale
    assert err <= rtol, f"CSR values differ: {err:.3e} > {rtol:.1e}"


def assert_close(a, b, rtol=1e-12, what=""):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    scale = max(float(np.abs(b).max(initial=0.0)), 1e-300)
    err = float(np.abs(a - b).max(initial=0.0)) / scale
    assert err <= rtol, f"{what}: rel err {err:.3e} > {rtol:.1e}"


# Entry-wise tolerance of matrix values. Each entry is a sum of element
# contributions; summed in another order it differs by a few ulps of the
# largest contribution, so an entry that cancels to (near) zero cannot be
# compared relative to itself. Entries are held to rtol of their own
# magnitude, with a floor of CANCEL_EPS times the largest entry of their row.
CANCEL_EPS = 64 * np.finfo(float).eps


def assert_csr_entrywise(A, B, rtol=1e-12, what="CSR"):
    """Bit-exact indptr / indices; every value within rtol of itself (floor:
    CANCEL_EPS of its row's largest entry). Returns (max entry-relative
    error over entries above the floor, count of entries at the floor)."""
    A = A.tocsr()
    B = B.tocsr()
    assert A.shape == B.shape, f"{what}: shape {A.shape} vs {B.shape}"
    np.testing.assert_array_equal(np.asarray(A.indptr, np.int64),
                                  np.asarray(B.indptr, np.int64))
    np.testing.assert_array_equal(np.asarray(A.indices, np.int64),
                                  np.asarray(B.indices, np.int64))
    absb = np.abs(B.data)
    rows = np.repeat(np.arange(B.shape[0]), np.diff(B.indptr))
    rowmax = np.zeros(B.shape[0])
    np.maximum.at(rowmax, rows, absb)
    floor = CANCEL_EPS * rowmax[rows]
    diff = np.abs(A.data - B.data)
    bad = diff > rtol * absb + floor
    assert not bad.any(), (
        f"{what}: {int(bad.sum())} entries differ beyond {rtol:.0e} "
        f"(worst {float((diff / np.maximum(absb, 1e-300)).max()):.3e})")
    big = absb > floor / rtol
    worst = float((diff[big] / absb[big]).max(initial=0.0))
    return worst, int((~big).sum())


def assert_entrywise(a, b, rtol=1e-12, what="vector"):
    """Every entry within rtol of itself, floor CANCEL_EPS of the largest."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    floor = CANCEL_EPS * float(np.abs(b).max(initial=0.0))
    diff = np.abs(a - b)
    bad = diff > rtol * np.abs(b) + floor
    assert not bad.any(), f"{what}: {int(bad.sum())} entries beyond {rtol:.0e}"


def rel_err(a, b):
    """max |a - b| / max |b| (the solution error measure of the tests)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return float(np.abs(a - b).max(initial=0.0)) / max(
        float(np.abs(b).max(initial=0.0)), 1e-300)
