"""Error behaviour of the public entry points that needs no GPU: the
reference's ValueError for bad arguments where it raises before any work
(tet_heat.py:220-222, tet10.py transient, em3d_tet10.py:310-330), and no
CPU fallback: without a CUDA device a computing call raises RuntimeError."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def meshes():
    from cloudfem_b200.mesh import box_mesh, box_mesh_tet10
    return box_mesh(2, 2, 2), box_mesh_tet10(1, 1, 1)


def test_bad_method_and_excitation_raise_value_error(meshes):
    from cloudfem_b200.fem import tet10, tet_heat
    from cloudfem_b200.physics import em3d_tet10 as em
    m, m10 = meshes
    with pytest.raises(ValueError, match="unknown method"):
        tet_heat.transient_heat_tet(m, method="bogus")
    with pytest.raises(ValueError, match="unknown method"):
        tet10.transient_heat_tet10(m10, method="leapfrog")
    with pytest.raises(ValueError, match="omega"):
        em.solve_eddy_current_tet10(m10, omega=0.0, J_s=lambda x, y, z: (0.0, 0.0, 1.0))
    with pytest.raises(ValueError, match="excitation"):
        em.solve_eddy_current_tet10(m10, omega=1.0)


def test_no_cpu_fallback(meshes):
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from cloudfem_b200.fem import tet_poisson
    m, _ = meshes
    with pytest.raises(RuntimeError, match="no CPU fallback|There is no CPU fallback"):
        tet_poisson.solve_tet_poisson(m, k=1.0, f=1.0, bc={"all": 0.0})
    with pytest.raises(RuntimeError, match="CUDA device"):
        tet_poisson.assemble(m)
