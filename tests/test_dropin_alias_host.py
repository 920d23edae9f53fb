"""The module aliasing that switches unchanged CloudFEM code to this
package: with the aliases in place, `from cloudfem.fem.tet_poisson import
assemble` and the other hot-path imports resolve to cloudfem_b200's
modules (checked against a stand-in `cloudfem` package with empty
subpackages, on the CPU)."""

import importlib
import sys

import pytest

pytest.importorskip("torch")

NAMES = ("mesh.tet_mesh", "mesh.tet10_mesh", "fem.tet_poisson", "fem.tet_heat",
         "fem.tet10", "physics.elastic3d", "physics.elastic_tet10",
         "physics.em3d_tet10", "physics.modal3d", "physics.dynamics3d")


def test_aliases_resolve_to_the_package(tmp_path, monkeypatch):
    root = tmp_path / "cloudfem"
    for sub in ("", "mesh", "fem", "physics"):
        d = root / sub
        d.mkdir(parents=True, exist_ok=True)
        (d / "__init__.py").write_text("")
    monkeypatch.syspath_prepend(str(tmp_path))
    saved = {k: v for k, v in sys.modules.items() if k == "cloudfem" or k.startswith("cloudfem.")}
    try:
        for name in NAMES:
            sys.modules["cloudfem." + name] = importlib.import_module("cloudfem_b200." + name)
        from cloudfem.fem.tet_poisson import assemble, solve_tet_poisson  # noqa: F401
        from cloudfem.fem.tet10 import _MASS_REF, element_operators  # noqa: F401
        from cloudfem.mesh.tet10_mesh import box_mesh_tet10
        from cloudfem.physics import elastic_tet10
        from cloudfem.physics.em3d_tet10 import assemble_tet10_av  # noqa: F401
        import cloudfem_b200.fem.tet_poisson as tp
        import cloudfem_b200.physics.elastic_tet10 as et
        assert assemble is tp.assemble and elastic_tet10 is et
        m = box_mesh_tet10(1, 1, 1)
        assert m.n_nodes == 27
    finally:
        for k in [k for k in sys.modules if k == "cloudfem" or k.startswith("cloudfem.")]:
            del sys.modules[k]
        sys.modules.update(saved)


def _reference_checkout():
    """The reference checkout: $CLOUDFEM_REFERENCE, else a `reference`
    directory beside this repository; None when neither exists."""
    import os
    cand = os.environ.get("CLOUDFEM_REFERENCE") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
        "reference")
    return cand if os.path.isfile(os.path.join(cand, "cloudfem", "__init__.py")) else None


ALIAS_SCRIPT = r"""
import importlib, sys
sys.path.insert(0, REF)
sys.path.insert(0, REPO)
import cloudfem  # the reference package itself
for name in NAMES:
    sys.modules["cloudfem." + name] = importlib.import_module("cloudfem_b200." + name)
# the reference's own callers of the replaced modules import unchanged
import cloudfem.physics.induction3d_tet10 as ind
import cloudfem.physics.inductance as L
import cloudfem.physics.thermomech as tm
import cloudfem_b200.physics.em3d_tet10 as em
import cloudfem_b200.fem.tet10 as t10
import cloudfem_b200.physics.elastic3d as e3
assert ind.assemble_tet10_av is em.assemble_tet10_av
assert ind._solve_phasor_with_K_tet10 is em._solve_phasor_with_K_tet10
assert ind._assemble_curl_curl_tet10_nu is em._assemble_curl_curl_tet10_nu
assert ind.bh_secant_mu_r is em.bh_secant_mu_r
assert ind.element_flux_density_tet10 is em.element_flux_density_tet10
assert ind.total_joule_power_tet10 is em.total_joule_power_tet10
assert ind.assemble_tet10 is t10.assemble_tet10
assert L.magnetic_energy_tet10 is em.magnetic_energy_tet10
assert L.source_complex_power_tet10 is em.source_complex_power_tet10
from cloudfem.physics.em3d_tet10 import solve_eddy_current_nonlinear_tet10
assert solve_eddy_current_nonlinear_tet10 is em.solve_eddy_current_nonlinear_tet10
assert tm.solve_elasticity_3d is e3.solve_elasticity_3d
from cloudfem.physics.dynamics3d import modal_superposition_3d, transient_3d
from cloudfem.physics.modal3d import solve_modes_3d
import cloudfem_b200.physics.dynamics3d as dyn
import cloudfem_b200.physics.modal3d as mod
assert transient_3d is dyn.transient_3d and solve_modes_3d is mod.solve_modes_3d
assert modal_superposition_3d is dyn.modal_superposition_3d
print("ALIAS_OK")
"""


def test_aliases_into_the_reference_package():
    """Aliasing into the real reference package: the reference's own
    callers of the replaced modules (induction3d_tet10, inductance,
    thermomech) import unchanged and bind this package's functions."""
    import os
    import subprocess
    ref = _reference_checkout()
    if ref is None:
        pytest.skip("reference checkout not found ($CLOUDFEM_REFERENCE)")
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = f"REF = {ref!r}\nREPO = {repo!r}\nNAMES = {NAMES!r}\n" + ALIAS_SCRIPT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True,
                         text=True, timeout=300)
    assert "ALIAS_OK" in out.stdout, out.stdout + out.stderr
