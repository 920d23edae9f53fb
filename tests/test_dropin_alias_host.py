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
         "physics.em3d_tet10")


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
