"""Tet10 mesh container and the Tet4 -> Tet10 converter.

Mirrors cloudfem/mesh/tet10_mesh.py: ``EDGES`` (:33), ``Tet10Mesh``
(:36-74), ``tet4_to_tet10`` (:77-112) and ``box_mesh_tet10`` (:115-135).
Midpoint nodes are appended in sorted-unique edge order, which here is
obtained by a 1-D unique over the packed key a * N + b (a < b) - the same
lexicographic order as the reference's row-wise unique.
"""

import numpy as np

from .tet_mesh import box_mesh

EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))


class Tet10Mesh:
    """Ten-node tetrahedral mesh (corners first, then edge midpoints)."""

    def __init__(self, nodes, elements, boundaries=None, n_corners=None):
        self.nodes = np.asarray(nodes, dtype=float)
        self.elements = np.asarray(elements, dtype=int)
        self.boundaries = dict(boundaries) if boundaries else {}
        if n_corners is None:
            n_corners = len(np.unique(self.elements[:, :4]))
        self.n_corners = int(n_corners)
        self._volumes = None

    @property
    def n_nodes(self):
        return self.nodes.shape[0]

    @property
    def n_elements(self):
        return self.elements.shape[0]

    def element_volumes(self):
        """Volumes from the corner nodes (tet10_mesh.py:66-74)."""
        if self._volumes is None:
            p = self.nodes[self.elements[:, :4]]
            m = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                          p[:, 3] - p[:, 0]], axis=2)
            self._volumes = np.abs(np.linalg.det(m)) / 6.0
        return self._volumes


def tet4_to_tet10(mesh):
    """Add edge-midpoint nodes; corner ids are preserved."""
    els = np.asarray(mesh.elements, dtype=np.int64)
    n0 = mesh.n_nodes
    e = np.array(EDGES)
    a = els[:, e[:, 0]]
    b = els[:, e[:, 1]]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = (lo * n0 + hi).ravel()
    uniq, inv = np.unique(key, return_inverse=True)
    ua, ub = uniq // n0, uniq % n0
    mid = 0.5 * (mesh.nodes[ua] + mesh.nodes[ub])
    elements = np.column_stack([els, n0 + inv.reshape(-1, 6)]).astype(int)
    nodes = np.vstack([mesh.nodes, mid])
    boundaries = {}
    for name, ids in mesh.boundaries.items():
        ids = np.asarray(ids, dtype=int)
        inset = np.zeros(n0, dtype=bool)
        inset[ids] = True
        extra = n0 + np.nonzero(inset[ua] & inset[ub])[0]
        boundaries[name] = np.sort(np.concatenate([ids, extra])).astype(int)
    return Tet10Mesh(nodes, elements, boundaries, n_corners=n0)


def box_mesh_tet10(nx, ny, nz, xlim=(0.0, 1.0), ylim=(0.0, 1.0),
                   zlim=(0.0, 1.0)):
    """Tet10 box mesh; face sets selected by coordinate (exact)."""
    mesh = tet4_to_tet10(box_mesh(nx, ny, nz, xlim=xlim, ylim=ylim,
                                  zlim=zlim))
    tol = 1e-9 * max(1.0, float(np.ptp(mesh.nodes)))
    lims = {"xmin": (0, xlim[0]), "xmax": (0, xlim[1]),
            "ymin": (1, ylim[0]), "ymax": (1, ylim[1]),
            "zmin": (2, zlim[0]), "zmax": (2, zlim[1])}
    mesh.boundaries = {
        name: np.nonzero(np.abs(mesh.nodes[:, ax] - v) <= tol)[0].astype(int)
        for name, (ax, v) in lims.items()}
    return mesh
