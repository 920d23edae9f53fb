"""Tet4 mesh container and the Kuhn box mesher.

Mirrors cloudfem/mesh/tet_mesh.py: ``TetMesh`` (:11-44) with the same
attributes, and ``box_mesh`` (:47-102) producing bit-identical node
coordinates, connectivity and boundary sets. The mesher is vectorised over
cells instead of looping in Python; the node numbering
``(i*(ny+1)+j)*(nz+1)+k`` and the k, j, i cell order fix the CSR column
order of every assembled matrix, so they are kept exactly.
"""

import numpy as np


class TetMesh:
    """Tetrahedral mesh: nodes (N, 3) float, elements (M, 4) int,
    boundaries {name: node ids}."""

    def __init__(self, nodes, elements, boundaries=None):
        self.nodes = np.asarray(nodes, dtype=float)
        self.elements = np.asarray(elements, dtype=int)
        self.boundaries = dict(boundaries) if boundaries else {}
        self._volumes = None

    @property
    def n_nodes(self):
        return self.nodes.shape[0]

    @property
    def n_elements(self):
        return self.elements.shape[0]

    def element_volumes(self):
        """Absolute tetrahedron volumes, shape (M,) (tet_mesh.py:36-44)."""
        if self._volumes is None:
            p = self.nodes[self.elements[:, :4]]
            m = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0],
                          p[:, 3] - p[:, 0]], axis=2)
            self._volumes = np.abs(np.linalg.det(m)) / 6.0
        return self._volumes


# Six tetrahedra around the cell diagonal c0 -> c7, corners numbered
# c = di + 2 dj + 4 dk (tet_mesh.py:75-82).
KUHN_TETS = np.array([[0, 1, 3, 7], [0, 1, 7, 5], [0, 5, 7, 4],
                      [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7]])


def box_mesh(nx, ny, nz, xlim=(0.0, 1.0), ylim=(0.0, 1.0), zlim=(0.0, 1.0)):
    """Uniform Kuhn mesh of a box, 6 tets per cell; tags xmin..zmax."""
    x = np.linspace(xlim[0], xlim[1], nx + 1)
    y = np.linspace(ylim[0], ylim[1], ny + 1)
    z = np.linspace(zlim[0], zlim[1], nz + 1)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    nodes = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    sy, sx = nz + 1, (ny + 1) * (nz + 1)          # strides of j and i

    # cell origins in k, j, i order (slowest k)
    kk, jj, ii = np.indices((nz, ny, nx)).reshape(3, -1)
    origin = ii * sx + jj * sy + kk
    corner = np.array([di * sx + dj * sy + dk
                       for dk in (0, 1) for dj in (0, 1) for di in (0, 1)])
    cells = origin[:, None] + corner[None, :]           # (C, 8)
    elements = cells[:, KUHN_TETS].reshape(-1, 4).astype(int)

    def plane(axis, val):
        if axis == 0:   # k outer, j inner
            b, a = np.indices((nz + 1, ny + 1)).reshape(2, -1)
            return val * sx + a * sy + b
        if axis == 1:   # k outer, i inner
            b, a = np.indices((nz + 1, nx + 1)).reshape(2, -1)
            return a * sx + val * sy + b
        b, a = np.indices((ny + 1, nx + 1)).reshape(2, -1)   # j outer, i inner
        return a * sx + b * sy + val

    bnd = {"xmin": plane(0, 0), "xmax": plane(0, nx), "ymin": plane(1, 0),
           "ymax": plane(1, ny), "zmin": plane(2, 0), "zmax": plane(2, nz)}
    return TetMesh(nodes, elements,
                   {k: np.asarray(v, dtype=int) for k, v in bnd.items()})
