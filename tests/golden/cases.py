"""Shared inputs of the golden-vector cases.

The same functions are used by ``make_golden.py`` (which runs the
reference package on them) and by the tests (which run the oracle and
the CUDA path on them), so coefficient callables are defined once.
Meshes are small so that every case runs in well under a second on
the CPU.
"""

import numpy as np

FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")

# Box shapes (nx, ny, nz, xlim, ylim, zlim).
P1_BOX = (3, 4, 5, (0.0, 2.0), (0.0, 1.0), (0.0, 0.5))
P1_CUBE = 4
TET10_BOX = (2, 2, 3, (0.0, 1.0), (0.0, 0.5), (0.0, 1.5))
TET10_BEAM = (6, 1, 2, (0.0, 0.6), (0.0, 0.05), (0.0, 0.1))
AV_BOX = (2, 2, 2, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
# phasor A-V solves: conductor everywhere, source current, A = 0 outside
AVP_N = 3
AVP_SIGMA = 1.0e6
AVP_OMEGA = 2.0 * np.pi * 1000.0


def k_fn(x, y, z):
    return 1.0 + 0.5 * x + 0.25 * y * z


def f_fn(x, y, z):
    return np.sin(np.pi * x) * np.cos(0.5 * np.pi * y) + z


def rho_fn(x, y, z):
    return 2.0 + x * y + 0.1 * z


def bc_fn(x, y, z):
    return 1.0 + x - 2.0 * y + 0.5 * z * z


def q_fn(x, y, z):
    return 3.0 + x + y * z


def h_fn(x, y, z):
    return 5.0 + 0.5 * x


def tinf_fn(x, y, z):
    return 20.0 + y


def bx_fn(x, y, z):
    return 1.0e3 * (1.0 + x)


def t_fn(x, y, z):
    return 50.0 + 10.0 * x - 5.0 * y * z


def sigma_fn(x, y, z):
    return 5.8e7 if x < 0.5 else 0.0


def nu_fn(x, y, z):
    return 1.0 / (4e-7 * np.pi) * (1.0 + 0.1 * y)


def exact_sss(x, y, z):
    return np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)


def f_sss(x, y, z):
    return 3.0 * np.pi ** 2 * exact_sss(x, y, z)


def t_nodal(n_nodes):
    """Seeded nodal temperature field used by the thermal-load cases."""
    rng = np.random.default_rng(7)
    return 20.0 + 30.0 * rng.random(n_nodes)


def avp_js(x, y, z):
    """Complex source current density of the phasor A-V cases."""
    s = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    return np.array([(1.0 + 2.0j) * 1e9 * s, 0.5e9 * s * (1.0 + x), 0.3j * 1e9 * y * z])


# transient A-V: half-conducting box, sinusoidal source, a few CN steps
AVT_N = 3
AVT_T_END, AVT_DT = 4e-3, 1e-3


def avt_js(x, y, z):
    """Real source current density pattern of the transient A-V case."""
    s = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    return np.array([1e8 * s, 0.5e8 * s * (1.0 + x), 0.2e8 * y * z])


def avt_scale(t):
    return np.sin(2.0 * np.pi * 250.0 * t)
