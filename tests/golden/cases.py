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


# ------------------------------------------------ configuration-scale cases
# These reproduce the benchmark configurations (or seeded subsets of them)
# at sizes the reference finishes in seconds to minutes; their reference
# answers are in config_fixtures.npz (make_config_golden.py).

# C1: P1 steady heat, unit cube 20^3 Kuhn box, k = 1, f = 3 pi^2 sin sin sin
# at centroids, T = 0 on all six faces
C1_N = 20

# C3: seeded Tet10 unit cubes, lognormal(0, 1) conductivity per hex cell,
# f = 1, T = 0 on all faces; the reference is run on the small ones
C3_SEED = 11
C3_GOLDEN_NS = (4, 5, 6, 8)


def c3_draw(ns, seed=C3_SEED):
    """One lognormal(0, 1) conductivity per hex cell (cell order k, j, i)."""
    rng = np.random.default_rng(seed)
    return [rng.lognormal(0.0, 1.0, int(n) ** 3) for n in ns]


def c3_cell_fn(n, kc):
    """Per-cell conductivity as a callable k(x, y, z) of the unit cube,
    the form the reference's API takes (Keast points are interior, so every
    point of an element looks up its own cell)."""
    kc3 = np.asarray(kc).reshape(n, n, n)

    def k(x, y, z):
        i = np.minimum((np.asarray(x) * n).astype(int), n - 1)
        j = np.minimum((np.asarray(y) * n).astype(int), n - 1)
        kk = np.minimum((np.asarray(z) * n).astype(int), n - 1)
        return kc3[kk, j, i]
    return k


# C4: P1 transient heat, Crank-Nicolson, Robin on all faces, Gaussian source
# at the centre, at n = 32 for 20 steps of 1 s
C4_N = 32
C4_STEPS = 20
C4 = dict(k=45.0, rho_cp=3.6e6, t0=20.0, h=25.0, t_inf=20.0, q0=1e7,
          sigma=0.1, dt=1.0)


def c4_source(x, y, z):
    r2 = ((np.asarray(x) - 0.5) ** 2 + (np.asarray(y) - 0.5) ** 2
          + (np.asarray(z) - 0.5) ** 2)
    return C4["q0"] * np.exp(-r2 / (2.0 * C4["sigma"] ** 2))


def c4_robin():
    return {f: (C4["h"], C4["t_inf"]) for f in FACES}


# C2 at quarter resolution: Tet10 cantilever 2.0 x 0.25 x 0.25 m, 40 x 5 x 5
# cells, clamped at x = 0, 1 MPa traction in -z on x = 2
C2Q_BOX = (40, 5, 5, (0.0, 2.0), (0.0, 0.25), (0.0, 0.25))
C2_E, C2_NU = 210e9, 0.3
C2_BC = {"xmin": (0.0, 0.0, 0.0)}
C2_TRACTION = {"xmax": (0.0, 0.0, -1e6)}


# nonlinear (secant B-H) phasor A-V: iron and conductor in x < 0.5, a
# background field strong enough to saturate part of the iron
AVN_N = 3
AVN_OMEGA = 2.0 * np.pi * 50.0
AVN_B = (0.0, 0.0, 2.5)
AVN_KW = dict(tol=1e-3, max_iter=40, relax=0.8)


def avn_sigma(x, y, z):
    return 2.0e6 if x < 0.5 else 0.0


def avn_iron(x, y, z):
    return x < 0.5


# B-H curve sample points [A/m], including the small-h series branch
BH_H = np.array([0.0, 1e-9, 1.0, 30.0, 500.0, 3e3, 2e4, 1e5, 1e6])


# staggered EM -> heat induction heating of a steel block (x < 0.5) in a
# background field: two EM intervals of two heat steps each; the second
# case adds the temperature-dependent capacity and a second stagger pass
IND_N = 3
IND_KW = dict(omega=2.0 * np.pi * 50.0, B_applied=(0.0, 0.0, 1.5),
              boundary=list(FACES), T0=20.0, t_end=0.04, dt=0.01, em_every=2,
              k_th=30.0, rho_cp=3.768e6, method="be", em_tol=1e-3,
              em_max_iter=40, em_relax=0.8)
IND_KW2 = dict(IND_KW, method="cn", stagger_iter=2, cp_slope=1e-3,
               cp_peak_h=2e6, cp_peak_w=25.0)


def ind_iron(x, y, z):
    return x < 0.5


# P1 structural dynamics: a steel beam clamped at x = 0 (modal3d /
# dynamics3d), a vertical tip load ramped in over the first steps
DYN_BOX = (8, 2, 2, (0.0, 1.0), (0.0, 0.125), (0.0, 0.125))
DYN_E, DYN_NU, DYN_RHO = 210e9, 0.3, 7800.0
DYN_BC = {"xmin": (0.0, 0.0, 0.0)}
DYN_T_END, DYN_DT = 4e-3, 2e-4


def dyn_load(mesh):
    """F(t) on the full 3N DOFs: -z force on the x = 1 face, ramped."""
    n3 = 3 * mesh.n_nodes
    tip = np.asarray(mesh.boundaries["xmax"])
    base = np.zeros(n3)
    base[3 * tip + 2] = -1e4 / len(tip)

    def F(t):
        return base * min(1.0, t / 1e-3)
    return F
