"""Shared definitions of the small parity cases.

The same definitions build the inputs of the golden fixtures
(``tests/golden/make_golden.py``, upstream solver), of the oracle checks
(CPU) and of the device parity tests (GPU), so all three see identical
grids, masks, materials and seeded initial fields.
"""

import numpy as np

# -- tiny stepping cases (fields after a few one_step calls) ------------------

_BCS = [
    (["pec"] * 3, ["pec"] * 3),
    (["periodic"] * 3, ["periodic"] * 3),
    (["pec", "pec", "abc"], ["pec", "pec", "abc"]),
    (["pmc", "pec", "periodic"], ["pmc", "pec", "periodic"]),
    (["pec", "pec", "pml"], ["pec", "pec", "pml"]),
    (["magnetic", "pmc", "pec"], ["pec", "abc", "pml"]),
    (["periodic", "pec", "pec"], ["periodic", "pec", "abc"]),
]
_MATS = [
    ({}, [1.0, 1.0]),
    ({"a": "vacuum"}, "pec"),
    ({"a": [4.0, 1.0, 10.0], "b": [2.0, 2.0]}, [1.0, 1.0, 50.0]),
]


def _step_cases():
    out = []
    seed = 0
    for dtype in ("float64", "float32"):
        for bcl, bch in _BCS:
            for solids, bg in _MATS:
                out.append(dict(
                    bounds=(-0.01, 0.012, -0.01, 0.01, -0.02, 0.021),
                    shape=(7, 5, 9), bc_low=bcl, bc_high=bch, dtype=dtype,
                    solids=solids, bg=bg, n_pml=3, steps=6, seed=seed,
                    beam=dict(q=1e-9, sigmaz=0.005, beta=1.0, xsource=0.0, ysource=0.0)))
                seed += 1
    return out


STEP_CASES = _step_cases()


def step_masks(case):
    """Two overlapping box solids on the (7, 5, 9) case grid."""
    Nx, Ny, Nz = case["shape"]
    a = np.zeros((Nx, Ny, Nz), bool)
    a[1:4, 1:3, 2:5] = True
    b = np.zeros((Nx, Ny, Nz), bool)
    b[2:5, 0:2, 1:3] = True
    return {"a": a, "b": b}


def initial_fields(case, N):
    rng = np.random.default_rng(case["seed"])
    dt = np.dtype(case["dtype"]).type
    H0 = rng.standard_normal(3 * N).astype(dt)
    E0 = (rng.standard_normal(3 * N) * 300).astype(dt)
    return E0, H0


# -- small wake cases (full wakesolve + WakeSolver.solve) ---------------------

WAKE_CASES = [
    dict(bounds=(-0.01, 0.01, -0.01, 0.01, -0.015, 0.015), shape=(16, 16, 24),
         bc_low=["pec"] * 3, bc_high=["pec"] * 3, bg="pec", material="vacuum",
         dtype="float64", compute_plane="both", wakelength=0.05,
         wake=dict(q=1e-9, sigmaz=0.004, beta=1.0, skip_cells=0)),
    dict(bounds=(-0.01, 0.01, -0.01, 0.01, -0.015, 0.015), shape=(16, 16, 24),
         bc_low=["pec"] * 3, bc_high=["pec"] * 3, bg="pec", material="vacuum",
         dtype="float32", compute_plane="both", wakelength=0.05,
         wake=dict(q=1e-9, sigmaz=0.004, beta=1.0, skip_cells=3)),
    dict(bounds=(-0.01, 0.01, -0.01, 0.01, -0.015, 0.015), shape=(16, 16, 24),
         bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"], bg="pec",
         material="vacuum", dtype="float64", compute_plane="longitudinal",
         wakelength=0.05, wake=dict(q=1e-9, sigmaz=0.004, beta=0.8, skip_cells=0)),
    dict(bounds=(-0.01, 0.01, -0.01, 0.01, -0.015, 0.015), shape=(14, 16, 22),
         bc_low=["pec", "pec", "pml"], bc_high=["pec", "pec", "pml"],
         bg=[1.0, 1.0, 100.0], material="vacuum", dtype="float64",
         compute_plane="both", wakelength=0.04,
         wake=dict(q=1e-9, sigmaz=0.004, beta=0.7, skip_cells=2, xtest=0.001)),
]


def wake_mask(case, x, y, z):
    """Box cavity (|x|,|y| <= 8 mm, |z| <= 6 mm) with a 3 mm-radius pipe
    along z; a cell is inside when any of its 8 vertices is inside."""
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    inside = (((np.abs(X) <= 0.008) & (np.abs(Y) <= 0.008) & (np.abs(Z) <= 0.006))
              | (X ** 2 + Y ** 2 < 0.003 ** 2))
    m = np.zeros((len(x) - 1, len(y) - 1, len(z) - 1), bool)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                m |= inside[a:a + m.shape[0], b:b + m.shape[1], c:c + m.shape[2]]
    return m


# emsolve with each hard source of upstream sources.py on a small vacuum box
# (square transverse grid: WavePacket builds its profile on meshgrid(x, y))
SOURCE_BOUNDS = (-0.01, 0.01, -0.01, 0.01, -0.015, 0.015)
SOURCE_CASES = [
    dict(kind="PlaneWave", kw=dict(zs=0, f=8e9, nodes=1), shape=(16, 16, 24),
         bc_low=["periodic", "periodic", "pec"], bc_high=["periodic", "periodic", "pml"], Nt=40),
    dict(kind="WavePacket", kw=dict(zs=0, sigmaz=0.004, sigmaxy=0.004, wavelength=0.01),
         shape=(16, 16, 24), bc_low=["pec", "pec", "pec"], bc_high=["pec", "pec", "pml"],
         Nt=40),
    dict(kind="Dipole", kw=dict(field="Ez", nodes=5), shape=(16, 16, 24),
         bc_low=["pec"] * 3, bc_high=["pec"] * 3, Nt=30),
    dict(kind="Dipole", kw=dict(field="H", component="y", f=6e9, xs=4, ys=5, zs=7,
                                amplitude=2.0, phase=0.3),
         shape=(16, 16, 24), bc_low=["pec"] * 3, bc_high=["pmc", "pec", "pml"], Nt=30),
    dict(kind="Pulse", kw=dict(field="Ez", shape="Harris", L=0.006), shape=(16, 16, 24),
         bc_low=["pec"] * 3, bc_high=["pec"] * 3, Nt=60),
    dict(kind="Pulse", kw=dict(field="Jz", shape="Gaussian", L=0.004, amplitude=1e3),
         shape=(16, 16, 24), bc_low=["pec", "pec", "pml"], bc_high=["pec", "pec", "pml"], Nt=60),
    dict(kind="Pulse", kw=dict(field="E", component="x", shape="Rectangular", L=0.002,
                               xs=slice(4, 9), ys=7, zs=10),
         shape=(16, 16, 24), bc_low=["pec"] * 3, bc_high=["pec"] * 3, Nt=40),
]


# -- the lossy-wall workload geometry (conductive background, z-PML) ---------
# The cavity + pipe of the lossy workload (wakis_b200.workloads, lossy_256)
# at sizes upstream runs in seconds: sigma = 1e4 S/m background (dt clamped
# to eps_0/sigma), PEC x/y faces, 10-cell PML on both z faces, the Gaussian
# beam on the axis.  "init" is "random" (seeded fields, every coefficient
# exercised) or "zero" (beam only; ti is then shortened so that the bunch is
# at the upstream end of the grid from the first step).
def _lossy_cases():
    out = []
    for shape, dtype, init, steps, seed in (((24, 24, 48), "float64", "random", 12, 100),
                                            ((24, 24, 48), "float32", "random", 12, 101),
                                            ((32, 32, 64), "float64", "zero", 40, 102)):
        ti = None if init == "random" else 2.0 * 0.005 / 299792458.0
        out.append(dict(shape=shape, dtype=dtype, init=init, steps=steps, seed=seed,
                        bg=[1.0, 1.0, 1e4], bc_low=["pec", "pec", "pml"],
                        bc_high=["pec", "pec", "pml"], n_pml=10,
                        beam=dict(q=1e-9, sigmaz=0.005, beta=1.0, xsource=0.0, ysource=0.0,
                                  ti=ti)))
    return out


LOSSY_CASES = _lossy_cases()


def lossy_edges(case):
    from wakis_b200 import workloads
    x0, x1, y0, y1, z0, z1 = workloads.BOUNDS
    Nx, Ny, Nz = case["shape"]
    return (np.linspace(x0, x1, Nx + 1), np.linspace(y0, y1, Ny + 1),
            np.linspace(z0, z1, Nz + 1))


def lossy_mask(case):
    from wakis_b200 import workloads
    return workloads.cavity_mask(*lossy_edges(case))


def case_fields(case, N):
    """Initial (E, H) of a case with an "init" entry (zero or seeded random)."""
    dt = np.dtype(case["dtype"]).type
    if case.get("init") == "zero":
        return np.zeros(3 * N, dt), np.zeros(3 * N, dt)
    return initial_fields(case, N)


# -- surface impedance (SIBC) on a pillbox wall ------------------------------
# A C4-style pillbox at 2 mm cells whose wall conductivity is above the
# resolvable one, so upstream replaces the wall by its surface cells with
# eps = sigma = 1/Z_s (wakis/solverFIT3D.py:446-466).  Upstream takes the
# surface cells from VTK's gradient of the solid mask (gridFIT3D.py:519-535);
# both sides here use wakis_b200.geometry.surface_mask of the same wall mask
# instead (injected into upstream for the fixtures).
SIBC_CASES = [
    dict(kind="step", pillbox=dict(R=0.020, L=0.030, cell=2e-3), sigma=1e4, dtype="float64",
         steps=10, seed=200, bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"],
         beam=dict(q=1e-9, sigmaz=0.008, beta=0.9, xsource=0.0, ysource=0.0)),
    dict(kind="wake", pillbox=dict(R=0.020, L=0.030, cell=2e-3), sigma=1e4, dtype="float64",
         bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"], wakelength=0.05,
         compute_plane="both", wake=dict(q=1e-9, sigmaz=0.008, beta=0.9)),
]


def sibc_geometry(case):
    """(bounds, shape, wall mask, surface mask) of a SIBC case."""
    from wakis_b200 import batch, geometry
    b, shape, wall = batch.pillbox_grid(**case["pillbox"])
    x = np.linspace(b[0], b[1], shape[0] + 1)
    y = np.linspace(b[2], b[3], shape[1] + 1)
    z = np.linspace(b[4], b[5], shape[2] + 1)
    m = wall(x, y, z)
    return b, shape, m, geometry.surface_mask(m)


# -- emsolve with ABC faces ---------------------------------------------------
# Upstream's get_abc keeps, on its CPU path, views of the live field arrays
# (wakis/boundaries.py:313-366 with field.py:223-300), so update_abc copies
# the current first interior plane onto a low face and leaves a high face as
# it is; on its GPU path (cupy .get()) the snapshots are copies, and both
# faces take the values of two steps before.  "abc_copies" selects the GPU
# semantics (the fixtures emulate them by copying the snapshots).  An axis
# has ABC on one side only: upstream keeps one snapshot dict per axis, and
# the second side's dict replaces the first.
ABC_SOURCE_CASES = [
    dict(kind="Dipole", kw=dict(field="Ez", nodes=5), shape=(16, 16, 24),
         bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "pec"], Nt=40, abc_copies=False),
    dict(kind="Dipole", kw=dict(field="Ez", nodes=5), shape=(16, 16, 24),
         bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "pec"], Nt=40, abc_copies=True),
    dict(kind="Pulse", kw=dict(field="Jz", shape="Gaussian", L=0.004, amplitude=1e3),
         shape=(16, 16, 24), bc_low=["abc", "pec", "pec"], bc_high=["pec", "abc", "abc"],
         Nt=50, abc_copies=False),
    dict(kind="Pulse", kw=dict(field="Jz", shape="Gaussian", L=0.004, amplitude=1e3),
         shape=(16, 16, 24), bc_low=["abc", "pec", "pec"], bc_high=["pec", "abc", "abc"],
         Nt=50, abc_copies=True),
]


# -- Field storage and indexing ----------------------------------------------
# A small random field and the index patterns, assignments and arithmetic of
# upstream wakis/field.py (to_matrix, get_abs, __getitem__/__setitem__ with
# (i, j, k, comp) tuples, lexicographic ints and slices, __mul__/__add__ with
# scalars, flat arrays, (Nx, Ny, Nz) matrices and fields, compute_ijk).
FIELD_CASE = dict(shape=(5, 4, 6), seed=300)


def field_inputs():
    """(flat field array, second flat field, (Nx, Ny, Nz) matrix, flat 3N array)."""
    Nx, Ny, Nz = FIELD_CASE["shape"]
    N = Nx * Ny * Nz
    rng = np.random.default_rng(FIELD_CASE["seed"])
    return (rng.standard_normal(3 * N), rng.standard_normal(3 * N),
            rng.standard_normal((Nx, Ny, Nz)), rng.standard_normal(3 * N))


# (name, key) of the reads compared, and the writes applied in order
FIELD_READS = [("g_point", (2, 1, 3, "y")), ("g_block", (slice(1, 4), 2, slice(None), "z")),
               ("g_abs", (slice(None), 1, 2, "Abs")), ("g_x0", (0, slice(None), 5, 0)),
               ("g_int", 17), ("g_slice", slice(5, 40, 3))]
FIELD_WRITES = [((slice(1, 3), slice(None), 2, "x"), 7.5), ((0, 0, 0, "z"), -1.0), (10, 3.0),
                (slice(20, 25), "arange5"), ((slice(None), slice(None), 4, "y"), "plane_y4")]
FIELD_IJK = [0, 7, 33, 119]
