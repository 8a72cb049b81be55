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
