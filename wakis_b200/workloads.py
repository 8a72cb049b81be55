"""Synthetic wakefield workloads used by the tests and the benchmark.

Each workload is a PEC-like box with a 30 mm cubic vacuum cavity centred at
the origin and a 5 mm-radius vacuum beam pipe along z, on a uniform grid
over x, y in [-25, 25] mm and z in [-50, 50] mm; cells are vacuum when any
of their corners is inside the cavity or the pipe.

* ``cavity_40``   40x40x80 cells, PEC background, PEC on x/y faces, ABC
  (first-order extrapolation faces) on z; bunch sigma_z = 10 mm, beta = 1,
  wakelength 0.5 m, fmax = 5 GHz.
* ``lossy_256``   256x256x512 cells (33.5 M), walls are a lossy conductor
  (sigma = 1e4 S/m background, eps_r = mu_r = 1), 10-cell PML at both z
  ends; bunch sigma_z = 5 mm, beta = 1, wakelength 5 m.  The conductive
  background clamps dt to the relaxation time eps_0/sigma = 8.85e-16 s, as
  upstream does (wakis/solverFIT3D.py:301-310).
"""

import numpy as np

from . import geometry

BOUNDS = (-0.025, 0.025, -0.025, 0.025, -0.05, 0.05)


def cavity_shape():
    return geometry.Box(-0.015, 0.015, -0.015, 0.015, -0.015, 0.015, tol=1e-12) | \
        geometry.CylinderZ(0.005)


def spec(name):
    if name == "cavity_40":
        return dict(shape=(40, 40, 80), bg="pec", bc_low=["pec", "pec", "abc"],
                    bc_high=["pec", "pec", "abc"], n_pml=10,
                    wake=dict(q=1e-9, sigmaz=10e-3, beta=1.0, xsource=0.0, ysource=0.0,
                              xtest=0.0, ytest=0.0, fmax=5e9),
                    wakelength=0.5)
    if name == "lossy_256":
        return dict(shape=(256, 256, 512), bg=[1.0, 1.0, 1e4], bc_low=["pec", "pec", "pml"],
                    bc_high=["pec", "pec", "pml"], n_pml=10,
                    wake=dict(q=1e-9, sigmaz=5e-3, beta=1.0, xsource=0.0, ysource=0.0,
                              xtest=0.0, ytest=0.0),
                    wakelength=5.0)
    raise KeyError(name)


def cavity_mask(x, y, z):
    return geometry.cell_mask(cavity_shape(), x, y, z)


def build_b200(name, dtype=np.float64, shape=None, precision=None):
    """(grid, wake, solver) of a workload on the device."""
    from .gridFIT3D import GridFIT3D
    from .solverFIT3D import SolverFIT3D
    from .wakeSolver import WakeSolver
    sp = spec(name)
    shp = shape or sp["shape"]
    g = GridFIT3D(*BOUNDS, *shp, verbose=0)
    g.add_solid("cavity", cavity_mask(g.x, g.y, g.z), "vacuum")
    w = WakeSolver(save=False, verbose=0, **sp["wake"])
    s = SolverFIT3D(g, w, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
                    dtype=dtype, n_pml=sp["n_pml"], verbose=0, precision=precision)
    return g, w, s
