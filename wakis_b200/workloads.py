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
* ``precision_448`` 448x448x896 cells (180 M), the cavity_40 geometry and
  boundaries plus a dielectric cube insert (eps_r = 4, sigma = 10 S/m, 20 mm
  side, centred at x = +5 mm); sigma_z = 10 mm, beta = 1, wakelength 3 m.
  The FP32-compensated state is compared with FP64 on this grid.
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
    if name == "precision_448":
        sp = spec("cavity_40")
        sp.update(shape=(448, 448, 896), wakelength=3.0,
                  insert=dict(box=(-0.005, 0.015, -0.010, 0.010, -0.010, 0.010),
                              material=[4.0, 1.0, 10.0]))
        return sp
    raise KeyError(name)


def cavity_mask(x, y, z):
    return geometry.cell_mask(cavity_shape(), x, y, z)


def build_b200(name, dtype=np.float64, shape=None, precision=None, dt=None):
    """(grid, wake, solver) of a workload on the device (``dt``: a given time
    step instead of the CFL one, as SolverFIT3D's argument)."""
    from .gridFIT3D import GridFIT3D
    from .solverFIT3D import SolverFIT3D
    from .wakeSolver import WakeSolver
    sp = spec(name)
    shp = shape or sp["shape"]
    g = GridFIT3D(*BOUNDS, *shp, verbose=0)
    g.add_solid("cavity", cavity_mask(g.x, g.y, g.z), "vacuum")
    if "insert" in sp:
        ins = sp["insert"]
        g.add_solid("insert", geometry.cell_mask(geometry.Box(*ins["box"], tol=1e-12),
                                                 g.x, g.y, g.z), ins["material"])
    w = WakeSolver(save=False, verbose=0, **sp["wake"])
    s = SolverFIT3D(g, w, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
                    dtype=dtype, n_pml=sp["n_pml"], verbose=0, precision=precision, dt=dt)
    return g, w, s


def stacked_edges(name, n_blocks, shape=None):
    """Edges of a chain of n_blocks copies of a workload grid stacked along
    z (block b spans z in [-50 + 100 b, 50 + 100 b] mm); one block is the
    workload's own grid."""
    Nx, Ny, Nz = shape or spec(name)["shape"]
    x0, x1, y0, y1, z0, z1 = BOUNDS
    return (np.linspace(x0, x1, Nx + 1), np.linspace(y0, y1, Ny + 1),
            np.linspace(z0, z0 + n_blocks * (z1 - z0), n_blocks * Nz + 1))


def build_stacked(name, n_blocks, shape=None, planes=None, dtype=np.float64, precision=None,
                  device=None):
    """(grid, wake, solver) of a chain of n_blocks copies of a workload
    stacked along z: the beam pipe runs through all of them, every block
    holds its own cavity (and insert), the workload's z boundaries (PML,
    ABC, PEC) close the two ends of the chain.  With planes = (lo, hi) only
    the planes [lo, hi) of the chain are built, on the chain's own edges, as
    one z-slab for ``slab.py``: an end of the slab inside the chain is an
    internal face (no PML; the PEC mask there touches only the padding).  Weak-scaling workload of the slab
    decomposition: each GPU steps one block."""
    from .gridFIT3D import GridFIT3D
    from .solverFIT3D import SolverFIT3D
    from .wakeSolver import WakeSolver
    sp = spec(name)
    x, y, z = stacked_edges(name, n_blocks, shape)
    Nz = len(z) - 1
    lo, hi = planes if planes is not None else (0, Nz)
    zl = z[lo:hi + 1]
    Lz = BOUNDS[5] - BOUNDS[4]
    cav = geometry.CylinderZ(0.005)
    ins = None
    for b in range(n_blocks):
        cav = cav | geometry.Box(-0.015, 0.015, -0.015, 0.015, -0.015 + b * Lz,
                                 0.015 + b * Lz, tol=1e-12)
        if "insert" in sp:
            bx = list(sp["insert"]["box"])
            box = geometry.Box(*bx[:4], bx[4] + b * Lz, bx[5] + b * Lz, tol=1e-12)
            ins = box if ins is None else ins | box
    # the CFL step of the whole chain (the builder's expression on the global
    # edges: a slab's own minimum spacing can differ in the last bit)
    from .coefficients import C_LIGHT
    dt = 0.5 / (C_LIGHT * np.sqrt(1 / np.min(np.diff(x)) ** 2 + 1 / np.min(np.diff(y)) ** 2
                                  + 1 / np.min(np.diff(z)) ** 2))
    g = GridFIT3D(x=x, y=y, z=zl, verbose=0)
    g.add_solid("cavity", geometry.cell_mask(cav, g.x, g.y, g.z), "vacuum")
    if ins is not None:
        g.add_solid("insert", geometry.cell_mask(ins, g.x, g.y, g.z), sp["insert"]["material"])
    # an end of the slab inside the chain: the PEC column mask (it reaches
    # only the slab's padding plane, slab.py) when the grid has a PEC-like
    # face already, so the slab keeps the full-domain kernel and the H-row
    # summation order; else no mask
    bc_low, bc_high = list(sp["bc_low"]), list(sp["bc_high"])
    pec_like = any(b.lower() in ("pec", "electric", "pml") for b in bc_low + bc_high)
    inner = "pec" if pec_like else "abc"
    if lo > 0:
        bc_low[2] = inner
    if hi < Nz:
        bc_high[2] = inner
    w = WakeSolver(save=False, verbose=0, **sp["wake"])
    s = SolverFIT3D(g, w, dt=dt, bc_low=bc_low, bc_high=bc_high, use_stl=True, bg=sp["bg"],
                    dtype=dtype, n_pml=sp["n_pml"], verbose=0, precision=precision,
                    device=device)
    return g, w, s


def precision_compare(name="precision_448", shape=None, wakelength=None, max_steps=None):
    """Run wakesolve twice on the same grid, FP64 and FP32-compensated, and
    return the relative errors (max|a-b| / max|b|) of the FP32c results
    against FP64 together with both stepping rates.  The FP64 solver is
    released before the FP32c one is built."""
    import time

    import torch

    sp = spec(name)
    wl = wakelength if wakelength is not None else sp["wakelength"]

    def rel(a, b):
        a, b = np.asarray(a), np.asarray(b)
        den = np.max(np.abs(b)) if b.size else 0.0
        return float(np.max(np.abs(a - b)) / den) if den else 0.0

    out, res = {}, {}
    # the same geometry on a small grid first, so that loading the kernels
    # and the wake post-processing of the first call is not timed
    for prec in (None, "fp32c"):
        _, _, s = build_b200(name, dtype=np.float64, shape=(32, 32, 64), precision=prec)
        s.wakesolve(wakelength=0.01)
        del s
    for prec in (None, "fp32c"):
        t0 = time.perf_counter()
        g, w, s = build_b200(name, dtype=np.float64, shape=shape, precision=prec)
        t_build = time.perf_counter() - t0
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        s.wakesolve(wakelength=wl)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        key = "fp32c" if prec else "fp64"
        res[key] = {n: np.array(getattr(w, n)) for n in ("s", "WP", "WPx", "WPy", "f", "Z",
                                                        "Zx", "Zy")}
        out[key] = {"steps": int(s.Nt), "cells": int(s.N), "wakesolve_ms": ms,
                    "gcell_steps_per_s": s.N * s.Nt / (ms / 1e3) / 1e9, "build_s": t_build}
        del g, w, s
        torch.cuda.empty_cache()
    a, b = res["fp32c"], res["fp64"]
    out["errors"] = {"WP": rel(a["WP"], b["WP"]), "WPx": rel(a["WPx"], b["WPx"]),
                     "WPy": rel(a["WPy"], b["WPy"]), "absZ": rel(np.abs(a["Z"]), np.abs(b["Z"])),
                     "ReZ": rel(a["Z"].real, b["Z"].real), "ImZ": rel(a["Z"].imag, b["Z"].imag),
                     "absZx": rel(np.abs(a["Zx"]), np.abs(b["Zx"]))}
    out["wakelength"] = wl
    return out
