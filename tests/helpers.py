"""Builders shared by the CPU and GPU tests: the same case definition gives
an oracle solver (CPU restatement of upstream) and, on a GPU, a
``wakis_b200`` solver with identical grid, masks, materials and fields."""

import numpy as np

import cases
from oracle import fit as ofit
from oracle import wake as owake


def oracle_step_case(c):
    masks = cases.step_masks(c)
    solids = {k: masks[k] for k in c["solids"]} if c["solids"] else None
    g = ofit.Grid(*c["bounds"], *c["shape"], solids=solids, materials=c["solids"] or None)
    s = ofit.Solver(g, bc_low=c["bc_low"], bc_high=c["bc_high"], dtype=np.dtype(c["dtype"]).type,
                    bg=c["bg"], n_pml=c["n_pml"], use_stl=bool(c["solids"]), use_sibc=False)
    return s


def b200_grid(c):
    import wakis_b200 as wb
    g = wb.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
    if c["solids"]:
        masks = cases.step_masks(c)
        for k, mat in c["solids"].items():
            g.add_solid(k, masks[k], mat)
    return g


def b200_step_case(c, precision=None):
    import wakis_b200 as wb
    g = b200_grid(c)
    return wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"],
                          dtype=np.dtype(c["dtype"]).type, bg=c["bg"], n_pml=c["n_pml"],
                          use_stl=bool(c["solids"]), use_sibc=False, verbose=0,
                          precision=precision)


def oracle_wake_case(c):
    g0 = ofit.Grid(*c["bounds"], *c["shape"])
    m = cases.wake_mask(c, g0.x, g0.y, g0.z)
    g = ofit.Grid(*c["bounds"], *c["shape"], solids={"cav": m}, materials={"cav": c["material"]})
    w = owake.WakeOracle(**c["wake"])
    s = ofit.Solver(g, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True, bg=c["bg"],
                    dtype=np.dtype(c["dtype"]).type, wake_fmax=w.fmax)
    return s, w


def b200_wake_case(c):
    import wakis_b200 as wb
    g = wb.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
    g.add_solid("cav", cases.wake_mask(c, g.x, g.y, g.z), c["material"])
    w = wb.WakeSolver(save=False, verbose=0, **c["wake"])
    s = wb.SolverFIT3D(g, w, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True, bg=c["bg"],
                       dtype=np.dtype(c["dtype"]).type, verbose=0)
    return s, w


def rel_err(a, b):
    """max|a-b| / max|b| (0 when both vanish)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if b.size else 0.0
    return 0.0 if den == 0 and num == 0 else num / (den if den else 1.0)


def oracle_lossy_case(c):
    from wakis_b200 import workloads
    g = ofit.Grid(*workloads.BOUNDS, *c["shape"], solids={"cavity": cases.lossy_mask(c)},
                  materials={"cavity": "vacuum"})
    return ofit.Solver(g, bc_low=c["bc_low"], bc_high=c["bc_high"],
                       dtype=np.dtype(c["dtype"]).type, bg=c["bg"], n_pml=c["n_pml"],
                       use_stl=True, use_sibc=False)


def b200_lossy_case(c, precision=None):
    """The lossy case through the same builder as the benchmark workload
    (``workloads.build_b200('lossy_256', shape=...)``)."""
    from wakis_b200 import workloads
    dtype = np.float64 if precision == "fp32c" else np.dtype(c["dtype"]).type
    return workloads.build_b200("lossy_256", dtype=dtype, shape=c["shape"], precision=precision)


def oracle_sibc_case(c, wake=None):
    b, shape, wall, surf = cases.sibc_geometry(c)
    g = ofit.Grid(*b, *shape, solids={"wall": wall}, materials={"wall": [1.0, 1.0, c["sigma"]]})
    return ofit.Solver(g, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True, use_sibc=True,
                       bg="vacuum", dtype=np.dtype(c["dtype"]).type, surface_masks={"wall": surf},
                       wake_fmax=wake.fmax if wake is not None else None)


def b200_sibc_case(c, wake=None, precision=None):
    import wakis_b200 as wb
    b, shape, wall, surf = cases.sibc_geometry(c)
    g = wb.GridFIT3D(*b, *shape, verbose=0)
    g.add_solid("wall", wall, [1.0, 1.0, c["sigma"]])
    return wb.SolverFIT3D(g, wake, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True,
                          use_sibc=True, bg="vacuum", dtype=np.dtype(c["dtype"]).type, verbose=0,
                          precision=precision)
