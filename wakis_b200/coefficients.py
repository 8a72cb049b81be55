"""Host-side construction of the compact coefficient set the step kernels read.

Upstream assembles two 3N x 3N sparse operators from per-cell, per-component
fields (wakis/solverFIT3D.py:203-322).  The kernels instead read

* separable metrics: 1-D primal/dual edge lengths per axis and 2-D inverse
  face-area tables (iAx[j,k], iAy[i,k], iAz[i,j] and the dual ones), with
  upstream's boundary edits applied (wakis/boundaries.py:35-70,152-181);
* a per-cell material id into a small table of (ieps, imu, sigma) x 3
  components, built by replaying upstream's material assignments
  (background 240-270, solids 416-480, PML boundaries.py:190-311) on ids;
* the PEC/PMC face flags (boundaries.py:72-150);
* the time step with the relaxation-time clamp (solverFIT3D.py:283-310).

All values are computed with the same numpy operations as upstream, then
cast to the solver dtype as upstream's ``diags(..., dtype)`` does, so the
kernels see exactly the operator entries upstream's matrices hold.
"""

from dataclasses import dataclass, field

import numpy as np
from scipy.constants import c as C_LIGHT
from scipy.constants import epsilon_0 as EPS_0
from scipy.constants import mu_0 as MU_0

from .materials import material_lib

PEC_LIKE = ("electric", "pec", "pml")


@dataclass
class Coefficients:
    dtype: type
    shape: tuple
    Lx: np.ndarray
    Ly: np.ndarray
    Lz: np.ndarray
    tLx: np.ndarray
    tLy: np.ndarray
    tLz: np.ndarray
    iAx: np.ndarray      # (Ny, Nz)
    iAy: np.ndarray      # (Nx, Nz)
    iAz: np.ndarray      # (Nx, Ny)
    itAx: np.ndarray
    itAy: np.ndarray
    itAz: np.ndarray
    ids: np.ndarray      # (N,) flat Fortran order
    table: np.ndarray    # (n_mat, 9): ieps xyz, imu xyz, sigma xyz
    pec_face: list
    pmc_face: list
    has_pec: bool
    has_pmc: bool
    h_sum_desc: bool
    use_conductivity: bool
    activate_pml: bool
    activate_abc: bool
    dt: object
    tau_min: object = None
    sigma_bg: float = 0.0
    info: dict = field(default_factory=dict)

    @property
    def id_bytes(self):
        return self.ids.dtype.itemsize


def _inv_outer(a, b):
    p = np.multiply.outer(a, b)
    return np.divide(1.0, p, out=np.zeros_like(p), where=p != 0)


def boundary_flags(bc_low, bc_high):
    """Face flags (x-lo, x-hi, y-lo, y-hi, z-lo, z-hi) of the PEC column
    mask and the PMC row mask.  The PMC flags start from the PEC ones, as
    upstream reuses the same face variables (boundaries.py:24-127)."""
    lo_f, hi_f = [1, 1, 1], [1, 1, 1]
    has_pec = any(b.lower() in PEC_LIKE for b in bc_low) or any(
        b.lower() in PEC_LIKE for b in bc_high)
    if has_pec:
        for a in range(3):
            if bc_low[a].lower() in PEC_LIKE:
                lo_f[a] = 0
            if bc_high[a].lower() in PEC_LIKE:
                hi_f[a] = 0
    pec_face = [lo_f[0], hi_f[0], lo_f[1], hi_f[1], lo_f[2], hi_f[2]]
    has_pmc = any(b.lower() in ("magnetic", "pmc") for b in bc_low) or any(
        b.lower() in ("magnetic", "pmc") for b in bc_high)
    if has_pmc:
        for a in range(3):
            if bc_low[a].lower() == "magnetic" or bc_low[a] == "pmc":
                lo_f[a] = 0
            if bc_high[a].lower() == "magnetic" or bc_high[a] == "pmc":
                hi_f[a] = 0
    pmc_face = [lo_f[0], hi_f[0], lo_f[1], hi_f[1], lo_f[2], hi_f[2]]
    return pec_face, pmc_face, has_pec, has_pmc


class _Table:
    """Deduplicated material rows in the solver dtype."""

    def __init__(self, dtype):
        self.dtype = dtype
        self.rows = []
        self.index = {}

    def add(self, row):
        row = tuple(self.dtype(v) for v in row)
        key = tuple(float(v) for v in row)
        if key not in self.index:
            self.index[key] = len(self.rows)
            self.rows.append(row)
        return self.index[key]


def build(grid, bc_low, bc_high, dtype=np.float64, bg=(1.0, 1.0), use_stl=False,
          use_sibc=True, fmax=1e9, n_pml=10, cfln=0.5, dt=None, verbose=0):
    """Compact coefficients of SolverFIT3D(grid, ...) (solverFIT3D.py:40-354)."""
    dt_ = np.dtype(dtype).type
    Nx, Ny, Nz = grid.Nx, grid.Ny, grid.Nz
    N = Nx * Ny * Nz
    bc_low, bc_high = list(bc_low), list(bc_high)

    # ---- metrics (gridFIT3D.py:264-300) + boundary edits ----------------
    Lx, Ly, Lz = grid.dx.copy(), grid.dy.copy(), grid.dz.copy()
    tLx, tLy, tLz = grid.tdx.copy(), grid.tdy.copy(), grid.tdz.copy()
    iAx = np.divide(1.0, np.multiply.outer(Ly, Lz))
    iAy = np.divide(1.0, np.multiply.outer(Lx, Lz))
    iAz = np.divide(1.0, np.multiply.outer(Lx, Ly))
    itAx, itAy, itAz = _inv_outer(tLy, tLz), _inv_outer(tLx, tLz), _inv_outer(tLx, tLy)

    def copy_high(axis):
        if axis == 0:
            tLx[-1] = Lx[0]
            itAy[-1, :] = iAy[0, :]
            itAz[-1, :] = iAz[0, :]
        elif axis == 1:
            tLy[-1] = Ly[0]
            itAx[-1, :] = iAx[0, :]
            itAz[:, -1] = iAz[:, 0]
        else:
            tLz[-1] = Lz[0]
            itAx[:, -1] = iAx[:, 0]
            itAy[:, -1] = iAy[:, 0]

    if any(b.lower() == "periodic" for b in bc_low):
        for a in range(3):
            if bc_low[a].lower() == "periodic" and bc_high[a].lower() == "periodic":
                copy_high(a)
    pec_face, pmc_face, has_pec, has_pmc = boundary_flags(bc_low, bc_high)
    activate_abc = any(b.lower() == "abc" for b in bc_low) or any(
        b.lower() == "abc" for b in bc_high)
    if activate_abc:
        for a in range(3):
            if bc_high[a].lower() == "abc":
                copy_high(a)
    activate_pml = any(b.lower() == "pml" for b in bc_low) or any(
        b.lower() == "pml" for b in bc_high)
    use_conductivity = activate_pml

    # ---- materials (solverFIT3D.py:240-270,416-480) ---------------------
    if isinstance(bg, str):
        bg = material_lib[bg.lower()]
    bg = list(bg)
    eps_bg, mu_bg = bg[0] * EPS_0, bg[1] * MU_0
    sigma_bg = 0.0
    if len(bg) == 3:
        sigma_bg = bg[2]
        use_conductivity = True
    one = np.ones(1, dtype=dt_)
    row_bg = [(one * (1.0 / eps_bg))[0]] * 3 + [(one * (1.0 / mu_bg))[0]] * 3 \
        + [(one * sigma_bg)[0]] * 3
    tab = _Table(dt_)
    tab.add(row_bg)
    ids = np.zeros(N, dtype=np.int32)

    if use_stl:
        dxm = min(grid.dx.min(), grid.dy.min(), grid.dz.min())
        for key in grid.stl_solids:
            mat = grid.stl_materials[key]
            mask = np.reshape(grid.grid[key], (Nx, Ny, Nz))
            eps = mat[0] * EPS_0
            mu = mat[1] * MU_0
            dn = np.sqrt(2) * dxm
            sigma_max = 10 / (np.pi * fmax * mu * dn ** 2)
            new_sigma = None          # None: keep the cell's sigma
            if len(mat) == 3:
                sig = mat[2]
                if use_sibc and mat[2] > sigma_max:
                    grid._mark_cells_in_surface(key)
                    mask = np.reshape(grid.grid[key], (Nx, Ny, Nz))
                    imp = np.sqrt(np.pi * fmax * mu / sig)
                    sig = 1 / imp
                    eps = 1 / imp
                new_sigma = sig
                use_conductivity = True
            elif sigma_bg > 0.0:
                new_sigma = 0.0
            m = mask.ravel(order="F")
            old = np.unique(ids[m])
            lut = np.arange(len(tab.rows) + len(old) + 1, dtype=np.int64)
            for o in old:
                r = tab.rows[o]
                sg = r[6:9] if new_sigma is None else [new_sigma] * 3
                lut[o] = tab.add([1.0 / eps] * 3 + [1.0 / mu] * 3 + list(sg))
            ids[m] = lut[ids[m]]

    # ---- PML (boundaries.py:190-311) ------------------------------------
    if activate_pml:
        ids3 = ids.reshape((Nx, Ny, Nz), order="F")
        dims = (Nx, Ny, Nz)
        for side in ("lo", "hi"):
            for a in range(3):
                b = bc_low[a] if side == "lo" else bc_high[a]
                if b.lower() != "pml":
                    continue
                s = np.zeros(dims[a])
                if side == "lo":
                    s[0:n_pml] = np.geomspace(10.0, 5.0e-3, n_pml)
                    pos = n_pml + 1
                else:
                    s[-n_pml:] = np.geomspace(5.0e-3, 10.0, n_pml)
                    pos = dims[a] - (n_pml + 1)
                probe = [Nx // 2, Ny // 2, Nz // 2]
                probe[a] = pos
                pid = ids3[tuple(probe)]
                prow = tab.rows[pid]
                ieps0 = [prow[d] for d in range(3)]
                sig0 = [prow[6 + d] for d in range(3)]
                mult = [1 if sig0[d] < 1 else sig0[d] for d in range(3)]
                for p in range(n_pml):
                    plane = p if side == "lo" else dims[a] - 1 - p
                    sv = [sig0[d] + mult[d] * s[plane] for d in range(3)]
                    sl = [slice(None)] * 3
                    sl[a] = plane
                    view = ids3[tuple(sl)]
                    old = np.unique(view)
                    lut = {}
                    for o in old:
                        r = tab.rows[o]
                        lut[o] = tab.add(ieps0 + list(r[3:6]) + sv)
                    lut_a = np.arange(max(max(lut) + 1, 1))
                    for o, v in lut.items():
                        lut_a[o] = v
                    ids3[tuple(sl)] = lut_a[view]

    # ---- compact the table to the ids in use ----------------------------
    used = np.unique(ids)
    remap = np.zeros(len(tab.rows), dtype=np.int64)
    remap[used] = np.arange(len(used))
    table = np.array([tab.rows[u] for u in used], dtype=dt_).reshape(len(used), 9)
    ids = remap[ids]
    id_t = np.uint8 if len(used) <= 256 else (np.uint16 if len(used) <= 65536 else np.uint32)
    ids = ids.astype(id_t)

    # ---- time step (solverFIT3D.py:286-310) -----------------------------
    if dt is None:
        dt = cfln / (C_LIGHT * np.sqrt(1 / np.min(grid.dx) ** 2 + 1 / np.min(grid.dy) ** 2
                                       + 1 / np.min(grid.dz) ** 2))
    dt = dt_(dt)
    tau_min = None
    if use_conductivity:
        ie = table[:, 0:3].ravel()
        sg = table[:, 6:9].ravel()
        m = np.logical_and(sg != 0, ie != 0)
        tau = (1 / ie[m]) / sg[m]
        tau_min = tau.min()          # ValueError when empty, as upstream
        if dt > tau_min:
            dt = tau_min

    cast = lambda a: np.ascontiguousarray(a, dtype=dt_)
    return Coefficients(
        dtype=dt_, shape=(Nx, Ny, Nz),
        Lx=cast(Lx), Ly=cast(Ly), Lz=cast(Lz), tLx=cast(tLx), tLy=cast(tLy), tLz=cast(tLz),
        iAx=cast(iAx), iAy=cast(iAy), iAz=cast(iAz),
        itAx=cast(itAx), itAy=cast(itAy), itAz=cast(itAz),
        ids=ids, table=table, pec_face=pec_face, pmc_face=pmc_face, has_pec=has_pec,
        has_pmc=has_pmc, h_sum_desc=(int(has_pec) + int(has_pmc)) == 1,
        use_conductivity=use_conductivity, activate_pml=activate_pml,
        activate_abc=activate_abc, dt=dt, tau_min=tau_min, sigma_bg=sigma_bg)


def dense_materials(coef):
    """Per-cell, per-component (ieps, imu, sigma) flat 3N arrays."""
    t = coef.table
    ids = coef.ids.astype(np.int64)
    out = []
    for base in (0, 3, 6):
        out.append(np.concatenate([t[ids, base + d] for d in range(3)]))
    return out
