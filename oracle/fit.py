"""CPU oracle for the Wakis FIT leap-frog stepper.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``wakis_b200`` package imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline / ``--impl reference`` arm use it, always as the checker or as the
timed CPU baseline, never as a product code path.

It restates the upstream algorithm (Wakis 0.7.0, pure Python) with numpy and
scipy.sparse, in the same floating-point operation order, so that on the same
inputs it reproduces the upstream solver value for value:

* grid metrics ``L, iA, tL, itA``             -- wakis/gridFIT3D.py:258-300
* curl matrix and boundary folding            -- wakis/solverFIT3D.py:206-227,
                                                 wakis/boundaries.py:14-188
* material tensors (background, solids, PML)  -- wakis/solverFIT3D.py:240-273,
                                                 416-480; wakis/boundaries.py:190-311
* time step with relaxation clamp             -- wakis/solverFIT3D.py:283-310
* operator products and ``_one_step``         -- wakis/solverFIT3D.py:312-322,
                                                 482-503, 820-840
* Gaussian beam source                        -- wakis/sources.py:65-110

Parity with the upstream code itself is pinned by ``tests/golden`` fixtures
generated from the upstream package (``tests/golden/make_golden.py``) and by
the upstream regression vectors of ``tests/test_001_pec_cubic_cavity.py``.

Field storage follows upstream ``Field``: one flat array of length 3N holding
the x, y and z blocks, each block in Fortran order (i fastest),
n = i + j*Nx + k*Nx*Ny (wakis/field.py:57-76,139-190).
"""

import numpy as np
import scipy.sparse as sps
from scipy.constants import c as C_LIGHT
from scipy.constants import epsilon_0 as EPS_0
from scipy.constants import mu_0 as MU_0

# Material library (wakis/materials.py:27-41): key -> [eps_r, mu_r(, sigma)]
MATERIALS = {
    "pec": [np.inf, 1.0],
    "vacuum": [1.0, 1.0],
    "dielectric": [10.0, 1.0],
    "lossy metal": [10, 1.0, 10],
    "copper": [5.8e07, 1.0, 5.8e07],
    "berillium": [2.5e07, 1.0, 2.5e07],
    "stainless steel": [1.4e06, 1.0, 1.4e06],
}

COMP = {"x": 0, "y": 1, "z": 2}


# ----------------------------------------------------------------------------
# grid
# ----------------------------------------------------------------------------
class Grid:
    """Uniform/non-uniform Cartesian grid (wakis/gridFIT3D.py:141-180,258-300).

    ``solids`` maps a key to a boolean (Nx, Ny, Nz) cell mask and ``materials``
    maps the same key to [eps_r, mu_r(, sigma)] or a library key.  Masks stand
    in for upstream's VTK voxelisation (wakis/gridFIT3D.py:470-517), whose
    result upstream reshapes in C order (wakis/solverFIT3D.py:440).
    """

    def __init__(self, xmin=None, xmax=None, ymin=None, ymax=None, zmin=None,
                 zmax=None, Nx=None, Ny=None, Nz=None, x=None, y=None, z=None,
                 solids=None, materials=None):
        if x is not None:
            self.x, self.y, self.z = np.asarray(x), np.asarray(y), np.asarray(z)
            self.Nx, self.Ny, self.Nz = len(x) - 1, len(y) - 1, len(z) - 1
        else:
            self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
            self.x = np.linspace(xmin, xmax, Nx + 1)
            self.y = np.linspace(ymin, ymax, Ny + 1)
            self.z = np.linspace(zmin, zmax, Nz + 1)
        self.xmin, self.xmax = self.x[0], self.x[-1]
        self.ymin, self.ymax = self.y[0], self.y[-1]
        self.zmin, self.zmax = self.z[0], self.z[-1]
        self.dx, self.dy, self.dz = np.diff(self.x), np.diff(self.y), np.diff(self.z)
        self.solids = dict(solids or {})
        self.materials = {}
        for key, mat in (materials or {}).items():
            if isinstance(mat, str):
                lib = MATERIALS[mat.lower()]
                mat = [lib[0], lib[1]] + ([lib[2]] if len(lib) == 3 else [])
            self.materials[key] = list(mat)
        self._metrics()

    def _metrics(self):
        """Primal lengths L, inverse areas iA, dual lengths tL (last entry 0
        because the dual axis repeats its last point) and inverse dual areas
        itA (0 where the dual area vanishes), gridFIT3D.py:264-300."""
        Nx, Ny, Nz = self.Nx, self.Ny, self.Nz
        X, Y, Z = np.meshgrid(self.x, self.y, self.z, indexing="ij")
        f = lambda a: np.reshape(a, Nx * Ny * Nz, order="F")
        Lx = f(X[1:, 1:, 1:] - X[:-1, :-1, :-1])
        Ly = f(Y[1:, 1:, 1:] - Y[:-1, :-1, :-1])
        Lz = f(Z[1:, 1:, 1:] - Z[:-1, :-1, :-1])
        self.L = np.concatenate([Lx, Ly, Lz])
        self.iA = np.concatenate([np.divide(1.0, Ly * Lz), np.divide(1.0, Lx * Lz),
                                  np.divide(1.0, Lx * Ly)])
        tx = np.append((self.x[1:] + self.x[:-1]) / 2, 0.0)
        ty = np.append((self.y[1:] + self.y[:-1]) / 2, 0.0)
        tz = np.append((self.z[1:] + self.z[:-1]) / 2, 0.0)
        tx[-1], ty[-1], tz[-1] = tx[-2], ty[-2], tz[-2]
        tX, tY, tZ = np.meshgrid(tx, ty, tz, indexing="ij")
        tLx = f(tX[1:, 1:, 1:] - tX[:-1, :-1, :-1])
        tLy = f(tY[1:, 1:, 1:] - tY[:-1, :-1, :-1])
        tLz = f(tZ[1:, 1:, 1:] - tZ[:-1, :-1, :-1])
        self.tL = np.concatenate([tLx, tLy, tLz])

        def inv(a):
            return np.divide(1.0, a, out=np.zeros_like(a), where=a != 0)

        self.itA = np.concatenate([inv(tLy * tLz), inv(tLx * tLz), inv(tLx * tLy)])


# ----------------------------------------------------------------------------
# helpers on flat 3N arrays
# ----------------------------------------------------------------------------
def comp_view(arr, d, shape):
    """(Nx, Ny, Nz) Fortran view of component d of a flat 3N array."""
    N = shape[0] * shape[1] * shape[2]
    return arr[d * N:(d + 1) * N].reshape(shape, order="F")


def _face_mask(shape, lo, hi):
    """Per-component 0/1 mask that zeroes tangential components on the faces
    whose flag is 0; later faces overwrite earlier ones in the order x-lo,
    x-hi, y-lo, y-hi, z-lo, z-hi (boundaries.py:90-101,130-141)."""
    m = np.ones(3 * shape[0] * shape[1] * shape[2], dtype=np.int8)
    for d in range(3):
        v = comp_view(m, d, shape)
        if d != 0:
            v[0, :, :] = lo[0]
            v[-1, :, :] = hi[0]
        if d != 1:
            v[:, 0, :] = lo[1]
            v[:, -1, :] = hi[1]
        if d != 2:
            v[:, :, 0] = lo[2]
            v[:, :, -1] = hi[2]
    return m


# ----------------------------------------------------------------------------
# solver
# ----------------------------------------------------------------------------
class Solver:
    """Restatement of ``SolverFIT3D`` (wakis/solverFIT3D.py:40-354) for the
    single-process CPU path, plus ``_one_step`` (482-503)."""

    def __init__(self, grid, bc_low=("periodic",) * 3, bc_high=("periodic",) * 3,
                 use_stl=False, use_sibc=True, fmax=1e9, dtype=np.float64,
                 n_pml=10, bg=(1.0, 1.0), cfln=0.5, dt=None, wake_fmax=None,
                 surface_masks=None):
        self.grid = grid
        self.dtype = dtype
        self.Nx, self.Ny, self.Nz = grid.Nx, grid.Ny, grid.Nz
        self.N = N = self.Nx * self.Ny * self.Nz
        self.shape = (self.Nx, self.Ny, self.Nz)
        self.dx, self.dy, self.dz = grid.dx, grid.dy, grid.dz
        self.x = grid.x[:-1] + self.dx / 2
        self.y = grid.y[:-1] + self.dy / 2
        self.z = grid.z[:-1] + self.dz / 2
        self.fmax = wake_fmax if (wake_fmax is not None and fmax == 1e9) else fmax
        self.bc_low, self.bc_high = list(bc_low), list(bc_high)
        self.use_conductivity = False
        self.activate_pml = False
        self.activate_abc = False
        self.step_0 = True

        self.E = np.zeros(3 * N, dtype=dtype)
        self.H = np.zeros(3 * N, dtype=dtype)
        self.J = np.zeros(3 * N, dtype=dtype)

        L, iA = grid.L, grid.iA
        tL, itA = grid.tL.copy(), grid.itA.copy()
        self._bcs(L, iA, tL, itA)

        # materials (solverFIT3D.py:240-270)
        if isinstance(bg, str):
            bg = MATERIALS[bg.lower()]
        bg = list(bg)
        eps_bg, mu_bg = bg[0] * EPS_0, bg[1] * MU_0
        self.sigma_bg = 0.0
        if len(bg) == 3:
            self.sigma_bg = bg[2]
            self.use_conductivity = True
        self.ieps = np.ones(3 * N, dtype=dtype) * (1.0 / eps_bg)
        self.imu = np.ones(3 * N, dtype=dtype) * (1.0 / mu_bg)
        self.sigma = np.ones(3 * N, dtype=dtype) * self.sigma_bg
        if use_stl:
            self._solids(use_sibc, surface_masks or {})
        if self.activate_pml:
            self.n_pml = n_pml
            self._pml()

        # time step (solverFIT3D.py:286-310)
        if dt is None:
            dt = cfln / (C_LIGHT * np.sqrt(1 / np.min(grid.dx) ** 2
                                           + 1 / np.min(grid.dy) ** 2
                                           + 1 / np.min(grid.dz) ** 2))
        self.dt = dtype(dt)
        if self.use_conductivity:
            m = np.logical_and(self.sigma != 0, self.ieps != 0)
            self.tau = (1 / self.ieps[m]) / self.sigma[m]
            if self.dt > self.tau.min():
                self.dt = self.tau.min()

        self._metrics = (L, iA, tL, itA)
        self._operators(L, iA, tL, itA)

    # -- boundaries (boundaries.py:14-188) ----------------------------------
    def _bcs(self, L, iA, tL, itA):
        Nx, Ny, Nz, N = self.Nx, self.Ny, self.Nz, self.N
        lo, hi = self.bc_low, self.bc_high
        Px = sps.diags([-1, 1], [0, 1], shape=(N, N), dtype=np.int8)
        Py = sps.diags([-1, 1], [0, Nx], shape=(N, N), dtype=np.int8)
        Pz = sps.diags([-1, 1], [0, Nx * Ny], shape=(N, N), dtype=np.int8)
        Z0 = sps.csc_matrix((N, N))
        C = sps.vstack([sps.hstack([Z0, -Pz, Py]), sps.hstack([Pz, Z0, -Px]),
                        sps.hstack([-Py, Px, Z0])], dtype=np.int8)

        def copy_high(axis):
            # dual length of the last cell := first primal length; inverse
            # dual areas of the two transverse components := first primal ones
            for d in range(3):
                t, ia, ita = (comp_view(tL, d, self.shape), comp_view(iA, d, self.shape),
                              comp_view(itA, d, self.shape))
                l = comp_view(L, d, self.shape)
                sl_hi = [slice(None)] * 3
                sl_lo = [slice(None)] * 3
                sl_hi[axis], sl_lo[axis] = -1, 0
                if d == axis:
                    t[tuple(sl_hi)] = l[tuple(sl_lo)]
                else:
                    ita[tuple(sl_hi)] = ia[tuple(sl_lo)]

        if any(b.lower() == "periodic" for b in lo):
            for a in range(3):
                if lo[a].lower() == "periodic" and hi[a].lower() == "periodic":
                    copy_high(a)
        lo_f, hi_f = [1, 1, 1], [1, 1, 1]
        pec = ("electric", "pec", "pml")
        self.pec_mask = None
        if any(b.lower() in pec for b in lo) or any(b.lower() in pec for b in hi):
            for a in range(3):
                if lo[a].lower() in pec:
                    lo_f[a] = 0
                if hi[a].lower() in pec:
                    hi_f[a] = 0
            self.pec_mask = _face_mask(self.shape, lo_f, hi_f)
            C = C @ sps.diags(self.pec_mask, shape=(3 * N, 3 * N), dtype=np.int8)
        raw_lo, raw_hi = lo, hi
        self.pmc_mask = None
        if any(b.lower() in ("magnetic", "pmc") for b in raw_lo) or any(
                b.lower() in ("magnetic", "pmc") for b in raw_hi):
            for a in range(3):
                if raw_lo[a].lower() == "magnetic" or raw_lo[a] == "pmc":
                    lo_f[a] = 0
                if raw_hi[a].lower() == "magnetic" or raw_hi[a] == "pmc":
                    hi_f[a] = 0
            self.pmc_mask = _face_mask(self.shape, lo_f, hi_f)
            C = sps.diags(self.pmc_mask, shape=(3 * N, 3 * N), dtype=np.int8) @ C
        if any(b.lower() == "abc" for b in lo) or any(b.lower() == "abc" for b in hi):
            for a in range(3):
                if hi[a].lower() == "abc":
                    copy_high(a)
            self.activate_abc = True
        if any(b.lower() == "pml" for b in lo) or any(b.lower() == "pml" for b in hi):
            self.activate_pml = True
            self.use_conductivity = True
        self.C = C

    # -- solids (solverFIT3D.py:416-480) ------------------------------------
    def _solids(self, use_sibc, surface_masks):
        dt_ = self.dtype
        for key, mask in self.grid.solids.items():
            mat = self.grid.materials[key]
            mask = np.asarray(mask, dtype=bool)
            eps = mat[0] * EPS_0
            mu = mat[1] * MU_0
            dn = np.sqrt(2) * min(self.dx.min(), self.dy.min(), self.dz.min())
            sigma_max = 10 / (np.pi * self.fmax * mu * dn ** 2)
            m3 = np.tile(mask.ravel(order="F"), 3)
            if len(mat) == 3:
                sig = mat[2]
                if use_sibc and mat[2] > sigma_max:
                    mask = np.asarray(surface_masks[key], dtype=bool)
                    m3 = np.tile(mask.ravel(order="F"), 3)
                    imp = np.sqrt(np.pi * self.fmax * mu / sig)
                    sig = 1 / imp
                    eps = 1 / imp
                self.sigma[m3] = dt_(sig)
                self.use_conductivity = True
            elif self.sigma_bg > 0.0:
                self.sigma[m3] = dt_(0.0)
            self.ieps[m3] = dt_(1.0 / eps)
            self.imu[m3] = dt_(1.0 / mu)

    # -- PML (boundaries.py:190-311) ----------------------------------------
    def _pml(self):
        n = self.n_pml
        lo_hi = np.geomspace(10.0, 5.0e-3, n)
        hi_lo = np.geomspace(5.0e-3, 10.0, n)
        Nx, Ny, Nz = self.shape
        probe = {0: lambda p: (p, Ny // 2, Nz // 2), 1: lambda p: (Nx // 2, p, Nz // 2),
                 2: lambda p: (Nx // 2, Ny // 2, p)}
        for side in ("lo", "hi"):
            for a in range(3):
                b = self.bc_low[a] if side == "lo" else self.bc_high[a]
                if b.lower() != "pml":
                    continue
                prof = lo_hi if side == "lo" else hi_lo
                pos = n + 1 if side == "lo" else -(n + 1)
                for d in range(3):
                    ie = comp_view(self.ieps, d, self.shape)
                    sg = comp_view(self.sigma, d, self.shape)
                    ie0 = ie[probe[a](pos)]
                    s0 = sg[probe[a](pos)]
                    mult = 1 if s0 < 1 else s0
                    for p in range(n):
                        idx = p if side == "lo" else -(p + 1)
                        prof_v = prof[p] if side == "lo" else prof[n - 1 - p]
                        sl = [slice(None)] * 3
                        sl[a] = idx
                        ie[tuple(sl)] = ie0
                        sg[tuple(sl)] = s0 + mult * prof_v

    # -- operators (solverFIT3D.py:212-217,315-322) -------------------------
    def _operators(self, L, iA, tL, itA):
        N3 = 3 * self.N
        dt_ = self.dtype
        D = lambda v: sps.diags(v, shape=(N3, N3), dtype=dt_)
        Ds, iDa, tDs, itDa = D(L), D(iA), D(tL), D(itA)
        iDeps, iDmu = D(self.ieps), D(self.imu)
        self.A = iDa * iDmu * self.C * Ds
        self.B = iDeps * itDa * self.C.transpose() * tDs
        self._dtA = None

    def update_tensors(self):
        """Re-form the operators after edits of ieps / imu / sigma
        (solverFIT3D.py:356-414, tensor='all'); dt is not re-evaluated and
        the first-step ghost zeroing is skipped, as upstream."""
        self._operators(*self._metrics)
        self.step_0 = False

    # -- time stepping ------------------------------------------------------
    def zero_ghosts(self):
        """solverFIT3D.py:820-840: tangential H on the high faces and the
        E component along each axis in the last cell of that axis."""
        s = self.shape
        for d in range(3):
            h = comp_view(self.H, d, s)
            if d != 0:
                h[-1, :, :] = 0.0
            if d != 1:
                h[:, -1, :] = 0.0
            if d != 2:
                h[:, :, -1] = 0.0
        comp_view(self.E, 0, s)[-1, :, :] = 0.0
        comp_view(self.E, 1, s)[:, -1, :] = 0.0
        comp_view(self.E, 2, s)[:, :, -1] = 0.0

    def set_threads(self, threads):
        """Split both operators into row blocks evaluated by a thread pool
        (scipy's CSR mat-vec releases the GIL); each row keeps its stored
        order, so results are unchanged."""
        self._threads = int(threads)
        self._pool = None
        self._dtA = None
        if self._threads > 1:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(self._threads)

    def _matvec(self, M, blocks, x):
        if blocks is None:
            return M * x
        parts = list(self._pool.map(lambda b: b * x, blocks))
        return np.concatenate(parts)

    def _blocks(self, M):
        t = getattr(self, "_threads", 1)
        if t <= 1:
            return None
        n = M.shape[0]
        cuts = [n * i // t for i in range(t + 1)]
        return [M[cuts[i]:cuts[i + 1]] for i in range(t)]

    def one_step(self):
        """H <- H - dt*A*E; E <- E + dt*(B*H - ieps*J); J <- sigma*E
        (solverFIT3D.py:482-503).  ``dt*A`` is formed as a scaled matrix as in
        upstream's left-to-right evaluation of ``dt * A * E``."""
        if self.step_0:
            self.zero_ghosts()
            self.step_0 = False
        if self._dtA is None or self._dtA_dt != self.dt:
            self._dtA = self.dt * self.A
            self._dtA_dt = self.dt
            self._dtA_blocks = self._blocks(self._dtA)
            self._B_blocks = self._blocks(self.B)
        self.H[:] = self.H - self._matvec(self._dtA, self._dtA_blocks, self.E)
        self.E[:] = self.E + self.dt * (self._matvec(self.B, self._B_blocks, self.H)
                                        - self.ieps * self.J)
        if self.use_conductivity:
            self.J[:] = self.sigma * self.E


# ----------------------------------------------------------------------------
# beam source (sources.py:22-110)
# ----------------------------------------------------------------------------
class Beam:
    def __init__(self, xsource=0.0, ysource=0.0, beta=1.0, q=1e-9, sigmaz=None, ti=None):
        self.xsource, self.ysource = xsource, ysource
        self.sigmaz, self.q, self.beta = sigmaz, q, beta
        self.v = C_LIGHT * beta
        self.ti = ti if ti is not None else 8.548921333333334 * self.sigmaz / self.v
        self.first = True

    def line(self, solver, t):
        """Jz values on the beam line at time t (float64, before the cast to
        the solver dtype done by the Field assignment)."""
        if self.first:
            self.ixs = np.abs(solver.x - self.xsource).argmin()
            self.iys = np.abs(solver.y - self.ysource).argmin()
            self.zmin = solver.z.min()
            self.first = False
        s0 = self.zmin - self.v * self.ti
        s = solver.z - self.v * t
        prof = (1 / np.sqrt(2 * np.pi * self.sigmaz ** 2)
                * np.exp(-((s - s0) ** 2) / (2 * self.sigmaz ** 2)))
        return self.q * self.v * prof / solver.dx[self.ixs] / solver.dy[self.iys]

    def update(self, solver, t):
        vals = self.line(solver, t)
        jz = comp_view(solver.J, 2, solver.shape)
        jz[self.ixs, self.iys, :] = vals
