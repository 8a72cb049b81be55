"""CPU oracle for the Wakis ``wakesolve`` loop and wake post-processing.

TEST INFRASTRUCTURE ONLY (see ``oracle/fit.py``).  Restates, in the same
floating-point order:

* ``RoutinesMixin.wakesolve`` time loop: beam injection, Ez window capture
  before each step, step count from the wakelength
  -- wakis/routines.py:322-476
* ``WakeSolver`` injection time and defaults   -- wakis/wakeSolver.py:133-173
* ``calc_long_WP_3d`` (incl. the carry-over of the running sum from one
  transverse position to the next, 485/530/536)  -- wakis/wakeSolver.py:422-554
* ``calc_long_WP``                             -- wakis/wakeSolver.py:310-420
* ``calc_trans_WP`` (Panofsky-Wenzel)          -- wakis/wakeSolver.py:556-629
* ``calc_long_Z`` / ``calc_trans_Z``           -- wakis/wakeSolver.py:631-781
* ``calc_lambdas_analytic``                    -- wakis/wakeSolver.py:838-870

The Ez history is held in memory as a dict keyed like the upstream HDF5 file
(``'#' + zfill(5)``), and read back in sorted key order as upstream does
(wakeSolver.py:488-491).
"""

import numpy as np
from scipy.constants import c as C_LIGHT

from .fit import Beam, comp_view


class WakeOracle:
    def __init__(self, q=1e-9, sigmaz=1e-3, beta=1.0, xsource=0.0, ysource=0.0,
                 xtest=0.0, ytest=0.0, ti=None, fmax=None, skip_cells=0,
                 counter_moving=False, compute_plane="both"):
        self.q, self.sigmaz, self.beta = q, sigmaz, beta
        self.v = self.beta * C_LIGHT
        self.xsource, self.ysource = xsource, ysource
        self.xtest, self.ytest = xtest, ytest
        self.fmax = self.v / (3.0 * self.sigmaz) if fmax is None else fmax
        self.skip_cells = skip_cells
        self.counter_moving = counter_moving
        self.compute_plane = compute_plane
        if ti is not None:
            self.ti = ti
        else:
            self.ti = 8.548921333333334 * self.sigmaz / (np.sqrt(self.beta) * self.v)
        self.wakelength = None
        self.n_transverse_cells = 1
        self.lambdas = None
        self.hist = None

    # ------------------------------------------------------------------
    def solve(self, compute_plane=None):
        cp = (compute_plane or self.compute_plane).lower()
        if cp in ("both", "transverse"):
            self.calc_long_WP_3d()
            self.calc_trans_WP()
            self.calc_long_Z()
            self.calc_trans_Z()
        elif cp == "longitudinal":
            self.calc_long_WP()
            self.calc_long_Z()

    def _keys(self):
        return sorted(k for k in self.hist if isinstance(k, str) and k.startswith("#"))

    def _s_axis(self):
        nt = len(self.t)
        dt = self.t[2] - self.t[1]
        zmax, zmin = np.max(self.zf), np.min(self.zf)
        zz = slice(self.skip_cells, -self.skip_cells) if self.skip_cells != 0 else np.s_[:]
        z = self.zf[zz]
        if self.wakelength is not None:
            wakelength = self.wakelength
        else:
            wakelength = nt * dt * self.v - (zmax - zmin) - self.ti * self.v
            self.wakelength = wakelength
        s = np.arange(-self.ti * self.v, wakelength, dt * self.v)
        return nt, dt, zmin, zmax, zz, z, s

    def calc_long_WP_3d(self):
        nt, dt, zmin, zmax, zz, z, s = self._s_axis()
        nz = len(z)
        i0 = j0 = self.n_transverse_cells
        WP = np.zeros_like(s)
        WP_3d = np.zeros((2 * i0 + 1, 2 * j0 + 1, len(s)))
        Ezt = np.zeros((nz, nt))
        keys = self._keys()
        nt = min(nt, len(keys))
        for i in range(-i0, i0 + 1):
            for j in range(-j0, j0 + 1):
                for n in range(nt):
                    Ez = self.hist[keys[n]]
                    Ezt[:, n] = Ez[Ez.shape[0] // 2 + i, Ez.shape[1] // 2 + j, zz]
                WP = self._integrate(WP, Ezt, s, z, zmin, zmax, dt, nt, nz)
                WP = WP / (self.q * 1e12)
                WP_3d[i0 + i, j0 + j, :] = WP
        self.s = s
        self.WP = WP_3d[i0, j0, :]
        self.WP_3d = WP_3d

    def calc_long_WP(self):
        nt, dt, zmin, zmax, zz, z, s = self._s_axis()
        nz = len(z)
        WP = np.zeros_like(s)
        keys = self._keys()
        nt = min(nt, len(keys))
        Ezt = np.zeros((nz, nt))
        Ez = self.hist[keys[0]]
        if len(Ez.shape) == 3:
            for n in range(nt):
                Ez = self.hist[keys[n]]
                Ezt[:, n] = Ez[Ez.shape[0] // 2 + 1, Ez.shape[1] // 2 + 1, zz]
        elif len(Ez.shape) == 1:
            for n in range(nt):
                Ezt[:, n] = self.hist[keys[n]]
        self.Ezt = Ezt
        WP = self._integrate_plain(WP, Ezt, s, z, zmin, dt, nt, nz)
        self.s = s
        self.WP = WP / (self.q * 1e12)

    def _integrate_plain(self, WP, Ezt, s, z, zmin, dt, nt, nz):
        """Sequential-in-k sum of Ez(k, int(ts/dt))*dz[k] for every s
        (wakeSolver.py:398-404), vectorised over s only."""
        for k in range(nz):
            ts = (z[k] + s) / self.v - zmin / self.v - self.t[0] + self.ti
            it = (ts / dt).astype(np.int64)
            ok = it < nt
            WP[ok] = WP[ok] + Ezt[k, it[ok]] * self.dz[k]
        return WP

    def _integrate(self, WP, Ezt, s, z, zmin, zmax, dt, nt, nz):
        if not self.counter_moving:
            return self._integrate_plain(WP, Ezt, s, z, zmin, dt, nt, nz)
        for k in range(nz):   # wakeSolver.py:503-517
            ts = (z[-k - 1] - s) / (-1 * self.v) - zmax / (-1 * self.v) - self.t[0] + self.ti
            it = (ts / dt).astype(np.int64)
            ok = it < nt
            WP[ok] = WP[ok] + (Ezt[-k - 1, it[ok]]) * (-1 * self.dz[k])
        return WP

    def calc_trans_WP(self):
        ds = self.s[2] - self.s[1]
        i0 = j0 = self.n_transverse_cells
        WPx = np.zeros_like(self.s)
        WPy = np.zeros_like(self.s)
        int_WP = np.zeros_like(self.WP_3d)
        dxf, dyf = np.diff(self.xf), np.diff(self.yf)
        for n in range(len(self.s)):
            for i in range(-i0, i0 + 1):
                for j in range(-j0, j0 + 1):
                    int_WP[i0 + i, j0 + j, n] = np.sum(self.WP_3d[i0 + i, j0 + j, 0:n]) * ds
            WPx[n] = -(int_WP[i0 + 1, j0, n] - int_WP[i0 - 1, j0, n]) / (dxf[i0 - 1] + dxf[i0])
            WPy[n] = -(int_WP[i0, j0 + 1, n] - int_WP[i0, j0 - 1, n]) / (dyf[j0 - 1] + dyf[j0])
        self.WPx, self.WPy = WPx, WPy

    def calc_lambdas_analytic(self):
        self.lambdas = (1 / (self.sigmaz * np.sqrt(2 * np.pi))
                        * np.exp(-(self.s ** 2) / (2 * self.sigmaz ** 2)))

    def _dft_setup(self, samples, fmax):
        ds = np.mean(self.s[1:] - self.s[:-1])
        fmax = self.fmax if fmax is None else fmax
        N = int((self.v / ds) // fmax * samples)
        return ds, fmax, N

    def calc_long_Z(self, samples=1001, fmax=None):
        if self.lambdas is None:
            self.calc_lambdas_analytic()
        ds, fmax, N = self._dft_setup(samples, fmax)
        lambdafft = np.fft.fft(self.lambdas * self.v, n=N)
        WPfft = np.fft.fft(self.WP * 1e12, n=N)
        ffft = np.fft.fftfreq(len(WPfft), ds / self.v)
        mask = np.logical_and(ffft >= 0, ffft < fmax)
        WPf = WPfft[mask] * ds
        lambdaf = lambdafft[mask] * ds
        self.f = ffft[mask]
        self.Z = -WPf / lambdaf
        self.lambdaf = lambdaf

    def calc_trans_Z(self, samples=1001, fmax=None):
        ds, fmax, N = self._dft_setup(samples, fmax)
        lambdafft = np.fft.fft(self.lambdas * self.v, n=N)
        ffft = np.fft.fftfreq(len(lambdafft), ds / self.v)
        mask = np.logical_and(ffft >= 0, ffft < fmax)
        lambdaf = lambdafft[mask] * ds
        WPxf = np.fft.fft(self.WPx * 1e12, n=N)[mask] * ds
        self.Zx = 1j * WPxf / lambdaf
        WPyf = np.fft.fft(self.WPy * 1e12, n=N)[mask] * ds
        self.Zy = 1j * WPyf / lambdaf
        self.fx = self.fy = ffft[mask]


def wakesolve(solver, wake, wakelength, compute_plane="both", max_steps=None):
    """Time loop of ``RoutinesMixin.wakesolve`` (routines.py:338-476) on the
    oracle solver; the Ez window is captured before every step.  ``max_steps``
    truncates the loop (for step-level comparisons) and skips the
    post-processing."""
    ixt = np.abs(solver.x - wake.xtest).argmin()
    iyt = np.abs(solver.y - wake.ytest).argmin()
    if compute_plane.lower() == "longitudinal":
        xx, yy = ixt, iyt
    else:
        xx, yy = slice(ixt - 1, ixt + 2), slice(iyt - 1, iyt + 2)
    wake.wakelength = wakelength
    z = solver.z
    tmax = (wakelength + wake.ti * wake.v + (z.max() - z.min())) / wake.v
    Nt = int(tmax / solver.dt)
    solver.Nt, solver.tmax = Nt, tmax
    beam = Beam(q=wake.q, sigmaz=wake.sigmaz, beta=wake.beta,
                xsource=wake.xsource, ysource=wake.ysource)
    wake.hist = {}
    wake.xf, wake.yf, wake.zf = solver.x[xx], solver.y[yy], z[slice(0, solver.Nz)]
    wake.dx, wake.dy, wake.dz = solver.grid.dx, solver.grid.dy, solver.grid.dz
    wake.t = np.arange(0, Nt * solver.dt, solver.dt)
    ez = lambda: comp_view(solver.E, 2, solver.shape)
    steps = Nt if max_steps is None else min(Nt, max_steps)
    for n in range(steps):
        beam.update(solver, n * solver.dt)
        wake.hist["#" + str(n).zfill(5)] = np.array(ez()[xx, yy, slice(0, solver.Nz)])
        solver.one_step()
    solver.beam = beam
    if max_steps is None:
        wake.solve(compute_plane)
    return Nt
