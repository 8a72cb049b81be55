"""Time-dependent sources (upstream wakis/sources.py).

``Beam`` keeps upstream's ``update(solver, t)`` contract (sources.py:76-110):
called by a user loop it writes the Gaussian line current into ``solver.J``.
Inside ``wakesolve`` the same current is computed by the step kernel
itself (``beam_params``), so no per-step host work or transfer is needed.
"""

import numpy as np
import torch
from scipy.constants import c as c_light


class Beam:
    def __init__(self, xsource=0.0, ysource=0.0, beta=1.0, q=1e-9, sigmaz=None, ti=None):
        self.xsource, self.ysource = xsource, ysource
        self.sigmaz = sigmaz
        self.q = q
        self.beta = beta
        self.v = c_light * beta
        if ti is not None:
            self.ti = ti
        else:
            self.ti = 8.548921333333334 * self.sigmaz / self.v
        self.is_first_update = True

    def _first(self, solver):
        if self.is_first_update:
            self.ixs = int(np.abs(solver.x - self.xsource).argmin())
            self.iys = int(np.abs(solver.y - self.ysource).argmin())
            self.zmin = solver.z.min()
            self.is_first_update = False

    def params(self, solver):
        """Kernel beam parameters (ixs, iys, q*v, v, s0, c0, 2*sigmaz^2, dx, dy)
        with every constant formed by the same expressions as upstream."""
        self._first(solver)
        s0 = self.zmin - self.v * self.ti
        c0 = 1 / np.sqrt(2 * np.pi * self.sigmaz ** 2)
        two_sig2 = 2 * self.sigmaz ** 2
        return (self.ixs, self.iys, float(self.q * self.v), float(self.v), float(s0), float(c0),
                float(two_sig2), float(solver.dx[self.ixs]), float(solver.dy[self.iys]))

    def profile(self, solver, t):
        self._first(solver)
        s0 = self.zmin - self.v * self.ti
        s = solver.z - self.v * t
        return (1 / np.sqrt(2 * np.pi * self.sigmaz ** 2)
                * np.exp(-((s - s0) ** 2) / (2 * self.sigmaz ** 2)))

    def update(self, solver, t):
        """Write the line current at time t into solver.J (generic path)."""
        prof = self.profile(solver, t)
        solver.J[self.ixs, self.iys, :, "z"] = (self.q * self.v * prof / solver.dx[self.ixs]
                                               / solver.dy[self.iys])


def beam_line_values(solver, beam_params, step):
    """Jz line of the fused beam at a given step, in the solver dtype, as a
    device tensor (used when J is materialised after a non-conductive run).
    Evaluated with numpy on the Nz-long line, with upstream's float32
    time arithmetic when the time step is a float32 scalar."""
    ixs, iys, qv, v, s0, c0, two_sig2, bdx, bdy = beam_params
    if isinstance(solver.dt, np.float32):
        t = step * solver.dt
        vt = v * t
    else:
        t = step * np.float64(solver.dt)
        vt = v * t
    s = solver.z - vt
    prof = c0 * np.exp(-((s - s0) ** 2) / two_sig2)
    vals = (qv * prof / bdx / bdy).astype(solver.dtype)
    return torch.as_tensor(vals, device=solver.device)
