"""Time-dependent sources (upstream wakis/sources.py).

Every source keeps upstream's duck-typed ``update(solver, t)`` contract
(sources.py:11-14): ``emsolve`` calls it before each step and it writes its
values into ``solver.E``, ``solver.H`` or ``solver.J`` (device fields).
``Beam`` (sources.py:76-110) is also computed by the step kernel itself
inside ``wakesolve`` (``beam_params``), so no per-step host work or transfer
is needed there.  ``PlaneWave``, ``WavePacket``, ``Dipole`` and ``Pulse``
(sources.py:142-762) are hard sources on a box (a plane or a point) of one
field component.  ``update`` forms their values on the host with upstream's
expressions and writes them with one device copy per field and step.
``device_terms`` tabulates the same values for all steps of an ``emsolve``
run at once, as (A(t) * P) * B(t) with the per-step factors A, B evaluated
by the same per-step expressions (same numpy types) and P the profile as
upstream's assignment places it; ``emsolve`` then writes them on the device
(``wk_source_write``) with no per-step host work.
"""

import numpy as np
import torch
from scipy.constants import c as c_light
from scipy.constants import mu_0


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


class PlaneWave:
    """Plane wave moving in +z, imposed on the plane zs over (xs, ys): Hy and
    Ex follow cos(w t + phase) until tmax = nodes / f, then 0
    (upstream sources.py:142-283)."""

    def __init__(self, xs=None, ys=None, zs=0, nodes=None, f=None, amplitude=1.0, beta=1.0,
                 phase=0):
        self.nodes, self.beta = nodes, beta
        self.xs, self.ys, self.zs = xs, ys, zs
        self.f, self.amplitude, self.phase = f, amplitude, phase
        self.is_first_update = True
        self.vp = self.beta * c_light
        self.w = 2 * np.pi * self.f
        self.kz = self.w / c_light
        self.tmax = np.inf if self.nodes is None else self.nodes / self.f

    def _first(self, solver):
        if self.is_first_update:
            self.xs = slice(0, solver.Nx) if self.xs is None else self.xs
            self.ys = slice(0, solver.Ny) if self.ys is None else self.ys
            self.is_first_update = False

    def _values(self, t):
        if t <= self.tmax:
            wave = np.cos(self.w * t + self.phase)
            return -self.amplitude * wave, self.amplitude * wave / (self.kz / (mu_0 * self.vp))
        return 0.0, 0.0

    def update(self, solver, t):
        self._first(solver)
        h, e = self._values(t)
        solver.H[self.xs, self.ys, self.zs, "y"] = h
        solver.E[self.xs, self.ys, self.zs, "x"] = e

    def device_terms(self, solver, n_steps):
        """Hy and Ex of steps 0..n_steps-1 (t = n*dt) as device terms."""
        self._first(solver)
        hv, ev = zip(*(self._values(n * solver.dt) for n in range(n_steps))) if n_steps else ((), ())
        terms = [_term(solver, "H", "y", self.xs, self.ys, self.zs, hv),
                 _term(solver, "E", "x", self.xs, self.ys, self.zs, ev)]
        return None if None in terms else terms


class WavePacket:
    """Gaussian wave packet (transverse sigmaxy, longitudinal sigmaz, delay
    tinj) imposed on the plane zs: Hy and Ex (upstream sources.py:285-456).
    The transverse profile is built on meshgrid(x, y) in upstream's default
    'xy' orientation."""

    def __init__(self, xs=None, ys=None, zs=0, sigmaz=None, sigmaxy=None, tinj=None,
                 wavelength=None, f=None, amplitude=1.0, beta=1.0, phase=0):
        self.beta = beta
        self.xs, self.ys, self.zs = xs, ys, zs
        self.f, self.wavelength = f, wavelength
        self.sigmaxy, self.sigmaz, self.tinj = sigmaxy, sigmaz, tinj
        self.amplitude, self.phase = amplitude, phase
        if self.f is None:
            self.f = c_light / self.wavelength
        self.w = 2 * np.pi * self.f
        if self.tinj is None and self.sigmaz is not None:
            self.tinj = 6 * self.sigmaz
        self.is_first_update = True

    def _first(self, solver):
        if self.is_first_update:
            self.xs = slice(0, solver.Nx) if self.xs is None else self.xs
            self.ys = slice(0, solver.Ny) if self.ys is None else self.ys
            if self.sigmaz is None:
                self.sigmaz = 10 * np.mean(solver.dz)
            if self.sigmaxy is None:
                self.sigmaxy = 5 * np.mean([np.mean(solver.dx), np.mean(solver.dy)])
            if self.tinj is None:
                self.tinj = 6 * self.sigmaz
            self.is_first_update = False

    def _gxy(self, solver):
        X, Y = np.meshgrid(solver.x[self.xs], solver.y[self.ys])
        return np.exp(-(X ** 2 + Y ** 2) / (2 * self.sigmaxy ** 2))

    def _factors(self, solver, t):
        """(-amp wave, amp mu0 c wave, gt) at time t: the value written is
        (factor * gxy) * gt, in upstream's order."""
        s0 = solver.z.min() - self.tinj
        s = solver.z.min() - self.beta * c_light * t
        gt = np.exp(-((s - s0) ** 2) / (2 * self.sigmaz ** 2))
        wave = np.cos(self.w * t + self.phase)
        return -self.amplitude * wave, self.amplitude * mu_0 * c_light * wave, gt

    def update(self, solver, t):
        self._first(solver)
        gxy = self._gxy(solver)
        ah, ae, gt = self._factors(solver, t)
        solver.H[self.xs, self.ys, self.zs, "y"] = ah * gxy * gt
        solver.E[self.xs, self.ys, self.zs, "x"] = ae * gxy * gt

    def device_terms(self, solver, n_steps):
        """Hy and Ex of steps 0..n_steps-1 (t = n*dt) as device terms."""
        self._first(solver)
        gxy = self._gxy(solver)
        f = [self._factors(solver, n * solver.dt) for n in range(n_steps)]
        ah, ae, gt = (zip(*f) if f else ((), (), ()))
        terms = [_term(solver, "H", "y", self.xs, self.ys, self.zs, ah, gt, gxy),
                 _term(solver, "E", "x", self.xs, self.ys, self.zs, ae, gt, gxy)]
        return None if None in terms else terms


def _span(idx, n):
    """[a, b) of an int or a unit-step slice over n entries; None otherwise."""
    if isinstance(idx, (int, np.integer)):
        i = int(idx) + (n if idx < 0 else 0)
        return (i, i + 1) if 0 <= i < n else None
    if isinstance(idx, slice) and idx.step in (None, 1):
        a, b, _ = idx.indices(n)
        return (a, max(a, b))
    return None


_COMPONENTS = {"x": 0, "y": 1, "z": 2, 0: 0, 1: 1, 2: 2}


def _term(solver, field, component, xs, ys, zs, A, B=None, values=None):
    """One device term: field name, component, box, profile P (as upstream's
    assignment of `values` places it in the box, None for a scalar), A, B."""
    comp = _COMPONENTS.get(component)
    box = (_span(xs, solver.Nx), _span(ys, solver.Ny), _span(zs, solver.Nz))
    if comp is None or field not in ("E", "H", "J") or None in box:
        return None
    prof = None
    if values is not None:
        img = np.zeros((solver.Nx, solver.Ny, solver.Nz))
        img[xs, ys, zs] = values
        (i0, i1), (j0, j1), (k0, k1) = box
        prof = img[i0:i1, j0:j1, k0:k1]
    return dict(field=field, component=comp, box=tuple(v for ab in box for v in ab),
                prof=prof, A=np.asarray(A, np.float64),
                B=None if B is None else np.asarray(B, np.float64))


def _field_of(solver, name):
    if name == "E":
        return solver.E
    if name == "H":
        return solver.H
    if name == "J":
        return solver.J
    return None


class Dipole:
    """Sinusoidal point (or slice) source amplitude*sin(w t + phase) on one
    component of E, H or J; f defaults to nodes periods over the z transit
    time of light (upstream sources.py:458-567)."""

    def __init__(self, field="E", component="z", xs=None, ys=None, zs=None, nodes=10, f=None,
                 amplitude=1.0, phase=0):
        self.nodes = nodes
        self.xs, self.ys, self.zs = xs, ys, zs
        self.f, self.field, self.component = f, field, component
        self.amplitude, self.phase = amplitude, phase
        if len(field) == 2:
            self.field, self.component = field[0], field[1]
        self.is_first_update = True

    def _first(self, solver):
        if self.is_first_update:
            self.xs = int(solver.Nx / 2) if self.xs is None else self.xs
            self.ys = int(solver.Ny / 2) if self.ys is None else self.ys
            self.zs = int(solver.Nz / 2) if self.zs is None else self.zs
            if self.f is None:
                self.f = self.nodes / ((solver.z.max() - solver.z.min()) / c_light)
            self.w = 2 * np.pi * self.f
            self.is_first_update = False

    def _value(self, t):
        return self.amplitude * np.sin(self.w * t + self.phase)

    def update(self, solver, t):
        self._first(solver)
        fld = _field_of(solver, self.field)
        if fld is None:
            print(f'Field "{self.field}" not valid, should be "E", "H" or "J"]')
            return
        fld[self.xs, self.ys, self.zs, self.component] = self._value(t)

    def device_terms(self, solver, n_steps):
        """The source component of steps 0..n_steps-1 (t = n*dt) as a device
        term (None when the field or the box is not one the device writes)."""
        self._first(solver)
        if _field_of(solver, self.field) is None:
            return None
        t = _term(solver, self.field, self.component, self.xs, self.ys, self.zs,
                  [self._value(n * solver.dt) for n in range(n_steps)])
        return None if t is None else [t]


class Pulse:
    """Pulse with a 'Harris', 'Gaussian' or 'Rectangular' time profile of
    width L (c*t units, default 50 dt) and delay on one component of E, H or
    J (upstream sources.py:569-762)."""

    def __init__(self, field="E", component="z", xs=None, ys=None, zs=None, shape="Harris",
                 L=None, amplitude=1.0, delay=0.0):
        self.xs, self.ys, self.zs = xs, ys, zs
        self.field, self.component = field, component
        self.shape, self.L, self.amplitude, self.delay = shape, L, amplitude, delay
        if len(field) == 2:
            self.field, self.component = field[0], field[1]
        shapes = {"harris": self.harris_pulse, "gaussian": self.gaussian_pulse,
                  "rectangular": self.rectangular_pulse}
        if shape.lower() in shapes:
            self.tprofile = shapes[shape.lower()]
        else:   # upstream prints and leaves the profile unset
            print('** shape does not, match available types: "Harris", "Gaussian", '
                  '"Rectangular"')
        self.is_first_update = True

    def harris_pulse(self, t):
        t = t * c_light - self.delay
        harris = lambda u: (10 - 15 * np.cos(2 * np.pi / self.L * u)
                            + 6 * np.cos(4 * np.pi / self.L * u)
                            - np.cos(6 * np.pi / self.L * u)) / 32
        if np.ndim(t) == 0:
            return harris(t) if t < self.L else 0.0
        return harris(t)

    def gaussian_pulse(self, t):
        t = t * c_light - self.delay
        return np.exp(-((t - 5 * (self.L / 10)) ** 2) / (2 * (self.L / 10) ** 2))

    def rectangular_pulse(self, t):
        t = t * c_light - self.delay
        return 1.0 if (t < self.L and t > 0.0) else 0.0

    def _first(self, solver):
        if self.is_first_update:
            self.xs = int(solver.Nx / 2) if self.xs is None else self.xs
            self.ys = int(solver.Ny / 2) if self.ys is None else self.ys
            self.zs = int(solver.Nz / 2) if self.zs is None else self.zs
            if self.L is None:
                self.L = 50 * solver.dt
            self.is_first_update = False

    def update(self, solver, t):
        self._first(solver)
        fld = _field_of(solver, self.field)
        if fld is None:
            print(f'Field "{self.field}" not valid, should be "E", "H" or "J"]')
            return
        fld[self.xs, self.ys, self.zs, self.component] = self.amplitude * self.tprofile(t)

    def device_terms(self, solver, n_steps):
        """The source component of steps 0..n_steps-1 (t = n*dt) as a device
        term (None without a time profile, or for a field or box the device
        does not write)."""
        self._first(solver)
        if _field_of(solver, self.field) is None or not hasattr(self, "tprofile"):
            return None
        t = _term(solver, self.field, self.component, self.xs, self.ys, self.zs,
                  [self.amplitude * self.tprofile(n * solver.dt) for n in range(n_steps)])
        return None if t is None else [t]
