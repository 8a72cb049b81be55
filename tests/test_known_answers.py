"""Known answers of upstream's own tests for the stepper, on the device.

* upstream tests/test_002_analytic_resonator.py: a 1 m cubic PEC cavity of
  30^3 cells started from the analytic (m, n, p) = (1, 0, 1) mode (H at
  t = -dt/2); the Ey probe at the centre, 5000 steps, peaks at the mode
  frequency 2.121e8 Hz within 5 %.
* upstream tests/test_005_pml_boundaries.py: a plane wave of amplitude 100
  launched from z = 0 into a 30-cell PML (20x20x200 cells, periodic x/y, PEC
  below, float32, dt = 1/(200 f)); after the wave has had time to cross the
  domain and come back, |H| and |E|/(mu_0 c) on the centre line stay below
  10 (10 % reflection) for vacuum, a lossy dielectric and a resistive
  background.
"""

import numpy as np
import pytest
from scipy.constants import c as C_LIGHT
from scipy.constants import mu_0

pytestmark = pytest.mark.gpu


def _mode_101_H(x, y, z, t, L):
    """H of the cubic cavity mode m = 1, n = 0, p = 1 (analytic; edge length
    L, origin at the centre), at cell positions x, y, z and time t."""
    m, n, p = 1, 0, 1
    kx, ky, kz = m * np.pi / L, n * np.pi / L, p * np.pi / L
    h2 = kx ** 2 + ky ** 2 + kz ** 2
    w = np.sqrt(2) * np.pi / L * C_LIGHT
    cx, sx = np.cos(kx * (x - L / 2)), np.sin(kx * (x - L / 2))
    cy, sy = np.cos(ky * (y - L / 2)), np.sin(ky * (y - L / 2))
    cz, sz = np.cos(kz * (z - L / 2)), np.sin(kz * (z - L / 2))
    ct = np.cos(w * t)
    hz = cx * cy * sz * ct
    hy = -2 / h2 * ky * kz * cx * sy * cz * ct
    hx = -2 / h2 * kx * kz * sx * cy * cz * ct
    return hx, hy, hz


def test_cubic_resonator_mode_101_frequency():
    import wakis_b200 as wb
    L, N = 1.0, 30
    d = L / N
    lo, hi = -L / 2 + d / 2, L / 2 + d / 2
    g = wb.GridFIT3D(lo, hi, lo, hi, lo, hi, N, N, N, verbose=0)
    s = wb.SolverFIT3D(g, bc_low=["pec"] * 3, bc_high=["pec"] * 3, verbose=0)
    # the cell positions the upstream test evaluates the mode at
    q = np.arange(N) * d + lo
    X, Y, Z = np.meshgrid(q, q, q, indexing="ij")
    hx, hy, hz = _mode_101_H(X, Y, Z, -0.5 * s.dt, L)
    s.H.fromarray(np.concatenate([a.ravel(order="F") for a in (hx, hy, hz)]))
    probe = []
    for _ in range(5000):
        probe.append(s.E[N // 2, N // 2, N // 2, "y"])
        s.one_step()
    probe = np.array(probe, dtype=np.float64)
    spec = np.fft.fftshift(np.fft.fft(probe))[len(probe) // 2:]
    freqs = np.fft.fftshift(np.fft.fftfreq(len(probe), d=s.dt))[len(probe) // 2:]
    f_peak = freqs[np.argmax(spec)]
    assert f_peak == pytest.approx(2.121e8, rel=0.05)


@pytest.mark.parametrize("eps_r,sigma", [(1.0, 0.0), (3.0, 1.0e-3), (1.0, 1.0)])
def test_pml_reflection_of_a_plane_wave(eps_r, sigma):
    import wakis_b200 as wb
    Nx, Ny, Nz = 20, 20, 200
    g = wb.GridFIT3D(-1.0, 1.0, -1.0, 1.0, 0.0, 1.0, Nx, Ny, Nz, verbose=0)
    s = wb.SolverFIT3D(g, use_stl=False, bg=[eps_r, 1.0, sigma],
                       bc_low=["periodic", "periodic", "pec"],
                       bc_high=["periodic", "periodic", "pml"], n_pml=30, dtype=np.float32,
                       verbose=0)
    amplitude = 100.0
    f = 15 / ((s.z.max() - s.z.min()) / C_LIGHT)
    wave = wb.sources.PlaneWave(xs=slice(0, Nx), ys=slice(0, Ny), zs=0, beta=1.0,
                                amplitude=amplitude, f=f, nodes=7, phase=np.pi / 2)
    s.dt = 1 / f / 200
    z_pml = sum(s.dz[Nz - 1 - k] for k in range(s.n_pml))
    Nt = int(eps_r * 2.0 * (1.0 - z_pml) / C_LIGHT / s.dt)
    for n in range(Nt):
        wave.update(s, n * s.dt)
        s.one_step()
    assert int(s._status.item()) == 0
    refl_H = s.H.get_abs()[Nx // 2, Ny // 2, :].max()
    refl_E = s.E.get_abs()[Nx // 2, Ny // 2, :].max() / (mu_0 * C_LIGHT)
    assert np.isfinite(refl_H) and np.isfinite(refl_E)
    assert refl_H <= 10, refl_H
    assert refl_E <= 10, refl_E
