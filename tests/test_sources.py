"""Host logic of the device-written sources: ``device_terms`` of PlaneWave,
WavePacket, Dipole and Pulse tabulate, for every step of a run, exactly the
values that ``update(solver, t)`` assigns (upstream wakis/sources.py:142-762),
as (A[n] * P) * B[n] over the source's box.  Checked bit for bit on numpy
stand-ins of the solver fields (no device needed)."""

import numpy as np
import pytest

import cases
from wakis_b200 import sources
from wakis_b200.gridFIT3D import GridFIT3D


class _NumpyField:
    """The (i, j, k, component) assignment of wakis Field on a numpy array."""

    def __init__(self, shape):
        self.a = np.zeros((3,) + shape)

    def __setitem__(self, key, value):
        d = {"x": 0, "y": 1, "z": 2}.get(key[3], key[3])
        self.a[d][key[0], key[1], key[2]] = value


class _Solver:
    def __init__(self, case, dt):
        g = GridFIT3D(*cases.SOURCE_BOUNDS, *case["shape"], verbose=0)
        self.Nx, self.Ny, self.Nz = case["shape"]
        self.x, self.y, self.z = g.x, g.y, g.z
        self.dx, self.dy, self.dz = g.dx, g.dy, g.dz
        self.dt = dt
        self.fresh()

    def fresh(self):
        shape = (self.Nx, self.Ny, self.Nz)
        self.E, self.H, self.J = (_NumpyField(shape) for _ in range(3))


@pytest.mark.parametrize("dt", [np.float64(1.3e-12), np.float32(1.3e-12)])
@pytest.mark.parametrize("idx", range(len(cases.SOURCE_CASES)))
def test_device_terms_equal_update(idx, dt):
    c = cases.SOURCE_CASES[idx]
    s = _Solver(c, dt)
    n_steps = 9
    terms = getattr(sources, c["kind"])(**c["kw"]).device_terms(s, n_steps)
    assert terms, c["kind"]
    src = getattr(sources, c["kind"])(**c["kw"])
    for n in range(n_steps):
        s.fresh()
        src.update(s, n * s.dt)
        written = np.zeros((3, 3, s.Nx, s.Ny, s.Nz), bool)
        for t in terms:
            f = "EHJ".index(t["field"])
            i0, i1, j0, j1, k0, k1 = t["box"]
            v = t["A"][n]
            if t["prof"] is not None:
                v = v * t["prof"]
            if t["B"] is not None:
                v = v * t["B"][n]
            got = getattr(s, t["field"]).a[t["component"]][i0:i1, j0:j1, k0:k1]
            assert np.array_equal(got, np.broadcast_to(v, got.shape)), (c["kind"], n)
            written[f, t["component"], i0:i1, j0:j1, k0:k1] = True
        # update wrote nothing outside the terms' boxes
        for f, name in enumerate("EHJ"):
            assert not np.any(getattr(s, name).a[~written[f]]), (c["kind"], n, name)


def test_unsupported_box_falls_back():
    """A box the device does not write (a strided slice) gives no terms, so
    emsolve keeps update()."""
    c = cases.SOURCE_CASES[2]
    s = _Solver(c, np.float64(1e-12))
    src = sources.Dipole(field="Ez", xs=slice(0, 8, 2), ys=3, zs=4)
    assert src.device_terms(s, 4) is None
