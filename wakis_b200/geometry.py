"""Solid geometry -> cell masks, without VTK.

Upstream marks the grid *points* enclosed by an STL surface with VTK's
``select_enclosed_points`` and turns the point flags into cell flags by
averaging the 8 corner values and thresholding above a tiny tolerance
(wakis/gridFIT3D.py:470-517): a cell belongs to a solid when any of its 8
corners is inside.  This module applies the same any-corner rule to

* analytic shapes (``Box``, ``CylinderZ``, ``Sphere`` and their unions,
  intersections and differences), and
* triangulated STL surfaces (ASCII or binary), with a point-in-solid test by
  ray parity along +z for each (x, y) column of grid points.

Masks are (Nx, Ny, Nz) boolean arrays indexed [i, j, k].
"""

import struct

import numpy as np


class Shape:
    def contains(self, X, Y, Z):
        raise NotImplementedError

    def __or__(self, other):
        return _Op(self, other, np.logical_or)

    def __and__(self, other):
        return _Op(self, other, np.logical_and)

    def __sub__(self, other):
        return _Op(self, other, lambda a, b: a & ~b)


class _Op(Shape):
    def __init__(self, a, b, op):
        self.a, self.b, self.op = a, b, op

    def contains(self, X, Y, Z):
        return self.op(self.a.contains(X, Y, Z), self.b.contains(X, Y, Z))


class Box(Shape):
    """Closed box [xmin, xmax] x [ymin, ymax] x [zmin, zmax]."""

    def __init__(self, xmin, xmax, ymin, ymax, zmin, zmax, tol=0.0):
        self.b = (xmin, xmax, ymin, ymax, zmin, zmax)
        self.tol = tol

    def contains(self, X, Y, Z):
        x0, x1, y0, y1, z0, z1 = self.b
        t = self.tol
        return ((X >= x0 - t) & (X <= x1 + t) & (Y >= y0 - t) & (Y <= y1 + t)
                & (Z >= z0 - t) & (Z <= z1 + t))


class CylinderZ(Shape):
    """Cylinder of radius r along z through (x0, y0), open radius test
    (points on the mantle are outside), z in [zmin, zmax]."""

    def __init__(self, r, x0=0.0, y0=0.0, zmin=-np.inf, zmax=np.inf):
        self.r, self.x0, self.y0, self.zmin, self.zmax = r, x0, y0, zmin, zmax

    def contains(self, X, Y, Z):
        return (((X - self.x0) ** 2 + (Y - self.y0) ** 2 < self.r ** 2)
                & (Z >= self.zmin) & (Z <= self.zmax))


class Sphere(Shape):
    def __init__(self, r, x0=0.0, y0=0.0, z0=0.0):
        self.r, self.c = r, (x0, y0, z0)

    def contains(self, X, Y, Z):
        x0, y0, z0 = self.c
        return (X - x0) ** 2 + (Y - y0) ** 2 + (Z - z0) ** 2 < self.r ** 2


class Points(Shape):
    """Explicit inside flags of the grid points, shape (Nx+1, Ny+1, Nz+1)."""

    def __init__(self, flags):
        self.flags = np.asarray(flags, bool)

    def contains(self, X, Y, Z):
        return self.flags


# ------------------------------------------------------------------ STL ----
def read_stl(path):
    """Triangles of an ASCII or binary STL file as a (T, 3, 3) float64 array."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) >= 84:
        ntri = struct.unpack("<I", data[80:84])[0]
        if 84 + 50 * ntri == len(data):
            rec = np.frombuffer(data[84:], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)),
                                                           ("a", "<u2")]))
            return rec["v"].astype(np.float64)
    verts = [list(map(float, line.split()[1:4])) for line in data.decode(errors="replace")
             .splitlines() if line.strip().startswith("vertex")]
    return np.asarray(verts, dtype=np.float64).reshape(-1, 3, 3)


def _rot(axis, deg):
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    if axis == 0:
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == 1:
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


class STLSolid(Shape):
    """Closed triangulated surface.  Transform order as upstream read_stl
    (wakis/gridFIT3D.py:537-565): rotate x, y, z (degrees), translate, scale."""

    def __init__(self, path, rotate=(0.0, 0.0, 0.0), translate=(0.0, 0.0, 0.0), scale=1.0):
        tri = read_stl(path)
        v = tri.reshape(-1, 3)
        for ax in range(3):
            if rotate[ax]:
                v = v @ _rot(ax, rotate[ax]).T
        v = v + np.asarray(translate, dtype=np.float64)
        v = v * scale
        self.tri = v.reshape(-1, 3, 3)

    def contains(self, X, Y, Z):
        """Ray parity along +z on the grid's point columns (X, Y, Z from
        meshgrid(x, y, z, indexing='ij'))."""
        x = X[:, 0, 0]
        y = Y[0, :, 0]
        z = Z[0, 0, :]
        inside = np.zeros((len(x), len(y), len(z)), bool)
        # small deterministic offsets avoid rays through edges/vertices
        ex = 1e-9 * (np.ptp(x) + 1.0) * np.pi
        ey = 1e-9 * (np.ptp(y) + 1.0) * np.e
        xs = x + ex
        ys = y + ey
        t = self.tri
        p0, p1, p2 = t[:, 0], t[:, 1], t[:, 2]
        for ii, px in enumerate(xs):
            m = (np.minimum(np.minimum(p0[:, 0], p1[:, 0]), p2[:, 0]) <= px) & \
                (np.maximum(np.maximum(p0[:, 0], p1[:, 0]), p2[:, 0]) >= px)
            if not m.any():
                continue
            a, b, c = p0[m], p1[m], p2[m]
            for jj, py in enumerate(ys):
                # barycentric test of (px, py) in the triangle projection
                d = (b[:, 1] - c[:, 1]) * (a[:, 0] - c[:, 0]) + (c[:, 0] - b[:, 0]) * (a[:, 1] - c[:, 1])
                ok = np.abs(d) > 0
                if not ok.any():
                    continue
                l1 = ((b[:, 1] - c[:, 1]) * (px - c[:, 0]) + (c[:, 0] - b[:, 0]) * (py - c[:, 1]))
                l2 = ((c[:, 1] - a[:, 1]) * (px - c[:, 0]) + (a[:, 0] - c[:, 0]) * (py - c[:, 1]))
                with np.errstate(divide="ignore", invalid="ignore"):
                    l1 = np.where(ok, l1 / d, -1)
                    l2 = np.where(ok, l2 / d, -1)
                l3 = 1 - l1 - l2
                hit = (l1 >= 0) & (l2 >= 0) & (l3 >= 0)
                if not hit.any():
                    continue
                zc = np.sort(l1[hit] * a[hit, 2] + l2[hit] * b[hit, 2] + l3[hit] * c[hit, 2])
                # parity: number of crossings below each point
                cnt = np.searchsorted(zc, z, side="right")
                inside[ii, jj, :] = (cnt % 2) == 1
        return inside


# ------------------------------------------------------------ cell masks ---
def cell_mask(shape, x, y, z, chunk=64):
    """(Nx, Ny, Nz) mask: a cell is inside when any of its 8 corners is.
    Corner tests run in slabs of `chunk` cell planes along z, so large grids
    need no full-size coordinate arrays."""
    x, y, z = (np.asarray(v, float) for v in (x, y, z))
    nx, ny, nz = len(x) - 1, len(y) - 1, len(z) - 1
    m = np.zeros((nx, ny, nz), bool)
    for k0 in range(0, nz, chunk):
        k1 = min(nz, k0 + chunk)
        X, Y, Z = np.meshgrid(x, y, z[k0:k1 + 1], indexing="ij")
        inside = np.asarray(shape.contains(X, Y, Z), bool)
        n = k1 - k0
        for a in (0, 1):
            for b in (0, 1):
                for c in (0, 1):
                    m[:, :, k0:k1] |= inside[a:a + nx, b:b + ny, c:c + n]
    return m


def surface_mask(mask):
    """Cells on either side of the solid's boundary: cells whose value
    differs from at least one face neighbour.  Stand-in for the non-zero
    cell gradient upstream takes from VTK (wakis/gridFIT3D.py:519-535)."""
    m = np.asarray(mask, bool)
    out = np.zeros_like(m)
    for ax in range(3):
        d = np.diff(m.astype(np.int8), axis=ax) != 0
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[ax] = slice(0, -1)
        sl_hi[ax] = slice(1, None)
        out[tuple(sl_lo)] |= d
        out[tuple(sl_hi)] |= d
    return out
