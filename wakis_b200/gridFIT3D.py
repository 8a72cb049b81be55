"""``GridFIT3D``: Cartesian grid, metrics and solid masks.

Mirrors the upstream constructor (wakis/gridFIT3D.py:32-256) for uniform
grids from extents or explicit x, y, z axes.  ``stl_solids`` values may be
STL file paths (voxelised without VTK by ``geometry.STLSolid``), analytic
``geometry.Shape`` objects, or precomputed boolean (Nx, Ny, Nz) cell masks.
The masks end up in ``grid.grid[key]`` flattened in C order, the layout
upstream's solver reshapes (wakis/solverFIT3D.py:440).

The metrics are kept separable: 1-D edge lengths per axis, and the solver
builds the 2-D inverse-area tables the kernels read, with values identical
to upstream's per-cell ``L, iA, tL, itA`` fields (gridFIT3D.py:258-300).
"""

import time

import numpy as np

from . import geometry
from .logger import Logger
from .materials import material_lib


class GridFIT3D:
    def __init__(self, xmin=None, xmax=None, ymin=None, ymax=None, zmin=None, zmax=None,
                 Nx=None, Ny=None, Nz=None, x=None, y=None, z=None, use_mpi=False,
                 stl_solids=None, stl_materials=None, stl_rotate=(0.0, 0.0, 0.0),
                 stl_translate=(0.0, 0.0, 0.0), stl_scale=1.0, stl_colors=None,
                 stl_tol=1e-3, verbose=1, **unused):
        t0 = time.time()
        self.logger = Logger()
        self.verbose = verbose
        if use_mpi:
            raise ValueError("use_mpi: multi-process runs use wakis_b200.slab, not the grid flag")
        self.use_mpi = False
        if x is not None and y is not None and z is not None:
            self.x, self.y, self.z = (np.asarray(a, dtype=np.float64) for a in (x, y, z))
            self.Nx, self.Ny, self.Nz = len(self.x) - 1, len(self.y) - 1, len(self.z) - 1
        elif all(v is not None for v in (xmin, xmax, ymin, ymax, zmin, zmax)):
            self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
            self.x = np.linspace(xmin, xmax, self.Nx + 1)
            self.y = np.linspace(ymin, ymax, self.Ny + 1)
            self.z = np.linspace(zmin, zmax, self.Nz + 1)
        else:
            raise ValueError(
                "[!] Error initializing GridFIT3D:\n"
                "  - Provide grid axis arrays: x, y, z\n"
                "  - OR domain extents and number of cells: "
                "xmin, xmax, ymin, ymax, zmin, zmax, Nx, Ny, Nz")
        self.xmin, self.xmax = self.x[0], self.x[-1]
        self.ymin, self.ymax = self.y[0], self.y[-1]
        self.zmin, self.zmax = self.z[0], self.z[-1]
        self.dx, self.dy, self.dz = np.diff(self.x), np.diff(self.y), np.diff(self.z)
        self.N = self.Nx * self.Ny * self.Nz
        self._axes_metrics()

        self.stl_tol = stl_tol
        self.stl_solids = {}
        self.stl_materials = {}
        self.stl_colors = {}
        self.grid = {}
        if stl_solids is not None:
            if not isinstance(stl_solids, dict):
                stl_solids = {"Solid 1": stl_solids}
            if not isinstance(stl_materials, dict):
                stl_materials = {k: stl_materials for k in stl_solids}
            for key, sol in stl_solids.items():
                rot = stl_rotate[key] if isinstance(stl_rotate, dict) else stl_rotate
                tr = stl_translate[key] if isinstance(stl_translate, dict) else stl_translate
                sc = stl_scale[key] if isinstance(stl_scale, dict) else stl_scale
                self.add_solid(key, sol, stl_materials[key], rotate=rot, translate=tr, scale=sc)
        self.gridInitializationTime = time.time() - t0
        self.logger.grid.update(dict(Nx=self.Nx, Ny=self.Ny, Nz=self.Nz, xmin=self.xmin,
                                     xmax=self.xmax, ymin=self.ymin, ymax=self.ymax,
                                     zmin=self.zmin, zmax=self.zmax))

    def _axes_metrics(self):
        """1-D primal lengths (x[i+1]-x[i]) and dual lengths of the axes; the
        dual axis repeats its last point, so the last dual length is 0
        (gridFIT3D.py:278-291)."""
        def dual(a):
            t = np.append((a[1:] + a[:-1]) / 2, 0.0)
            t[-1] = t[-2]
            return t[1:] - t[:-1]

        self.tdx, self.tdy, self.tdz = dual(self.x), dual(self.y), dual(self.z)

    def add_solid(self, key, solid, material, rotate=(0.0, 0.0, 0.0),
                  translate=(0.0, 0.0, 0.0), scale=1.0):
        """Register a solid: STL path, ``geometry.Shape`` or (Nx,Ny,Nz) mask."""
        if isinstance(solid, str):
            shape = geometry.STLSolid(solid, rotate=rotate, translate=translate, scale=scale)
            mask = geometry.cell_mask(shape, self.x, self.y, self.z)
        elif isinstance(solid, geometry.Shape):
            mask = geometry.cell_mask(solid, self.x, self.y, self.z)
        else:
            mask = np.asarray(solid, dtype=bool)
            if mask.shape != (self.Nx, self.Ny, self.Nz):
                raise ValueError(f"mask for {key} has shape {mask.shape}")
        if isinstance(material, str):
            lib = material_lib[material.lower()]
            material = [lib[0], lib[1]] + ([lib[2]] if len(lib) == 3 else [])
        self.stl_solids[key] = solid if isinstance(solid, str) else key
        self.stl_materials[key] = list(material)
        self.stl_colors[key] = "white"
        self.grid[key] = mask.ravel(order="C")

    def mask(self, key):
        """(Nx, Ny, Nz) boolean mask of a solid."""
        return np.reshape(self.grid[key], (self.Nx, self.Ny, self.Nz))

    def _mark_cells_in_surface(self, key):
        """Replace a solid's mask by its surface cells (SIBC, upstream
        gridFIT3D.py:519-535; see geometry.surface_mask)."""
        self.grid[key] = geometry.surface_mask(self.mask(key)).ravel(order="C")
