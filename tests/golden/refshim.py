"""Load the upstream Wakis package (pure Python) in a container that lacks
h5py, pyvista and matplotlib, so that its own solver can produce golden
fixtures.

This module is fixture-generation tooling only: it is imported by
``tests/golden/make_golden.py`` on the machine that holds the upstream source
tree, never by the test suite, the benchmark or the package.

Stand-ins installed in ``sys.modules``:

* ``h5py``: an in-memory ``File`` keyed by file name.  Datasets written with
  ``hf[key] = array`` are kept as numpy copies, so ``wakesolve`` (upstream
  ``wakis/routines.py:400-440``) and ``WakeSolver.read_Ez``
  (``wakis/wakeSolver.py:1313-1357``) exchange the Ez history through it.
* ``pyvista``: ``StructuredGrid`` is a dict of cell arrays (the solver reads
  ``grid.grid[key]``, ``wakis/solverFIT3D.py:440``); geometry masks are
  injected directly instead of VTK's ``select_enclosed_points``.
* ``matplotlib`` / ``matplotlib.pyplot``: empty modules (plots are not run).
"""

import importlib
import os
import sys
import types

import numpy as np

UPSTREAM = os.environ.get("WAKIS_UPSTREAM")

_H5_STORE = {}


class _H5File:
    def __init__(self, name, mode="r"):
        self.name = name
        if mode == "w" or name not in _H5_STORE:
            _H5_STORE[name] = {}
            # upstream reads the file size for a log line (wakeSolver.py:1337)
            d = os.path.dirname(name)
            if d:
                os.makedirs(d, exist_ok=True)
            open(name, "wb").close()
        self._d = _H5_STORE[name]

    def __setitem__(self, key, value):
        self._d[key] = np.array(value, copy=True)

    def __getitem__(self, key):
        return self._d[key]

    def keys(self):
        return list(self._d.keys())

    def __contains__(self, key):
        return key in self._d

    def create_dataset(self, key, data=None):
        self[key] = data

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class _StructuredGrid(dict):
    def __init__(self, *args, **kwargs):
        super().__init__()


def install():
    """Install the stand-ins and import upstream ``wakis`` from UPSTREAM
    (the environment variable WAKIS_UPSTREAM: the root of the upstream
    source tree, the directory that holds the ``wakis`` package)."""
    if not UPSTREAM or not os.path.isdir(os.path.join(UPSTREAM, "wakis")):
        raise RuntimeError("set WAKIS_UPSTREAM to the root of the upstream Wakis source tree "
                           f"(got {UPSTREAM!r})")
    if "wakis" in sys.modules and getattr(sys.modules["wakis"], "_refshim", False):
        return sys.modules["wakis"]
    h5 = types.ModuleType("h5py")
    h5.File = _H5File
    sys.modules["h5py"] = h5

    pv = types.ModuleType("pyvista")
    pv.StructuredGrid = _StructuredGrid
    pv.read = None
    sys.modules["pyvista"] = pv

    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt

    if UPSTREAM not in sys.path:
        sys.path.insert(0, UPSTREAM)
    wakis = importlib.import_module("wakis")
    wakis._refshim = True
    return wakis


def inject_solids(grid, masks, materials):
    """Attach geometry masks to an upstream GridFIT3D built without STL.

    ``masks[key]`` is a boolean array of shape (Nx, Ny, Nz); upstream reshapes
    ``grid.grid[key]`` in C order (``wakis/solverFIT3D.py:440``), so the mask
    is flattened in C order here.
    """
    import wakis

    grid.stl_solids = {k: k for k in masks}
    mats = {}
    for key, mat in materials.items():
        if isinstance(mat, str):
            lib = wakis.materials.material_lib[mat.lower()]
            mat = [lib[0], lib[1]] + ([lib[2]] if len(lib) == 3 else [])
        mats[key] = list(mat)
    grid.stl_materials = mats
    grid.stl_colors = {k: "white" for k in masks}
    for key, m in masks.items():
        grid.grid[key] = np.asarray(m, dtype=bool).ravel(order="C")
    return grid
