"""Batched wakesolve: many independent cavities (uneven grids, each with its
own dt, beta and materials) stepped together on one GPU.

Upstream runs one ``SolverFIT3D.wakesolve`` per geometry (wakis/routines.py:
231-482); here every instance keeps its own solver, beam and Ez history, and
the stepping of all of them is one CUDA graph: two steps of every instance,
spread over a few streams, then an increment of a device step counter that
the kernels read (``wk_fit_desc.step_dev``).  The graph is captured once and
replayed Nt/2 times, so the host issues one launch per two steps of the whole
batch instead of ~3 launches per step per instance.  Before the run a small
autotuner times the candidate chunk lengths (planes per block of the TMA
kernels, ``SolverFIT3D.tile``) on each distinct grid and keeps the fastest.
Afterwards each ``WakeSolver`` integrates its own history as wakesolve does.
"""

import ctypes
import time

import numpy as np
import torch

from . import _native
from . import geometry

KC_CANDIDATES = (0, 4, 8, 16, 32)


def autotune(solver, candidates=KC_CANDIDATES, steps=4):
    """Pick ``solver.tile`` planes-per-block by timing `steps` source-free
    steps per candidate with CUDA events (wk_fit_step_timed).  The fields
    start at zero and stay zero (no source), and are reset afterwards."""
    best, best_ms = None, None
    tried = {}
    for kc in candidates:
        if kc and kc > solver.Nz - 4:
            continue
        solver.tile = (0, kc)
        timing = []
        solver._advance(1, 0, timing=timing)          # warm (first-step work)
        timing = []
        solver._advance(steps, 1, timing=timing)
        ms = sum(t[0] for t in timing)
        tried[kc] = ms
        if best_ms is None or ms < best_ms:
            best, best_ms = kc, ms
    solver.tile = (0, best if best is not None else 0)
    solver.reset_fields()
    solver.nstep = 0
    solver.step_0 = True
    return solver.tile[1], tried


class BatchedWakeSolve:
    """Run ``wakesolve`` for a list of solvers (each built with its own
    WakeSolver) in one captured CUDA graph per pair of steps.

    n_steps: steps per instance (every instance gets the same count; the
    wakelength of each is set so that upstream's Nt formula gives n_steps).
    streams: number of CUDA streams the instances are spread over inside the
    graph.  tune: run the chunk-length autotuner first.
    """

    def __init__(self, solvers, n_steps, compute_plane="both", streams=8, tune=True):
        if n_steps < 2:
            raise ValueError("n_steps must be >= 2")
        self.solvers = list(solvers)
        self.n_steps = int(n_steps)
        self.compute_plane = compute_plane
        self.n_streams = max(1, int(streams))
        self.tune = tune
        self.tuned = {}
        self.timing = {}

    @staticmethod
    def wakelength_for(solver, n_steps):
        """Wakelength whose upstream step count int(tmax/dt) is n_steps."""
        w = solver.wake
        z = solver.z
        return (n_steps + 0.5) * float(solver.dt) * w.v - w.ti * w.v - (z.max() - z.min())

    def run(self):
        dev = self.solvers[0].device
        lib = _native.lib()
        if self.tune:
            shapes = {}
            for s in self.solvers:
                key = (s.Nx, s.Ny, s.Nz, s.precision)
                if key not in shapes:
                    shapes[key] = autotune(s)
                else:
                    s.tile = (0, shapes[key][0])
            self.tuned = {str(k): v[0] for k, v in shapes.items()}
        states = []
        for s in self.solvers:
            wl = self.wakelength_for(s, self.n_steps)
            ws = s._wake_setup(wl, compute_plane=self.compute_plane)
            if ws["Nt"] != self.n_steps:
                raise RuntimeError(f"step count {ws['Nt']} != {self.n_steps}")
            if wl <= -s.wake.ti * s.wake.v:
                raise ValueError(f"{self.n_steps} steps do not reach past the domain "
                                 f"(wakelength {wl:.4g} m): no wake samples")
            states.append(ws)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        # first step eagerly (ghost zeroing, J = 0 for the first step of a
        # conductive instance, kernel caches)
        for s, ws in zip(self.solvers, states):
            s._advance(1, 0, beam=ws["beam_params"], capture=ws["capture"])
        counter = torch.ones(1, dtype=torch.int64, device=dev)
        descs = []
        for s, ws in zip(self.solvers, states):
            d = s._step_desc(ws["beam_params"], ws["capture"])
            copy = _native.FitDesc.from_buffer_copy(d)
            copy.step_dev = counter.data_ptr()
            descs.append(copy)
        main = torch.cuda.Stream(dev)
        side = [torch.cuda.Stream(dev) for _ in range(self.n_streams)]
        graph = torch.cuda.CUDAGraph()
        pairs = (self.n_steps - 1) // 2
        main.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.graph(graph, stream=main):
            for st in side:
                st.wait_stream(main)
            for q, (s, d) in enumerate(zip(self.solvers, descs)):
                st = side[q % self.n_streams]
                with torch.cuda.stream(st):
                    _native.check(lib.wk_fit_step(d, 2, 0, ctypes.c_void_p(st.cuda_stream)),
                                  "wk_fit_step")
            for st in side:
                main.wait_stream(st)
            _native.check(lib.wk_counter_add(ctypes.c_void_p(counter.data_ptr()), 2,
                                             ctypes.c_void_p(main.cuda_stream)),
                          "wk_counter_add")
        torch.cuda.current_stream(dev).wait_stream(main)
        # capture did not run anything: replay `pairs` times, then one last
        # single step when n_steps - 1 is odd
        for _ in range(pairs):
            graph.replay()
        torch.cuda.current_stream(dev).wait_stream(main)
        last = 1 + 2 * pairs
        for s, ws in zip(self.solvers, states):
            s.nstep += 2 * pairs
            if last < self.n_steps:
                s._advance(1, last, beam=ws["beam_params"], capture=ws["capture"])
        ev1.record()
        torch.cuda.synchronize(dev)
        ms = ev0.elapsed_time(ev1)
        wall = time.perf_counter() - t0
        del graph
        for q, s in enumerate(self.solvers):
            s.check_status(f"BatchedWakeSolve.run (instance {q})")
        cells = sum(s.N for s in self.solvers)
        self.timing = {"ms": ms, "wall_s": wall, "cells": cells, "steps": self.n_steps,
                       "gcell_steps_per_s": cells * self.n_steps / (ms / 1e3) / 1e9}
        for s, ws in zip(self.solvers, states):
            s._wake_finish(ws, wall)
        return self.timing


# ----------------------------------------------------------- pillboxes ----
def pillbox_params(n=64, seed=0):
    """Random pillbox cavities: radius U[20, 60] mm, length U[30, 100] mm,
    beta U[0.5, 1], wall conductivity log-uniform on [1e3, 1e6] S/m."""
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.020, 0.060, n)
    L = rng.uniform(0.030, 0.100, n)
    beta = rng.uniform(0.5, 1.0, n)
    sigma = 10.0 ** rng.uniform(3.0, 6.0, n)
    return [dict(R=float(R[q]), L=float(L[q]), beta=float(beta[q]), sigma=float(sigma[q]))
            for q in range(n)]


def pillbox_grid(R, L, cell=1e-3, pipe=0.008):
    """Bounds (x0, x1, y0, y1, z0, z1), cell counts (Nx, Ny, Nz) and a
    function of the grid edges (x, y, z) giving the wall mask of a pillbox:
    a vacuum cylinder of radius R and length L centred at the origin with a
    vacuum beam pipe along z, inside a conducting wall; the transverse size
    is rounded up to a multiple of 4 cells and the pipe runs max(45 mm, L)
    past each cavity end.  A cell is vacuum when any of its corners is
    inside the vacuum region."""
    nxy = int(np.ceil(2 * (R + 0.005) / cell / 4.0)) * 4
    half = nxy * cell / 2
    zl = L / 2 + max(0.045, L)
    nz = int(round(2 * zl / cell))
    vac = geometry.CylinderZ(R, zmin=-L / 2, zmax=L / 2) | geometry.CylinderZ(pipe)
    wall = geometry.Box(-2 * half, 2 * half, -2 * half, 2 * half, -2 * zl, 2 * zl) - vac

    def mask(x, y, z):
        m = geometry.cell_mask(wall, x, y, z)
        m &= ~geometry.cell_mask(vac, x, y, z)
        return m

    return (-half, half, -half, half, -zl, zl), (nxy, nxy, nz), mask


def build_pillbox(R, L, beta, sigma, cell=1e-3, pipe=0.008, sigmaz=0.008, precision=None,
                  dtype=np.float64, device=None):
    """(grid, wake, solver) of one pillbox (``pillbox_grid``): wall of
    conductivity sigma (surface impedance above the resolvable conductivity,
    as upstream does), 1 mm cells, PEC on x/y and ABC on z."""
    from .gridFIT3D import GridFIT3D
    from .solverFIT3D import SolverFIT3D
    from .wakeSolver import WakeSolver
    bounds, shape, wall_mask = pillbox_grid(R, L, cell=cell, pipe=pipe)
    g = GridFIT3D(*bounds, *shape, verbose=0)
    g.add_solid("wall", wall_mask(g.x, g.y, g.z), [1.0, 1.0, sigma])
    w = WakeSolver(q=1e-9, sigmaz=sigmaz, beta=beta, xsource=0.0, ysource=0.0, xtest=0.0,
                   ytest=0.0, save=False, verbose=0)
    s = SolverFIT3D(g, w, bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"],
                    use_stl=True, use_sibc=True, bg="vacuum", dtype=dtype, verbose=0,
                    precision=precision, device=device)
    return g, w, s
