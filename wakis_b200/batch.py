"""Batched wakesolve: many independent cavities (uneven grids, each with its
own dt, beta and materials) stepped together on one GPU.

Upstream runs one ``SolverFIT3D.wakesolve`` per geometry (wakis/routines.py:
231-482); here every instance keeps its own solver, beam and Ez history, and
the stepping of all of them is shared:

* ``launch="batched"`` (FP32-compensated instances, ``wk_batch_run``): one
  device work list of (instance, tile, z-chunk) items and boundary-plane
  items over all instances, run either as ONE persistent cooperative launch
  per chunk of steps (its blocks claim the items of every step in order and
  an item waits, bounded, only for its own instance's earlier work) or as
  one launch per list and step (form "phases").  The step index comes from
  a device counter, so the chunk is captured once in a CUDA graph and
  replayed.  An autotuner times both forms, the tile-shape policies (64x8
  or 32x16 tiles for every instance, or per instance the shape with fewer
  idle lanes) and the candidate planes per work item (the z depth of the
  tiles, ``SolverFIT3D.tile``) on the whole batch and keeps the fastest.
* ``launch="graph"``: one CUDA graph of two steps of every instance (one
  launch per instance and step, spread over a few streams) plus an increment
  of the device step counter (``wk_fit_desc.step_dev``), replayed Nt/2 times;
  the autotuner picks the planes per block of each distinct grid.

Afterwards each ``WakeSolver`` integrates its own history as wakesolve does.
"""

import ctypes
import time

import numpy as np
import torch

from . import _native
from . import geometry

KC_CANDIDATES = (0, 4, 8, 16, 32)
# planes per work item tried by the autotuner of the batched launches
BATCH_KC_CANDIDATES = (16, 32, 48, 64, 96, 128, 192)
# tile-shape policies of the batched launches: every instance on 64x8 or
# 32x16 tiles, or each on the shape whose tiles leave fewer lanes idle
TILE_POLICIES = ("64x8", "fill", "32x16")


def tile_fill(nx, ny, width):
    """Share of the tile lanes that hold a cell when an nx x ny plane is
    covered by width x (512 / width) tiles."""
    h = 512 // width
    return (nx * ny) / (-(-nx // width) * width * (-(-ny // h) * h))


def tile_rows_for(solver, policy):
    """wk_fit_desc.tile_rows of a batched instance under a tile policy:
    8 (64x8 tiles) or 16 (32x16 tiles)."""
    if policy == "64x8":
        return 8
    if policy == "32x16":
        return 16
    if policy == "fill":
        return 16 if tile_fill(solver.Nx, solver.Ny, 32) > tile_fill(solver.Nx, solver.Ny, 64) \
            else 8
    raise ValueError(f"tile policy {policy!r}")


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


FORMS = {"persistent": _native.WK_BATCH_PERSISTENT, "phases": _native.WK_BATCH_PHASES}


class BatchPlan:
    """A prepared batched run over a list of FP32-compensated solvers
    (``wk_batch_prepare``): the workspace (device memory owned here), the
    plan and the descriptors it was built from.  ``descs`` holds one
    ``FitDesc`` per solver (beam, capture and J mode filled in); the live
    buffers of step ``t_ref`` are each descriptor's ``par``.  ``form``:
    "persistent" or "phases" (``wk_batch_plan.form``)."""

    def __init__(self, solvers, descs, t_ref, form="persistent"):
        lib = _native.lib()
        self.solvers = list(solvers)
        n = len(self.solvers)
        arr = (_native.FitDesc * n)()
        for q, d in enumerate(descs):
            ctypes.memmove(ctypes.byref(arr[q]), ctypes.byref(d), ctypes.sizeof(d))
        self.descs = arr
        nbytes = lib.wk_batch_workspace_bytes(arr, n)
        if nbytes < 0:
            raise ValueError("wk_batch_workspace_bytes: " +
                             lib.wk_last_error().decode(errors="replace"))
        dev = self.solvers[0].device
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        self.plan = _native.BatchPlan()
        stream = torch.cuda.current_stream(dev).cuda_stream
        _native.check(lib.wk_batch_prepare(arr, n, int(t_ref), self.workspace.data_ptr(),
                                           int(nbytes), ctypes.byref(self.plan), stream),
                      "wk_batch_prepare")
        self.plan.form = FORMS[form]

    def run(self, n_steps, step0=0, step_dev=None, wait_ns=0, stream=None):
        """Enqueue n_steps steps (step indices step0 + s, plus *step_dev
        when given) on `stream`: one persistent launch, or the launches of
        every list and step."""
        lib = _native.lib()
        if stream is None:
            stream = torch.cuda.current_stream(self.solvers[0].device).cuda_stream
        _native.check(lib.wk_batch_run(ctypes.byref(self.plan), int(n_steps), int(step0),
                                       step_dev, int(wait_ns), stream), "wk_batch_run")


def batched_ok(solvers):
    """True when the batched launches can take these solvers: all
    FP32-compensated, on one device, with x/y faces PEC-masked and the same
    face mode, id width and J mode (checked again by wk_batch_prepare)."""
    if not solvers:
        return False
    s0 = solvers[0]
    for s in solvers:
        if s.precision != "fp32c" or s.device != s0.device or s.Nx % 4:
            return False
        if s._desc.id_bytes > 2 or s.use_conductivity != s0.use_conductivity:
            return False
        pec = list(s._desc.pec_face)
        if s._desc.has_pmc or not s._desc.has_pec or any(pec[:4]):
            return False
        if (pec[4] == 0 and pec[5] == 0) != (list(s0._desc.pec_face)[4:] == [0, 0]):
            return False
    return True


def autotune_batch(solvers, candidates=BATCH_KC_CANDIDATES, forms=tuple(FORMS), steps=4,
                   policies=TILE_POLICIES):
    """Pick the launch form, the tile-shape policy and the planes per work
    item of the batched run by timing `steps` source-free steps of the
    whole batch per candidate with CUDA events; every solver's ``tile`` is
    set to the winner ((8 or 16 tile rows, planes)).  The fields start at
    zero and stay zero (no source); they are reset afterwards.  Returns
    ((form, planes, policy), {(form, planes, policy): ms})."""
    dev = solvers[0].device
    tried = {}
    shapes_seen = set()
    for policy in policies:
        rows = tuple(tile_rows_for(s, policy) for s in solvers)
        if rows in shapes_seen:          # the same shapes as a policy timed before
            continue
        shapes_seen.add(rows)
        for kc in candidates:
            for s, r in zip(solvers, rows):
                s.tile = (r, kc)
                s._first_step()
            descs = [_native.FitDesc.from_buffer_copy(s._step_desc()) for s in solvers]
            for form in forms:
                plan = BatchPlan(solvers, descs, t_ref=0, form=form)
                plan.run(1, 0)                                   # warm
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record()
                plan.run(steps, 1)
                ev1.record()
                torch.cuda.synchronize(dev)
                tried[(form, kc, policy)] = ev0.elapsed_time(ev1)
    best = min(tried, key=tried.get)
    for s in solvers:
        s.tile = (tile_rows_for(s, best[2]), best[1])
        s.reset_fields()
        s.nstep = 0
        s.step_0 = True
        s.check_status("autotune_batch")
    return best, tried


class BatchedWakeSolve:
    """Run ``wakesolve`` for a list of solvers (each built with its own
    WakeSolver), sharing the stepping of all of them.

    n_steps: steps per instance (every instance gets the same count; the
    wakelength of each is set so that upstream's Nt formula gives n_steps).
    launch: "batched" (the device work list over all instances,
    wk_batch_run, for FP32-compensated instances), "graph" (replayed graph of
    per-instance launches) or "auto" (batched when ``batched_ok``).  form:
    the batched launch form, "persistent", "phases" or "auto" (chosen by the
    autotuner; "persistent" without tuning).  tiles: the tile shapes of the
    batched launch, "64x8", "32x16", "fill" (per instance, the shape with
    fewer idle lanes) or "auto" (chosen by the autotuner; "fill" without
    tuning).  streams: number of CUDA streams the instances are spread over
    inside the graph (launch="graph").
    chunk: steps per captured chunk of the batched launch.  tune: run the
    autotuner first.
    """

    def __init__(self, solvers, n_steps, compute_plane="both", streams=8, tune=True,
                 launch="auto", chunk=500, form="auto", tiles="auto"):
        if n_steps < 2:
            raise ValueError("n_steps must be >= 2")
        if launch not in ("auto", "batched", "graph"):
            raise ValueError(f"launch {launch!r}")
        if form not in ("auto",) + tuple(FORMS):
            raise ValueError(f"form {form!r}")
        if tiles not in ("auto",) + TILE_POLICIES:
            raise ValueError(f"tiles {tiles!r}")
        self.tiles = tiles
        self.solvers = list(solvers)
        self.n_steps = int(n_steps)
        self.compute_plane = compute_plane
        self.n_streams = max(1, int(streams))
        self.tune = tune
        self.tuned = {}
        self.timing = {}
        if launch == "auto":
            launch = "batched" if batched_ok(self.solvers) else "graph"
        elif launch == "batched" and not batched_ok(self.solvers):
            raise ValueError("launch='batched' needs FP32-compensated instances with "
                             "PEC-masked x/y faces, sharing face mode, id width and J mode")
        self.launch = launch
        self.form = form
        self.chunk = max(1, int(chunk))

    @staticmethod
    def wakelength_for(solver, n_steps):
        """Wakelength whose upstream step count int(tmax/dt) is n_steps."""
        w = solver.wake
        z = solver.z
        return (n_steps + 0.5) * float(solver.dt) * w.v - w.ti * w.v - (z.max() - z.min())

    def _setup(self):
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
        return states

    def run(self):
        dev = self.solvers[0].device
        if self.launch == "batched":
            form = self.form
            if self.tune:
                forms = tuple(FORMS) if form == "auto" else (form,)
                best, tried = autotune_batch(self.solvers, forms=forms,
                                             policies=TILE_POLICIES if self.tiles == "auto"
                                             else (self.tiles,))
                form = best[0]
                self.tuned = {"form": best[0], "planes_per_item": best[1],
                              "tile_policy": best[2],
                              "tiles_32x16": sum(1 for s in self.solvers if s.tile[0] == 16),
                              "tried_ms": {f"{k[0]}/{k[1]}/{k[2]}": v
                                           for k, v in tried.items()}}
            else:
                for s in self.solvers:
                    s.tile = (tile_rows_for(s, "fill" if self.tiles == "auto" else self.tiles),
                              s.tile[1])
            if form == "auto":
                form = "persistent"
            self.tuned["form"] = form
            states = self._setup()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record()
            for s, ws in zip(self.solvers, states):
                s._advance(1, 0, beam=ws["beam_params"], capture=ws["capture"])
            descs = [_native.FitDesc.from_buffer_copy(
                s._step_desc(ws["beam_params"], ws["capture"])) for s, ws in zip(self.solvers,
                                                                                 states)]
            plan = BatchPlan(self.solvers, descs, t_ref=1, form=form)
            rest = self.n_steps - 1
            chunk = min(self.chunk, rest)
            reps, tail = divmod(rest, chunk)
            counter = torch.ones(1, dtype=torch.int64, device=dev)
            main = torch.cuda.Stream(dev)
            main.wait_stream(torch.cuda.current_stream(dev))
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=main):
                plan.run(chunk, 0, step_dev=counter.data_ptr(), stream=main.cuda_stream)
                _native.check(_native.lib().wk_counter_add(
                    ctypes.c_void_p(counter.data_ptr()), chunk, ctypes.c_void_p(main.cuda_stream)),
                    "wk_counter_add")
            torch.cuda.current_stream(dev).wait_stream(main)
            for _ in range(reps):
                graph.replay()
            torch.cuda.current_stream(dev).wait_stream(main)
            if tail:
                plan.run(tail, 1 + reps * chunk)
            ev1.record()
            torch.cuda.synchronize(dev)
            ms = ev0.elapsed_time(ev1)
            wall = time.perf_counter() - t0
            del graph
            for s in self.solvers:
                s._par ^= rest & 1
                s.nstep += rest
            self.tuned["launches"] = reps + (1 if tail else 0)
            self.tuned["steps_per_launch"] = chunk
        else:
            ms, wall, states = self._run_graph(dev)
        for q, s in enumerate(self.solvers):
            s.check_status(f"BatchedWakeSolve.run (instance {q})")
        cells = sum(s.N for s in self.solvers)
        self.timing = {"ms": ms, "wall_s": wall, "cells": cells, "steps": self.n_steps,
                       "launch": self.launch,
                       "gcell_steps_per_s": cells * self.n_steps / (ms / 1e3) / 1e9}
        for s, ws in zip(self.solvers, states):
            s._wake_finish(ws, wall)
        return self.timing

    def _run_graph(self, dev):
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
        states = self._setup()
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
        return ms, wall, states


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


def pillbox_grid(R, L, cell=1e-3, pipe=0.008, multiple=4):
    """Bounds (x0, x1, y0, y1, z0, z1), cell counts (Nx, Ny, Nz) and a
    function of the grid edges (x, y, z) giving the wall mask of a pillbox:
    a vacuum cylinder of radius R and length L centred at the origin with a
    vacuum beam pipe along z, inside a conducting wall; the transverse size
    is rounded up to a multiple of `multiple` cells (8 lets the compensation
    words of every row arrive by TMA) and the pipe runs max(45 mm, L)
    past each cavity end.  A cell is vacuum when any of its corners is
    inside the vacuum region."""
    nxy = int(np.ceil(2 * (R + 0.005) / cell / multiple)) * multiple
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
                  dtype=np.float64, device=None, multiple=4):
    """(grid, wake, solver) of one pillbox (``pillbox_grid``): wall of
    conductivity sigma (surface impedance above the resolvable conductivity,
    as upstream does), 1 mm cells, PEC on x/y and ABC on z."""
    from .gridFIT3D import GridFIT3D
    from .solverFIT3D import SolverFIT3D
    from .wakeSolver import WakeSolver
    bounds, shape, wall_mask = pillbox_grid(R, L, cell=cell, pipe=pipe, multiple=multiple)
    g = GridFIT3D(*bounds, *shape, verbose=0)
    g.add_solid("wall", wall_mask(g.x, g.y, g.z), [1.0, 1.0, sigma])
    w = WakeSolver(q=1e-9, sigmaz=sigmaz, beta=beta, xsource=0.0, ysource=0.0, xtest=0.0,
                   ytest=0.0, save=False, verbose=0)
    s = SolverFIT3D(g, w, bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"],
                    use_stl=True, use_sibc=True, bg="vacuum", dtype=dtype, verbose=0,
                    precision=precision, device=device)
    return g, w, s
