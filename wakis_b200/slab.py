"""z-slab decomposition of the FIT step: one slab per GPU (one process per
GPU, ``torch.distributed`` carrying the plane exchange) or several slabs in
one process.

Upstream splits the grid into z-slabs, one per MPI rank (wakis/gridFIT3D.py:
320-356), and between the two half-steps of every step sends the boundary
plane of H to the +z neighbour and of E to the -z neighbour
(wakis/solverFIT3D.py:539-621).  Here each slab runs the fused single-GPU
step on its own planes plus ghost planes, and ONE exchange per step
refreshes the ghosts:

* a slab owning the planes [k0, k1) holds [lo, hi) = [max(k0-G-1, 0),
  min(k1+G+1, Nz)) for an exchange every G steps (the ghost depth, 1 by
  default); planes k0-G .. k0-1 and k1 .. k1+G-1 are ghosts carrying the
  neighbours' values, planes k0-G-1 and k1+G are padding whose values are
  never used.  A step spreads what a plane depends on by one plane each
  way, so G ghost planes carry the owned planes through G steps, and the
  slab runs G steps per call (G >= 4 lets the solver's steps_per_launch = 2
  run them in pairs per launch of the temporal-blocking kernel); larger G
  means fewer, larger messages and G + 1 extra planes computed per side;
* the step forms H of ghost plane k0-1 from E(k0-1) and E(k0), both
  current, so E(k0) reads the right new H(k0-1) without a mid-step
  exchange; H(k1-1) reads E(k1) from the upper ghost;
* the padding keeps the slab's own z faces away from the planes whose
  values matter: the face masks are applied face by face with the last face
  winning (a z face overrides the x/y masks of its plane), so whatever an
  internal z face masks touches only the padding plane.  Internal faces
  carry the PEC column mask (no PMC), so that a slab of a grid whose x/y
  faces are PEC-like runs the single-launch full-domain TMA kernel; the
  summation order of the H rows stays the global one.

After every G steps the ghost planes receive the neighbours' new E and H
(and, with precision="fp32c", their compensation words), so the fields
equal the single-domain run value for value.  The material ids and the z-dependent
metric tables are slices of the global compact coefficient set, built once
on the host; the time step is the global one.

The Ez history of the test line is captured by every slab on its own planes
and joined along z before the wake integration, which runs where the
history is joined (rank 0 with torch.distributed).
"""

import time
from dataclasses import dataclass, replace
from types import SimpleNamespace

import numpy as np
import torch

from .coefficients import build as build_coefficients
from .sources import Beam


def partition(Nz, n):
    """Owned plane ranges [k0, k1) of n slabs, as even as possible."""
    if n < 1 or n > Nz:
        raise ValueError(f"cannot split {Nz} planes into {n} slabs")
    base, extra = divmod(Nz, n)
    out, k = [], 0
    for r in range(n):
        m = base + (1 if r < extra else 0)
        out.append((k, k + m))
        k += m
    return out


@dataclass(frozen=True)
class Slab:
    """Slab r: owned planes [k0, k1), held planes [lo, hi) of Nz, ghost
    depth (planes exchanged, steps between exchanges) `depth`."""
    index: int
    k0: int
    k1: int
    lo: int
    hi: int
    depth: int = 1

    @property
    def n_local(self):
        return self.hi - self.lo


def layout(Nz, n, depth=1):
    """The slabs of an n-way split of Nz planes (ghost and padding planes
    included in [lo, hi)) for an exchange every `depth` steps; every slab
    owns at least `depth` planes."""
    depth = int(depth)
    if depth < 1:
        raise ValueError(f"ghost depth {depth}")
    parts = partition(Nz, n)
    if n > 1 and min(k1 - k0 for k0, k1 in parts) < depth:
        raise ValueError(f"slabs of {Nz} planes / {n} own fewer than {depth} planes")
    return [Slab(r, k0, k1, max(k0 - depth - 1, 0), min(k1 + depth + 1, Nz), depth)
            for r, (k0, k1) in enumerate(parts)]


def slice_coefficients(c, lo, hi):
    """The compact coefficient set of planes [lo, hi) of `c`: ids and the
    z-dependent metric tables sliced, the z faces of the slab keeping the
    global face flags only where they are the global faces; an internal face
    carries the PEC column mask and no PMC mask (it only reaches the padding
    plane), and the H-row summation order (h_sum_desc) stays the global one."""
    Nx, Ny, Nz = c.shape
    ids = np.asarray(c.ids).reshape((Nx, Ny, Nz), order="F")[:, :, lo:hi]
    pec = list(c.pec_face)
    pmc = list(c.pmc_face)
    internal = False
    if lo > 0:
        pec[4], pmc[4], internal = 0, 1, True
    if hi < Nz:
        pec[5], pmc[5], internal = 0, 1, True
    if internal and not c.has_pec:
        # no PEC face in the grid: the x/y flags were never read, make them
        # the unmasked value before the mask is switched on
        pec[0:4] = [1, 1, 1, 1]
    cz = lambda a: np.ascontiguousarray(np.asarray(a)[..., lo:hi])
    return replace(
        c, shape=(Nx, Ny, hi - lo), ids=np.ascontiguousarray(ids.ravel(order="F")),
        Lz=cz(c.Lz), tLz=cz(c.tLz), iAx=cz(c.iAx), iAy=cz(c.iAy), itAx=cz(c.itAx),
        itAy=cz(c.itAy), pec_face=pec, pmc_face=pmc, has_pec=c.has_pec or internal,
        info=dict(c.info, slab=(lo, hi)))


class _SlabGrid:
    """The grid attributes a solver reads, for planes [lo, hi) of `grid`."""

    def __init__(self, grid, lo, hi):
        self.Nx, self.Ny, self.Nz = grid.Nx, grid.Ny, hi - lo
        self.x, self.y = grid.x, grid.y
        self.z = np.asarray(grid.z)[lo:hi + 1]
        self.dx, self.dy = grid.dx, grid.dy
        self.dz = np.asarray(grid.dz)[lo:hi]
        self.logger = SimpleNamespace(grid=dict(getattr(grid.logger, "grid", {}), slab=(lo, hi)))


def _planes(solver):
    """The live state buffers of a slab solver as (3, Nz_local, Nx*Ny)
    views: E, H and, with fp32c, the compensation words."""
    p = solver._par
    bufs = [solver._E[p], solver._H[p]]
    if solver.precision == "fp32c":
        bufs += [solver._Ec[p], solver._Hc[p]]
    nxy = solver.Nx * solver.Ny
    return [b.view(3, solver.Nz, nxy) for b in bufs]


def side_streams(solvers, mine):
    """One stream per slab of `mine` when this process holds more than one
    slab on a CUDA device (else None): ``advance`` then runs the slabs of
    one device concurrently, so that one slab's step kernel fills the last
    wave of another's."""
    devs = [solvers[r].device for r in mine]
    if len(mine) < 2 or any(getattr(d, "type", None) != "cuda" for d in devs):
        return None
    return {r: torch.cuda.Stream(device=solvers[r].device) for r in mine}


def advance(solvers, mine, count, n0, beam=None, captures=None, streams=None):
    """`count` steps from step n0 of the slabs `mine` (fused beam parameters
    and Ez capture per slab optional).  With `streams` (``side_streams``)
    each slab's launches go to its own stream, ordered after the work on
    the device's current stream and joined back into it before the return,
    so what follows on the current stream (the exchange) sees every slab's
    steps."""
    if streams is None:
        for r in mine:
            solvers[r]._advance(count, n0, beam=beam,
                                capture=captures[r] if captures is not None else None)
        return
    for r in mine:
        s = streams[r]
        s.wait_stream(torch.cuda.current_stream(solvers[r].device))
        with torch.cuda.stream(s):
            solvers[r]._advance(count, n0, beam=beam,
                                capture=captures[r] if captures is not None else None)
    for r in mine:
        torch.cuda.current_stream(solvers[r].device).wait_stream(streams[r])


class LocalExchange:
    """Ghost-plane exchange between slabs held by this process (any devices)."""

    def __call__(self, slabs, solvers):
        for a, b in zip(slabs[:-1], slabs[1:]):
            G = a.depth
            pa, pb = _planes(solvers[a.index]), _planes(solvers[b.index])
            for fa, fb in zip(pa, pb):
                # last G owned planes of a -> lower ghosts of b; first G owned
                # planes of b -> upper ghosts of a
                fb[:, a.k1 - G - b.lo:a.k1 - b.lo].copy_(fa[:, a.k1 - G - a.lo:a.k1 - a.lo],
                                                         non_blocking=True)
                fa[:, b.k0 - a.lo:b.k0 + G - a.lo].copy_(fb[:, b.k0 - b.lo:b.k0 + G - b.lo],
                                                         non_blocking=True)


class DistExchange:
    """Ghost-plane exchange with the neighbouring ranks through
    torch.distributed point-to-point messages (NCCL over NVLink between GPUs,
    gloo on CPU): rank r holds slab r, sends its first G owned planes down
    and its last G owned planes up, and receives its ghost planes.  Each
    message is one field component over G consecutive planes, a contiguous
    range of the state buffer itself: nothing is packed, copied or
    allocated per exchange (the message lists of the two ping-pong buffers
    are built once).  The sends and receives of an exchange go out as one
    batch (``batch_isend_irecv``), so the order in which neighbours post
    them cannot deadlock."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._ops = {}

    def _global(self, r):
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def _op_list(self, s, solver):
        key = (id(solver), solver._par, s.depth)
        ops = self._ops.get(key)
        if ops is None:
            dist, G = self.dist, s.depth
            ops = []
            for f in _planes(solver):
                for d in range(f.shape[0]):
                    for nb, send0, recv0 in ((s.index - 1, s.k0, s.k0 - G),
                                             (s.index + 1, s.k1 - G, s.k1)):
                        if nb < 0 or nb >= self.world:
                            continue
                        peer = self._global(nb)
                        snd = f[d, send0 - s.lo:send0 - s.lo + G]
                        rcv = f[d, recv0 - s.lo:recv0 - s.lo + G]
                        ops.append(dist.P2POp(dist.isend, snd, peer, self.group))
                        ops.append(dist.P2POp(dist.irecv, rcv, peer, self.group))
            self._ops[key] = ops
        return ops

    def __call__(self, slabs, solvers):
        if self.world == 1:
            return
        s = slabs[self.rank]
        for req in self.dist.batch_isend_irecv(self._op_list(s, solvers[self.rank])):
            req.wait()


class SlabWakeSolve:
    """``wakesolve`` over z-slabs.

    grid, wake and the boundary / material / dtype arguments are those of
    ``SolverFIT3D``.  With ``n_slabs`` every slab lives in this process
    (``devices``: one device or one per slab; default the current CUDA
    device) and the ghost planes are copied device to device; without it and
    with torch.distributed initialised, rank r of ``group`` steps slab r on
    its current CUDA device and the ghosts travel as point-to-point messages.
    ``depth``: ghost planes per side = steps between exchanges.
    """

    def __init__(self, grid, wake=None, n_slabs=None, group=None, cfln=0.5, dt=None,
                 bc_low=("Periodic", "Periodic", "Periodic"),
                 bc_high=("Periodic", "Periodic", "Periodic"), use_stl=False, use_sibc=True,
                 fmax=None, dtype=np.float64, n_pml=10, bg=(1.0, 1.0), precision=None,
                 devices=None, verbose=0, depth=1):
        from .solverFIT3D import SolverFIT3D
        self.grid, self.wake = grid, wake
        self.Nx, self.Ny, self.Nz = grid.Nx, grid.Ny, grid.Nz
        self.N = self.Nx * self.Ny * self.Nz
        if n_slabs is None:
            import torch.distributed as dist
            if not (dist.is_available() and dist.is_initialized()):
                raise ValueError("give n_slabs, or initialise torch.distributed (one rank per slab)")
            self.exchange = DistExchange(group)
            n = self.exchange.world
            mine = [self.exchange.rank]
        else:
            self.exchange = LocalExchange()
            n = int(n_slabs)
            mine = list(range(n))
        self.slabs = layout(self.Nz, n, depth)
        self.depth = int(depth)
        self.mine = mine
        if fmax is None:
            fmax = wake.fmax if wake is not None else 1e9
        self.bc_low, self.bc_high = list(bc_low), list(bc_high)
        c = build_coefficients(grid, self.bc_low, self.bc_high, dtype=np.dtype(dtype).type,
                               bg=bg, use_stl=use_stl, use_sibc=use_sibc, fmax=fmax,
                               n_pml=n_pml, cfln=cfln, dt=dt, verbose=verbose)
        self.coefficients = c
        self.dt = c.dt
        if devices is None:
            devices = [torch.device("cuda", torch.cuda.current_device())] * n
        elif not isinstance(devices, (list, tuple)):
            devices = [torch.device(devices)] * n
        self.solvers = {}
        for r in mine:
            s = self.slabs[r]
            self.solvers[r] = SolverFIT3D(
                _SlabGrid(grid, s.lo, s.hi), wake=None, bc_low=bc_low, bc_high=bc_high,
                dtype=dtype, verbose=0, precision=precision, device=devices[r],
                coefficients=slice_coefficients(c, s.lo, s.hi), fmax=fmax)
        self.precision = precision
        self.streams = side_streams(self.solvers, mine)
        self.x = grid.x[:-1] + grid.dx / 2
        self.y = grid.y[:-1] + grid.dy / 2
        self.z = grid.z[:-1] + grid.dz / 2

    # ----------------------------------------------------------- stepping
    def _block(self, n0, count, beam=None, captures=None):
        """Steps n0 .. n0+count-1 (count <= depth) of every slab, then the
        exchange."""
        advance(self.solvers, self.mine, count, n0, beam, captures, self.streams)
        self.exchange(self.slabs, self.solvers)

    def _steps(self, n0, n_steps, beam=None, captures=None):
        n = n0
        while n < n0 + n_steps:
            c = min(self.depth, n0 + n_steps - n)
            self._block(n, c, beam, captures)
            n += c

    def run(self, n_steps, step0=0, beam=None):
        """n_steps steps (optionally with the fused beam parameters)."""
        self._steps(step0, n_steps, beam)
        for r in self.mine:
            self.solvers[r].check_status(f"SlabWakeSolve.run (slab {r})")

    def fields(self):
        """(E, H) of the owned planes of this process's slabs joined along z,
        as flat 3N float64 numpy arrays in the single-domain layout (with
        torch.distributed, each rank fills its own planes; the others are 0)."""
        nxy = self.Nx * self.Ny
        out = []
        for which in ("E", "H"):
            g = np.zeros((3, self.Nz, nxy))
            for r in self.mine:
                s, so = self.slabs[r], self.solvers[r]
                buf = (so._E if which == "E" else so._H)[so._par].double()
                if self.precision == "fp32c":
                    cw = (so._Ec if which == "E" else so._Hc)[so._par].double()
                    buf = buf + cw
                v = buf.view(3, so.Nz, nxy)[:, s.k0 - s.lo:s.k1 - s.lo]
                g[:, s.k0:s.k1] = v.cpu().numpy()
            out.append(g.reshape(-1))
        return out

    # --------------------------------------------------------------- wake
    def wakesolve(self, wakelength, compute_plane="both"):
        """Upstream ``wakesolve`` (routines.py:231-482) over the slabs: the
        fused beam and the Ez capture run in every slab's step, the history
        is joined along z and integrated by ``self.wake``.  Returns the
        CUDA-event time of the stepping loop in ms."""
        w = self.wake
        if w is None:
            raise AttributeError("Wake solver information not passed to the solver instantiation")
        ixt = int(np.abs(self.x - w.xtest).argmin())
        iyt = int(np.abs(self.y - w.ytest).argmin())
        longitudinal = compute_plane.lower() == "longitudinal"
        if longitudinal:
            xx, yy, i0, j0, ni, nj = ixt, iyt, ixt, iyt, 1, 1
        else:
            xx, yy = slice(ixt - 1, ixt + 2), slice(iyt - 1, iyt + 2)
            i0, j0, ni, nj = ixt - 1, iyt - 1, 3, 3
            if i0 < 0 or j0 < 0 or i0 + 3 > self.Nx or j0 + 3 > self.Ny:
                raise ValueError("the 3x3 Ez window around the test line leaves the grid")
        w.wakelength = wakelength
        z = self.z
        tmax = (wakelength + w.ti * w.v + (z.max() - z.min())) / w.v
        Nt = int(tmax / self.dt)
        self.Nt = Nt
        view = SimpleNamespace(x=self.x, y=self.y, z=self.z, dx=self.grid.dx, dy=self.grid.dy)
        beam = Beam(q=w.q, sigmaz=w.sigmaz, beta=w.beta, xsource=w.xsource, ysource=w.ysource)
        bp = beam.params(view)
        hists, caps = {}, {}
        for r in self.mine:
            so = self.solvers[r]
            so.reset_fields()
            so.step_0, so.nstep = True, 0
            hists[r] = torch.zeros((ni * nj, so.Nz, max(Nt, 1)), dtype=so._cap_dtype,
                                   device=so.device)
            caps[r] = (hists[r], i0, j0, ni, nj)
        devs = {self.solvers[r].device for r in self.mine}
        for d in devs:
            torch.cuda.synchronize(d)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record()
        self._steps(0, Nt, bp, caps)
        ev1.record()
        for d in devs:
            torch.cuda.synchronize(d)
        for r in self.mine:
            self.solvers[r].check_status(f"SlabWakeSolve.wakesolve (slab {r})")
        ms = ev0.elapsed_time(ev1)
        elapsed = time.perf_counter() - t0
        hist = self._join_history(hists)
        if hist is not None:
            w.xf, w.yf, w.zf = self.x[xx], self.y[yy], z[slice(0, self.Nz)]
            w.dx, w.dy, w.dz = self.grid.dx, self.grid.dy, self.grid.dz
            w.t = np.arange(0, Nt * self.dt, self.dt)
            w.set_history(hist, n_steps=Nt, one_d=longitudinal)
            w.solve(compute_plane=compute_plane)
            w.logger.wakeSolver["simulationTime"] = elapsed
        self.timing = {"ms": ms, "steps": Nt, "cells": self.N,
                       "gcell_steps_per_s": self.N * Nt / (ms / 1e3) / 1e9 if ms > 0 else None}
        return ms

    def _join_history(self, hists):
        """The (window, Nz, Nt) history joined along z on the first slab's
        device (rank 0 with torch.distributed; None on the other ranks)."""
        if isinstance(self.exchange, LocalExchange):
            dev = self.solvers[self.mine[0]].device
            parts = [hists[r][:, self.slabs[r].k0 - self.slabs[r].lo:
                              self.slabs[r].k1 - self.slabs[r].lo].to(dev) for r in self.mine]
            return torch.cat(parts, dim=1).contiguous()
        dist, ex = self.exchange.dist, self.exchange
        r = ex.rank
        s = self.slabs[r]
        mine = hists[r][:, s.k0 - s.lo:s.k1 - s.lo].contiguous()
        if r != 0:
            dist.send(mine, ex._global(0), group=ex.group)
            return None
        parts = [mine]
        for q in range(1, ex.world):
            sq = self.slabs[q]
            buf = torch.empty((mine.shape[0], sq.k1 - sq.k0, mine.shape[2]), dtype=mine.dtype,
                              device=mine.device)
            dist.recv(buf, ex._global(q), group=ex.group)
            parts.append(buf)
        return torch.cat(parts, dim=1).contiguous()
