"""Time loops of the solver: ``wakesolve`` and ``emsolve`` (upstream
wakis/routines.py:17-482).

``wakesolve`` runs the whole loop on the device: the beam current and the
capture of the Ez window around the test line (3x3 cells, or the line
alone for compute_plane='longitudinal') are fused into the step kernel, the
Ez history stays in device memory, and ``WakeSolver.solve`` integrates it
there.  Only a user callback or field monitor makes the loop return to the
host between steps, as upstream calls them every step.
"""

import ctypes
import time

import numpy as np
import torch

from .sources import Beam


class RoutinesMixin:
    # the whole Ez history is kept on the device up to this size (bytes);
    # longer runs integrate it chunk by chunk (history="stream")
    HISTORY_MAX_BYTES = 4 << 30
    STREAM_CHUNK = 256

    def wakesolve(self, wakelength, wake=None, callback=None, compute_plane="both",
                  plot=False, save_J=False, add_space=None, use_field_monitor=False,
                  field_monitor=None, history="auto", **kwargs):
        """``history``: "full" keeps the whole Ez window history on the
        device and integrates it afterwards as upstream does (value for
        value); "stream" adds each chunk of steps into the wake-potential
        sums as it completes (memory O(samples) instead of O(steps), equal
        to the full form to rounding); "auto" streams when the full history
        would exceed HISTORY_MAX_BYTES."""
        ws = self._wake_setup(wakelength, wake, compute_plane, add_space, history=history)
        bp, cap, Nt = ws["beam_params"], ws["capture"], ws["Nt"]
        t0 = time.time()
        if ws["stream"]:
            self._wake_axes(ws)
            w = self.wake
            w.stream_begin(Nt, 1 if ws["longitudinal"] else 9, ws["longitudinal"], self.device)
            ring, rest = cap[0], cap[1:]
            R = ring.shape[-1]
            for n0 in range(0, Nt, R):
                c = min(R, Nt - n0)
                if callback is None and not (use_field_monitor and field_monitor is not None):
                    self._advance(c, n0, beam=bp, capture=(ring,) + rest + (n0,))
                else:
                    for n in range(n0, n0 + c):
                        self._advance(1, n, beam=bp, capture=(ring,) + rest + (n0,))
                        if use_field_monitor and field_monitor is not None:
                            field_monitor.update(self.E, self.dt)
                        if callback is not None:
                            callback(self, n * self.dt)
                w.stream_add(ring, n0, c)
        elif callback is None and not (use_field_monitor and field_monitor is not None):
            self._advance(Nt, 0, beam=bp, capture=cap)
        else:
            for n in range(Nt):
                self._advance(1, n, beam=bp, capture=cap)
                if use_field_monitor and field_monitor is not None:
                    field_monitor.update(self.E, self.dt)
                if callback is not None:
                    callback(self, n * self.dt)
        self.check_status("wakesolve")
        self._wake_finish(ws, time.time() - t0)

    def _wake_setup(self, wakelength, wake=None, compute_plane="both", add_space=None,
                    history="full"):
        """Everything wakesolve prepares before stepping (upstream
        routines.py:322-375): test indices, Nt from the wakelength, the beam
        parameters and the device Ez history with its capture window."""
        if wake is not None:
            self.wake = wake
        if self.wake is None:
            raise AttributeError("Wake solver information not passed to the solver instantiation")
        if add_space is not None:
            self.wake.skip_cells = add_space
        w = self.wake
        self.xtest, self.ytest = w.xtest, w.ytest
        self.ixt = int(np.abs(self.x - self.xtest).argmin())
        self.iyt = int(np.abs(self.y - self.ytest).argmin())
        longitudinal = compute_plane.lower() == "longitudinal"
        if longitudinal:
            xx, yy = self.ixt, self.iyt
            i0, j0, ni, nj = self.ixt, self.iyt, 1, 1
        else:
            xx = slice(self.ixt - 1, self.ixt + 2)
            yy = slice(self.iyt - 1, self.iyt + 2)
            i0, j0, ni, nj = self.ixt - 1, self.iyt - 1, 3, 3
            if i0 < 0 or j0 < 0 or i0 + 3 > self.Nx or j0 + 3 > self.Ny:
                raise ValueError("the 3x3 Ez window around the test line leaves the grid")
        w.wakelength = wakelength
        self.ti, self.v = w.ti, w.v
        z = self.z
        tmax = (wakelength + self.ti * self.v + (z.max() - z.min())) / self.v
        Nt = int(tmax / self.dt)
        self.tmax, self.Nt = tmax, Nt
        beam = Beam(q=w.q, sigmaz=w.sigmaz, beta=w.beta, xsource=w.xsource, ysource=w.ysource)
        esize = torch.tensor([], dtype=self._cap_dtype).element_size()
        full_bytes = ni * nj * self.Nz * max(Nt, 1) * esize
        if history not in ("auto", "full", "stream"):
            raise ValueError(f"history {history!r}: 'auto', 'full' or 'stream'")
        stream = history == "stream" or (history == "auto" and
                                         full_bytes > self.HISTORY_MAX_BYTES)
        cols = min(self.STREAM_CHUNK, max(Nt, 1)) if stream else max(Nt, 1)
        hist = torch.zeros((ni * nj, self.Nz, cols), dtype=self._cap_dtype, device=self.device)
        return {"beam": beam, "beam_params": beam.params(self), "hist": hist,
                "capture": (hist, i0, j0, ni, nj), "Nt": Nt, "longitudinal": longitudinal,
                "xx": xx, "yy": yy, "compute_plane": compute_plane, "stream": stream}

    def _wake_axes(self, ws):
        """The WakeSolver's axes of this run (upstream routines.py:462-476)."""
        w, z = self.wake, self.z
        w.xf, w.yf, w.zf = self.x[ws["xx"]], self.y[ws["yy"]], z[slice(0, self.Nz)]
        w.dx, w.dy, w.dz = self.grid.dx, self.grid.dy, self.grid.dz
        w.t = np.arange(0, ws["Nt"] * self.dt, self.dt)

    def _wake_finish(self, ws, elapsed=0.0):
        """Integrate the captured Ez history (upstream routines.py:462-482)."""
        w = self.wake
        self.beam = ws["beam"]
        self._wake_axes(ws)
        if not ws.get("stream"):
            w.set_history(ws["hist"], n_steps=ws["Nt"], one_d=ws["longitudinal"])
        w.solve(compute_plane=ws["compute_plane"])
        self.logger.wakeSolver = w.logger.wakeSolver
        self.logger.wakeSolver["wakelength"] = w.wakelength
        self.logger.wakeSolver["simulationTime"] = elapsed
        if getattr(w, "save", False):
            self.logger.save_logs(w.folder)

    def emsolve(self, Nt, source=None, callback=None, **kwargs):
        """Nt steps with an optional host source ``source.update(self, t)``
        and callback (upstream routines.py:17-229, without HDF5 saving or
        plotting).  ABC boundaries are updated after every step from the
        n-2 snapshot as upstream does.  A source that tabulates its values
        (``device_terms``: PlaneWave, WavePacket, Dipole, Pulse) is written
        on the device before every step (``wk_source_write``) instead of
        through ``update``; ``device_sources=False`` keeps ``update``."""
        self.Nt = Nt
        if source is not None:
            self.source = source
        terms = None
        if source is not None and kwargs.get("device_sources", True) and \
                hasattr(source, "device_terms"):
            terms = source.device_terms(self, Nt)
            if terms is not None:
                terms = [self._upload_source_term(t) for t in terms]
        if (terms is not None and not self.activate_abc and callback is None and
                kwargs.get("graph", True) and Nt > 2 * self._GRAPH_STEPS):
            self._emsolve_graph(terms, Nt)
            self.check_status("emsolve")
            return
        if self.activate_abc:
            E2, H2 = self.get_abc()
            E1, H1 = self.get_abc()
        for n in range(Nt):
            if terms is not None:
                for t in terms:
                    self._write_source_term(t, n, Nt)
            elif source is not None:
                source.update(self, n * self.dt)
            self.one_step()
            if self.activate_abc:
                self.update_abc(E2, H2)
                E2, H2 = E1, H1
                E1, H1 = self.get_abc()
            if callback is not None:
                callback(self, n * self.dt)
        self.check_status("emsolve")

    # steps per replay of the captured emsolve chunk (even: the ping-pong
    # parity at the start of every replay is the one it was captured with)
    _GRAPH_STEPS = 16

    def _emsolve_graph(self, terms, Nt):
        """emsolve with device sources, no ABC and no callback: the first two
        steps eagerly (ghost zeroing; the stored-J state settles once a
        source has written after a step), then chunks of _GRAPH_STEPS steps
        (source writes + step) captured once in a CUDA graph and replayed,
        the source tables indexed by a device step counter; the remaining
        steps eagerly."""
        from . import _native
        lib = self._lib
        for n in range(2):
            for t in terms:
                self._write_source_term(t, n, Nt)
            self.one_step()
        if self.use_conductivity and any(t["field"] in ("E", "J") for t in terms):
            # a write to E or J between conductive steps keeps upstream's
            # stored J = sigma*E of the step before (the eager loop
            # materialises it before each write): with the J array
            # materialised once, every captured step reads it and writes
            # sigma*E_new back for the next one
            self._materialize_J()
        K = self._GRAPH_STEPS
        reps = (Nt - 2) // K
        dev = self.device
        counter = torch.full((1,), 2, dtype=torch.int64, device=dev)
        par0 = self._par
        base = self._step_desc()
        descs = []
        for q in range(K):
            d = _native.FitDesc.from_buffer_copy(base)
            d.par = par0 ^ (q & 1)
            descs.append(d)
        main = torch.cuda.Stream(dev)
        main.wait_stream(torch.cuda.current_stream(dev))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=main):
            st = ctypes.c_void_p(main.cuda_stream)
            for q in range(K):
                self._par = par0 ^ (q & 1)
                for t in terms:
                    self._write_source_term(t, q, Nt, step_dev=counter, stream=st)
                _native.check(lib.wk_fit_step(descs[q], 1, 0, st), "wk_fit_step")
            _native.check(lib.wk_counter_add(ctypes.c_void_p(counter.data_ptr()), K, st),
                          "wk_counter_add")
        self._par = par0
        torch.cuda.current_stream(dev).wait_stream(main)
        for _ in range(reps):
            graph.replay()
        torch.cuda.current_stream(dev).wait_stream(main)
        del graph
        self.nstep += reps * K
        for n in range(2 + reps * K, Nt):
            for t in terms:
                self._write_source_term(t, n, Nt)
            self.one_step()

    def _upload_source_term(self, term):
        """The tables of a source term on the device (FP64)."""
        dev = self.device
        up = dict(term)
        for k in ("A", "B", "prof"):
            v = term[k]
            if v is not None:
                v = np.asarray(v, np.float64)
                if k == "prof":
                    v = v.ravel(order="F")      # i fastest, as the kernel reads it
                up[k] = torch.as_tensor(np.ascontiguousarray(v), device=dev)
        return up

    def _write_source_term(self, term, n, n_steps, step_dev=None, stream=None):
        """Write step n (+ *step_dev) of a source term into the live field
        (E, H: the live ping-pong buffer and, with fp32c, its compensation
        words; J: the stored current, materialised first)."""
        from . import _native
        fld = term["field"]
        comp = None
        if fld == "J":
            self._materialize_J()
            buf = self._J
            dtype = _native.WK_F64 if self._J.dtype == torch.float64 else _native.WK_F32
        else:
            self._field_written(self.E if fld == "E" else self.H, reset_comp=False)
            bufs = self._E if fld == "E" else self._H
            buf = bufs[self._par]
            if self.precision == "fp32c":
                comp = (self._Ec if fld == "E" else self._Hc)[self._par]
                dtype = _native.WK_F32C
            else:
                dtype = _native.WK_F64 if buf.dtype == torch.float64 else _native.WK_F32
        ptr = lambda t: None if t is None else t.data_ptr()
        i0, i1, j0, j1, k0, k1 = term["box"]
        _native.check(self._lib.wk_source_write(
            buf.data_ptr(), dtype, ptr(comp), self.Nx, self.Ny, self.Nz, term["component"],
            i0, i1, j0, j1, k0, k1, ptr(term["prof"]), ptr(term["A"]), ptr(term["B"]),
            n_steps, ptr(step_dev), n, self._stream() if stream is None else stream),
            "wk_source_write")

    # ABC snapshots (upstream boundaries.py:313-410).  One dict per axis, as
    # upstream keeps them: with ABC on both sides of an axis the high side's
    # dict replaces the low side's, and update_abc then raises KeyError as
    # upstream does.  With views (upstream's CPU path, use_gpu=False) an
    # entry reads its plane when update_abc uses it, so a low face takes the
    # current first interior plane and a high face keeps its own values;
    # with copies (upstream's GPU path) both take the values of the call.
    def get_abc(self):
        E_abc, H_abc = {}, {}
        snap = (lambda f, idx: _LivePlane(f, idx)) if self._abc_views else _plane_copy
        for a in range(3):
            if self.bc_low[a].lower() == "abc":
                E_abc[a], H_abc[a] = {}, {}
                for d in "xyz":
                    E_abc[a][d + "lo"] = snap(self.E, (*_plane(a, 1), d))
                    H_abc[a][d + "lo"] = snap(self.H, (*_plane(a, 1), d))
        for a in range(3):
            if self.bc_high[a].lower() == "abc":
                E_abc[a], H_abc[a] = {}, {}
                for d in "xyz":
                    E_abc[a][d + "hi"] = snap(self.E, (*_plane(a, -1), d))
                    H_abc[a][d + "hi"] = snap(self.H, (*_plane(a, -1), d))
        return E_abc, H_abc

    def update_abc(self, E_abc, H_abc):
        val = lambda v: v.read() if isinstance(v, _LivePlane) else v
        for a in range(3):
            if self.bc_low[a].lower() == "abc":
                for d in "xyz":
                    self.E[(*_plane(a, 0), d)] = val(E_abc[a][d + "lo"])
                    self.H[(*_plane(a, 0), d)] = val(H_abc[a][d + "lo"])
        for a in range(3):
            if self.bc_high[a].lower() == "abc":
                for d in "xyz":
                    self.E[(*_plane(a, -1), d)] = val(E_abc[a][d + "hi"])
                    self.H[(*_plane(a, -1), d)] = val(H_abc[a][d + "hi"])


def _plane(axis, p):
    """Index tuple (without the component) of plane p normal to `axis`."""
    idx = [slice(None)] * 3
    idx[axis] = p
    return tuple(idx)


def _plane_copy(field, idx):
    """Device copy of one component plane, idx = (i, j, k, component)."""
    return field._comp(idx[3])[idx[0], idx[1], idx[2]].clone()


class _LivePlane:
    """A plane of a field read when it is used (upstream's CPU snapshots are
    numpy views of the live field arrays)."""

    def __init__(self, field, idx):
        self.field, self.idx = field, idx

    def read(self):
        return _plane_copy(self.field, self.idx)
