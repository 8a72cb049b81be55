"""Gradients of an impedance-band loss with respect to per-cell eps_r and
sigma: reverse-mode (adjoint) FIT stepping with checkpointed forward states.

Upstream has no differentiation; this follows the forward path of
``wakesolve`` (wakis/routines.py:231-482) with the longitudinal wake
(wakis/wakeSolver.py:310-420) and impedance (631-700), and differentiates

    L = integral over [f0, f1] of |Z_par(f)|^2 df        (trapezoid on the bins)

with respect to eps_r and sigma of the cells of a design region, at a fixed
time step (the relaxation-time clamp of the constructor is not re-evaluated).

* Forward: the solver steps n_steps with the fused beam and the capture of Ez
  on the test line; (E, H) are copied every ``segment`` steps (sqrt(n_steps)
  by default).
* Loss: WP(s) and the kept DFT bins of Z are rebuilt from the captured
  history with torch operations (same s axis, int() time index and negative
  index wrap as the wake kernel), so torch autograd gives dL/dEz(k, n).
* Backward: segment by segment from the end, the forward states of the
  segment are recomputed from its checkpoint, then the adjoint steps
  (``wk_adj_h_fit``, ``wk_adj_e_fit``: A^T and B0^T applied as z-marching
  tiled stencils, with the cell factors formed once per backward pass from
  the compact coefficient tables the step kernels read
  (``wk_adj_factors``); ``operators="csr"``
  uses ``wk_adj_h`` / ``wk_adj_e`` with CSR matrices assembled on the host
  instead) run backwards with dL/dEz injected at the test line, and
  ``wk_adj_grad``
  accumulates the parameter adjoints of every step (the eps increment
  dt (B0 H' - J) of the design entries is re-formed in FP64 from the
  recomputed H', so a float state loses nothing to E' - E cancellation).
* A solver with ``precision="fp32c"`` runs the forward and recomputation
  passes in FP32 values plus bf16 compensation words: checkpoints hold both,
  and the states the parameter adjoints read are the FP64 sums v + c.  The
  plain float32 forward loses a few per cent of the gradient to its state
  rounding over ~1000 steps; the compensated forward keeps FP64 accuracy.

``ImpedanceLoss`` wraps this in a torch.autograd.Function.
"""

import ctypes

import numpy as np
import torch
from scipy import sparse
from scipy.constants import epsilon_0 as EPS_0

from . import _native

_TERMS_H = {0: [(1, "0", 1), (1, "z", -1), (2, "0", -1), (2, "y", 1)],
            1: [(0, "0", -1), (0, "z", 1), (2, "0", 1), (2, "x", -1)],
            2: [(0, "0", 1), (0, "y", -1), (1, "0", -1), (1, "x", 1)]}
_TERMS_E = {0: [(1, "z", 1), (1, "0", -1), (2, "y", -1), (2, "0", 1)],
            1: [(0, "z", -1), (0, "0", 1), (2, "x", 1), (2, "0", -1)],
            2: [(0, "y", 1), (0, "0", -1), (1, "x", -1), (1, "0", 1)]}


def _face_val(f, d, i, j, k, Nx, Ny, Nz):
    """Face mask of component d (later faces win: x-lo, x-hi, y-lo, y-hi,
    z-lo, z-hi; wakis/boundaries.py:92-101), vectorised over cells."""
    v = np.ones(i.shape, np.float64)
    if d != 0:
        v[i == 0] = f[0]
        v[i == Nx - 1] = f[1]
    if d != 1:
        v[j == 0] = f[2]
        v[j == Ny - 1] = f[3]
    if d != 2:
        v[k == 0] = f[4]
        v[k == Nz - 1] = f[5]
    return v


def assemble_operators(solver):
    """(A, B0) as scipy CSR (float64, 3N x 3N): H' = H - A E and
    E' = E + dt diag(ieps) (B0 H' - J), built from the solver's compact
    coefficient set with the kernels' conventions (flat-offset neighbours,
    PEC column / PMC row masks for A, PEC row / PMC column masks for B0)."""
    c = solver._coef
    Nx, Ny, Nz = solver.Nx, solver.Ny, solver.Nz
    N = Nx * Ny * Nz
    NxNy = Nx * Ny
    n = np.arange(N, dtype=np.int64)
    i, j, k = n % Nx, (n // Nx) % Ny, n // NxNy
    dt = float(solver.dt)
    imu = np.asarray(c.table, np.float64)[np.asarray(c.ids, np.int64)][:, 3:6]
    L = [np.asarray(c.Lx, np.float64), np.asarray(c.Ly, np.float64), np.asarray(c.Lz, np.float64)]
    tL = [np.asarray(c.tLx, np.float64), np.asarray(c.tLy, np.float64),
          np.asarray(c.tLz, np.float64)]
    iA = [np.asarray(c.iAx, np.float64)[j, k], np.asarray(c.iAy, np.float64)[i, k],
          np.asarray(c.iAz, np.float64)[i, j]]
    itA = [np.asarray(c.itAx, np.float64)[j, k], np.asarray(c.itAy, np.float64)[i, k],
           np.asarray(c.itAz, np.float64)[i, j]]
    off = {"0": 0, "x": 1, "y": Nx, "z": NxNy}
    rows_a, cols_a, vals_a, rows_b, cols_b, vals_b = [], [], [], [], [], []
    coord = lambda m: (m % Nx, (m // Nx) % Ny, m // NxNy)
    for d in range(3):
        R = iA[d] * imu[:, d]
        if c.has_pmc:
            R = R * _face_val(c.pmc_face, d, i, j, k, Nx, Ny, Nz)
        for e, o, sg in _TERMS_H[d]:
            m = n + off[o]
            ok = m < N
            nn, mm = n[ok], m[ok]
            im_, jm, km = coord(mm)
            col = L[e][(im_, jm, km)[e]]
            if c.has_pec:
                col = col * _face_val(c.pec_face, e, im_, jm, km, Nx, Ny, Nz)
            rows_a.append(d * N + nn)
            cols_a.append(e * N + mm)
            vals_a.append(sg * dt * R[ok] * col)
        R = itA[d].copy()
        if c.has_pec:
            R = R * _face_val(c.pec_face, d, i, j, k, Nx, Ny, Nz)
        for e, o, sg in _TERMS_E[d]:
            m = n - off[o]
            ok = m >= 0
            nn, mm = n[ok], m[ok]
            im_, jm, km = coord(mm)
            col = tL[e][(im_, jm, km)[e]]
            if c.has_pmc:
                col = col * _face_val(c.pmc_face, e, im_, jm, km, Nx, Ny, Nz)
            rows_b.append(d * N + nn)
            cols_b.append(e * N + mm)
            vals_b.append(sg * R[ok] * col)
    cat = np.concatenate
    A = sparse.csr_matrix((cat(vals_a), (cat(rows_a), cat(cols_a))), shape=(3 * N, 3 * N))
    B0 = sparse.csr_matrix((cat(vals_b), (cat(rows_b), cat(cols_b))), shape=(3 * N, 3 * N))
    return A, B0


class _DevCSR:
    """CSR matrix on the device: int64 row pointers, int32 columns."""

    def __init__(self, m, dtype, device):
        m = m.tocsr()
        m.sort_indices()
        self.n = m.shape[0]
        self.rowptr = torch.as_tensor(m.indptr.astype(np.int64), device=device)
        self.col = torch.as_tensor(m.indices.astype(np.int32), device=device)
        self.val = torch.as_tensor(m.data, dtype=dtype, device=device)


class ImpedanceDesign:
    """Loss and gradient of L = int_{f0}^{f1} |Z_par|^2 df over the per-cell
    eps_r and sigma of `design` (boolean (Nx, Ny, Nz) mask) for one solver
    (dtype float32 or float64, or precision "fp32c", built with its
    WakeSolver).  n_steps fixes Nt (the wakelength is set so that upstream's
    Nt formula gives it).  adjoint_dtype (np.float32 / np.float64) is the
    dtype of the adjoint state, by default the solver's coefficient dtype."""

    def __init__(self, solver, design, f_band=(0.5e9, 3e9), n_steps=4000, segment=None,
                 samples=1001, adjoint_dtype=None, operators="stencil"):
        s = self.s = solver
        if s.precision not in (None, "fp32c"):
            raise ValueError(f"ImpedanceDesign: precision {s.precision!r} not supported")
        self.comp = s.precision == "fp32c"
        self.dev = s.device
        # adjoint state dtype (default: the solver's); the forward states are
        # converted to it where the parameter adjoints read them
        adt = adjoint_dtype if adjoint_dtype is not None else s.dtype
        self.tdtype = torch.float64 if adt == np.float64 else torch.float32
        self.wk = _native.WK_F64 if adt == np.float64 else _native.WK_F32
        mask = np.asarray(design, bool)
        self.cells_np = np.flatnonzero(mask.ravel(order="F")).astype(np.int64)
        self.cells = torch.as_tensor(self.cells_np, device=self.dev)
        self.n_steps = int(n_steps)
        self.segment = int(segment) if segment else max(1, int(round(np.sqrt(self.n_steps))))
        self.f_band = f_band
        self.samples = samples
        if operators not in ("stencil", "csr"):
            raise ValueError(f"operators {operators!r}: 'stencil' or 'csr'")
        self.operators = operators
        A, B0 = assemble_operators(s)
        if operators == "csr":
            self.AT = _DevCSR(A.T, self.tdtype, self.dev)
            self.B0T = _DevCSR(B0.T, self.tdtype, self.dev)
        N = s.N
        nc = len(self.cells_np)
        # rows of B0 at the design entries (FP64): the E increment there is
        # formed as dt (B0 H' - J) instead of E' - E
        rows = np.concatenate([d * N + self.cells_np for d in range(3)])
        self.rows = torch.as_tensor(rows, device=self.dev)
        B0d = B0[rows, :].tocsr()
        self.Bd = _DevCSR(B0d, torch.float64, self.dev)
        # the same rows over only the H entries they read (for states whose
        # H' is first converted to FP64: only those entries are gathered)
        hcols = np.unique(B0d.indices)
        self.hcols = torch.as_tensor(hcols.astype(np.int64), device=self.dev)
        self.Bdc = _DevCSR(B0d[:, hcols], torch.float64, self.dev)
        # gather buffers of the design entries (E) and of the H entries the
        # design rows read, in the state types
        self._hv = torch.empty(len(hcols), dtype=s._H[0].dtype, device=self.dev)
        if self.comp:
            self._gv = torch.empty(len(rows), dtype=s._E[0].dtype, device=self.dev)
            self._gc = torch.empty(len(rows), dtype=s._Ec[0].dtype, device=self.dev)
            self._hc = torch.empty(len(hcols), dtype=s._Hc[0].dtype, device=self.dev)
        self.zd = torch.zeros(3 * nc, dtype=torch.float64, device=self.dev)
        ie, _, sg = s._dense_fields()
        self.ieps0 = ie.array.clone()
        self.sigma0 = sg.array.clone()
        self.eps_r = None
        self.sigma = None
        self.lib = _native.lib()
        # the beam line's z entries take the beam current, not sigma*E
        w = s.wake
        self.ixs = int(np.abs(s.x - w.xsource).argmin())
        self.iys = int(np.abs(s.y - w.ysource).argmin())
        sm = torch.ones(3 * N, dtype=self.tdtype, device=self.dev)
        beam_cells = self.ixs + self.iys * s.Nx + torch.arange(s.Nz, device=self.dev) * s.Nx * s.Ny
        sm[2 * N + beam_cells] = 0
        self.smask = sm
        ci = self.cells_np % s.Nx
        cj = (self.cells_np // s.Nx) % s.Ny
        on = np.flatnonzero((ci == self.ixs) & (cj == self.iys))
        self.beam_rows = torch.as_tensor(2 * nc + on, device=self.dev)
        self.beam_k = torch.as_tensor(self.cells_np[on] // (s.Nx * s.Ny), device=self.dev)
        self._ws = None
        self._prepare_loss()

    # ---------------------------------------------------------- parameters
    def set_params(self, eps_r, sigma):
        """Per-design-cell eps_r and sigma (length n_cells each)."""
        s, N = self.s, self.s.N
        er = torch.as_tensor(np.asarray(eps_r, np.float64), device=self.dev)
        sg = torch.as_tensor(np.asarray(sigma, np.float64), device=self.dev)
        ie = self.ieps0.clone().double()
        sgm = self.sigma0.clone().double()
        for d in range(3):
            ie[d * N + self.cells] = 1.0 / (er * EPS_0)
            sgm[d * N + self.cells] = sg
        f_ie, _, f_sg = s._dense_fields()
        f_ie.array.copy_(ie.to(f_ie.array.dtype))
        f_sg.array.copy_(sgm.to(f_sg.array.dtype))
        s.update_tensors()
        s.use_conductivity = bool((sgm != 0).any().item()) or s.use_conductivity
        self.ieps = f_ie.array.to(self.tdtype).contiguous()
        self.sig = f_sg.array.to(self.tdtype).contiguous()
        self.sig_d = self.sig.double()[self.rows]
        self.eps_r, self.sigma = er, sg

    # ---------------------------------------------------------------- loss
    def _prepare_loss(self):
        s, w = self.s, self.s.wake
        z = s.z
        self.wakelength = ((self.n_steps + 0.5) * float(s.dt) * w.v - w.ti * w.v
                           - (z.max() - z.min()))
        nt, dt = self.n_steps, float(s.dt)
        zmin = float(np.min(z))
        s_axis = np.arange(-w.ti * w.v, self.wakelength, dt * w.v)
        it = np.empty((len(s_axis), s.Nz), np.int64)
        for k in range(s.Nz):
            ts = (z[k] + s_axis) / w.v - zmin / w.v - 0.0 + w.ti
            it[:, k] = (ts / dt).astype(np.int64)
        ok = (it < nt) & (it >= -nt)
        it = np.where(it < 0, it + nt, it)
        it[~ok] = 0
        self.s_axis = s_axis
        self.it = torch.as_tensor(it, device=self.dev)
        self.itok = torch.as_tensor(ok, device=self.dev, dtype=torch.float64)
        self.dz = torch.as_tensor(np.asarray(s.grid.dz, np.float64)[:s.Nz], device=self.dev)
        ds = float(np.mean(s_axis[1:] - s_axis[:-1]))
        N = int((w.v / ds) // w.fmax * self.samples)
        f = np.fft.fftfreq(N, ds / w.v)
        keep = np.flatnonzero((f >= 0) & (f < w.fmax))
        band = keep[(f[keep] >= self.f_band[0]) & (f[keep] <= self.f_band[1])]
        self.f = torch.as_tensor(f[band], device=self.dev)
        idx = np.arange(len(s_axis))
        F = np.exp(-2j * np.pi * np.outer(band, idx) / N)
        self.F = torch.as_tensor(F, device=self.dev)
        lam = (1 / (w.sigmaz * np.sqrt(2 * np.pi))) * np.exp(-(s_axis ** 2) / (2 * w.sigmaz ** 2))
        self.lamf = self.F @ torch.as_tensor(lam * w.v, device=self.dev).to(torch.complex128)
        self.qscale = w.q * 1e12

    def loss_from_history(self, ez):
        """L from the test-line history ez (Nz, Nt) float64 (torch, may
        require grad): WP(s) = sum_k Ez(k, it(s, k)) dz_k / (q 1e12),
        Z = -DFT(WP 1e12) / DFT(lambda v) on the kept bins in the band."""
        nz = ez.shape[0]
        vals = ez[torch.arange(nz, device=self.dev)[None, :], self.it]
        WP = (vals * self.itok * self.dz[None, :]).sum(dim=1) / self.qscale
        Z = -(self.F @ (WP * 1e12).to(torch.complex128)) / self.lamf
        p = Z.real ** 2 + Z.imag ** 2
        return torch.trapezoid(p, self.f)

    # ------------------------------------------------------------- forward
    def _live(self):
        """The live state buffers: (E, H), and (Ec, Hc) with fp32c."""
        s = self.s
        if self.comp:
            return s._E[s._par], s._H[s._par], s._Ec[s._par], s._Hc[s._par]
        return s._E[s._par], s._H[s._par]

    def _values(self):
        """(E, H) of the live state: the state tensors, or the FP64 sums
        v + c of the compensated state."""
        st = self._live()
        if self.comp:
            return (st[0].double() + st[2].double(), st[1].double() + st[3].double())
        return st[0], st[1]

    def forward(self, keep=True):
        """Step n_steps from zero fields with beam and test-line capture;
        returns L (float).  With keep, (E, H) are copied every `segment`
        steps for the backward pass."""
        s = self.s
        s.reset_fields()
        s.step_0 = True
        s.nstep = 0
        ws = s._wake_setup(self.wakelength, compute_plane="longitudinal")
        if ws["Nt"] != self.n_steps:
            raise RuntimeError(f"step count {ws['Nt']} != {self.n_steps}")
        self._ws = ws
        self.ckpt = {}
        K = self.segment
        n = 0
        while n < self.n_steps:
            if keep:
                self.ckpt[n] = tuple(t.clone() for t in self._live())
            m = min(K, self.n_steps - n)
            s._advance(m, n, beam=ws["beam_params"], capture=ws["capture"])
            n += m
        s.check_status("ImpedanceDesign.forward")
        self.hist = ws["hist"][0].double()
        return float(self.loss_from_history(self.hist).item())

    # ------------------------------------------------------------ backward
    def _restore(self, n):
        s = self.s
        for t, c in zip(self._live(), self.ckpt[n]):
            t.copy_(c)
        s.step_0 = False
        s.nstep = n
        s._j_state = 1 if (n >= 1 and s.use_conductivity) else 0   # WK_J_SIGMA_E / ZERO

    def _beam_rows_J(self, bp):
        """Jz of the fused beam at the design entries on the beam line, for
        every step (n_steps x entries, FP64 device tensor; None without such
        entries): the expressions of ``sources.beam_line_values`` evaluated
        for all steps at once (float32 time arithmetic with a float32 dt)."""
        if not len(self.beam_rows):
            return None
        s = self.s
        _, _, qv, v, s0, c0, two_sig2, bdx, bdy = bp
        steps = np.arange(self.n_steps)
        if isinstance(s.dt, np.float32):
            vt = v * (steps.astype(np.float32) * s.dt)
        else:
            vt = v * (steps * np.float64(s.dt))
        z = np.asarray(s.z)[self.beam_k.cpu().numpy()]
        sz = z[None, :] - vt[:, None]
        prof = c0 * np.exp(-((sz - s0) ** 2) / two_sig2)
        vals = (qv * prof / bdx / bdy).astype(s.dtype).astype(np.float64)
        return torch.as_tensor(vals, device=self.dev)

    def _design_h_into(self, out):
        """H of the live state at the entries the design rows of B0 read
        (self.hcols) into `out` as FP64 (the values, or the sums v + c)."""
        st = self._live()
        if self.comp:
            torch.index_select(st[1], 0, self.hcols, out=self._hv)
            torch.index_select(st[3], 0, self.hcols, out=self._hc)
            out.copy_(self._hv)
            out.add_(self._hc)
        else:
            torch.index_select(st[1], 0, self.hcols, out=self._hv)
            out.copy_(self._hv)

    def _design_e_into(self, out):
        """E of the live state at the design entries (self.rows) into `out`
        (3 x n_cells entries: the state values, or the FP64 sums v + c)."""
        st = self._live()
        if self.comp:
            torch.index_select(st[0], 0, self.rows, out=self._gv)
            torch.index_select(st[2], 0, self.rows, out=self._gc)
            out.copy_(self._gv)
            out.add_(self._gc)
        else:
            torch.index_select(st[0], 0, self.rows, out=out)

    def _segment(self, a, m, B, graph_descs=None):
        """Recompute steps a .. a+m-1 from the restored state and run their
        reverse steps.  With graph_descs (one step descriptor per step, the
        step index read from the device counter B['ctr']) the steps are
        launched directly, as inside a captured CUDA graph; else through
        the solver.  All per-step data live in the buffers B."""
        s, lib, N = self.s, self.lib, self.s.N
        st = torch.cuda.current_stream(self.dev).cuda_stream
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        dt = float(s.dt)
        cond = bool(s.use_conductivity)
        bp = self._ws["beam_params"]
        Es, incs, J = B["Es"], B["incs"], B["J"]
        self._design_e_into(Es[0])
        par0 = s._par
        for q in range(m):
            n = a + q
            if graph_descs is None:
                s._advance(1, n, beam=bp)
            else:
                _native.check(lib.wk_fit_step(graph_descs[q], 1, 0, ctypes.c_void_p(st)),
                              "wk_fit_step")
                _native.check(lib.wk_counter_add(ptr(B["ctr"]), 1, ctypes.c_void_p(st)),
                              "wk_counter_add")
                s._par = par0 ^ ((q + 1) & 1)
            self._design_e_into(Es[q + 1])
            # dt (B0 H' - J) at the design entries, FP64
            if B["Hd"] is None:
                Hd, Bd = self._live()[1], self.Bd
            else:
                Hd, Bd = B["Hd"], self.Bdc
                self._design_h_into(Hd)
            _native.check(lib.wk_adj_e(
                _native.WK_F64, ptr(Bd.rowptr), ptr(Bd.col), ptr(Bd.val),
                Bd.n, ptr(Hd), ptr(self.zd), ptr(self.zd), ptr(incs[q]),
                ctypes.c_void_p(st)), "wk_adj_e")
            if cond and n >= 1:
                J.copy_(Es[q])
                J.mul_(self.sig_d)
                if B["bJ"] is not None:
                    J.index_copy_(0, self.beam_rows, B["bJ"][q])
                incs[q].add_(J)
            elif B["bJ"] is not None:
                incs[q].index_add_(0, self.beam_rows, B["bJ"][q])
            incs[q].mul_(-dt)
        lE, lH, gI, gS = B["lE"], B["lH"], B["gI"], B["gS"]
        for q in range(m - 1, -1, -1):
            n = a + q
            use_sig = int(cond and n >= 1)
            if B["E0"] is None:
                E0 = Es[q]
            else:
                E0 = B["E0"]
                E0.copy_(Es[q])
            _native.check(lib.wk_adj_grad(
                self.wk, ptr(self.cells), len(self.cells_np), N, ptr(lE), ptr(incs[q]),
                ptr(E0), ptr(self.ieps), ptr(self.smask), use_sig, dt, ptr(gI),
                ptr(gS), ctypes.c_void_p(st)), "wk_adj_grad")
            if self.operators == "stencil":
                d = B["coef_desc"]
                _native.check(lib.wk_adj_h_fit(d, self.wk, ptr(B["fu"]), ptr(lE), ptr(lH),
                                               ptr(lH), ctypes.c_void_p(st)), "wk_adj_h_fit")
                _native.check(lib.wk_adj_e_fit(
                    d, self.wk, ptr(B["fw"]), ptr(lH), ptr(lE),
                    ptr(B["decay"]) if use_sig else None, ptr(lE), ctypes.c_void_p(st)),
                    "wk_adj_e_fit")
            else:
                _native.check(lib.wk_adj_h(
                    self.wk, ptr(self.B0T.rowptr), ptr(self.B0T.col), ptr(self.B0T.val),
                    self.B0T.n, ptr(lE), ptr(self.ieps), dt, ptr(lH), ptr(lH),
                    ctypes.c_void_p(st)), "wk_adj_h")
                _native.check(lib.wk_adj_e(
                    self.wk, ptr(self.AT.rowptr), ptr(self.AT.col), ptr(self.AT.val),
                    self.AT.n, ptr(lH), ptr(lE), ptr(B["decay"] if use_sig else B["ones"]),
                    ptr(lE), ctypes.c_void_p(st)), "wk_adj_e")
            lE.index_add_(0, B["zidx"], B["gh"][:, q])

    def backward(self, graph=True):
        """(dL/d eps_r, dL/d sigma) of the design cells (numpy float64).

        Segment by segment from the end: restore the checkpoint, recompute
        the segment's steps, run their reverse steps.  With ``graph`` the
        full-length segments after the first run as one captured CUDA graph
        (captured on the first of them, replayed for the others: the step
        kernels read their step index from a device counter, the beam
        current and dL/dEz of the segment are staged into static buffers);
        the first segment, a shorter last one and the CSR operators run
        step by step."""
        s, N = self.s, self.s.N
        ez = self.hist.clone().requires_grad_(True)
        L = self.loss_from_history(ez)
        (g_hist,) = torch.autograd.grad(L, ez)
        g_hist = g_hist.to(self.tdtype)
        ixt = int(np.abs(s.x - s.wake.xtest).argmin())
        iyt = int(np.abs(s.y - s.wake.ytest).argmin())
        dev, K = self.dev, self.segment
        dt = float(s.dt)
        cond = bool(s.use_conductivity)
        vdt = torch.float64 if self.comp else self._live()[0].dtype
        beam_J = self._beam_rows_J(self._ws["beam_params"])
        B = {
            # E of the design entries after each step of the segment
            "Es": torch.empty((K + 1, len(self.rows)), dtype=vdt, device=dev),
            "incs": torch.empty((K, len(self.zd)), dtype=torch.float64, device=dev),
            # FP64 H' for the B0 rows: the live buffer itself for a plain
            # FP64 state, else the entries those rows read (hcols)
            "Hd": None if (not self.comp and vdt == torch.float64) else torch.empty(
                len(self.hcols), dtype=torch.float64, device=dev),
            "E0": None if vdt == self.tdtype else torch.empty(len(self.rows), dtype=self.tdtype,
                                                              device=dev),
            "J": torch.empty_like(self.zd),
            "bJ": None if beam_J is None else torch.empty((K, beam_J.shape[1]),
                                                          dtype=torch.float64, device=dev),
            "gh": torch.empty((s.Nz, K), dtype=self.tdtype, device=dev),
            "ctr": torch.zeros(1, dtype=torch.int64, device=dev),
            "zidx": 2 * N + ixt + iyt * s.Nx + torch.arange(s.Nz, device=dev) * s.Nx * s.Ny,
            "lE": torch.zeros(3 * N, dtype=self.tdtype, device=dev),
            "lH": torch.zeros(3 * N, dtype=self.tdtype, device=dev),
            "gI": torch.zeros(len(self.cells_np), dtype=torch.float64, device=dev),
            "gS": torch.zeros(len(self.cells_np), dtype=torch.float64, device=dev),
            "decay": (1.0 - dt * self.ieps.double() * self.sig.double() * self.smask.double()
                      ).to(self.tdtype) if cond else None,
            "ones": torch.ones(3 * N, dtype=self.tdtype, device=dev),
        }
        B["coef_desc"] = _native.FitDesc.from_buffer_copy(s._sync_desc())
        if self.operators == "stencil":
            # the cell factors of the two transposes, formed once
            B["fu"] = torch.empty(3 * N, dtype=self.tdtype, device=dev)
            B["fw"] = torch.empty(3 * N, dtype=self.tdtype, device=dev)
            _native.check(self.lib.wk_adj_factors(
                B["coef_desc"], self.wk, ctypes.c_void_p(B["fu"].data_ptr()),
                ctypes.c_void_p(B["fw"].data_ptr()),
                ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)), "wk_adj_factors")

        def stage(a, m):
            if B["bJ"] is not None:
                B["bJ"][:m].copy_(beam_J[a:a + m])
            B["gh"][:, :m].copy_(g_hist[:, a:a + m])

        use_graph = graph and self.operators == "stencil" and cond
        cg, cg_par, descs = None, None, None
        for a in reversed(sorted(self.ckpt)):
            m = min(K, self.n_steps - a)
            stage(a, m)
            full = use_graph and m == K and a >= 1
            if full and cg is not None:
                # replay: restore into the buffers the graph was captured on
                s._par = cg_par
                self._restore(a)
                B["ctr"].fill_(a)
                cg.replay()
                s._par = cg_par ^ (K & 1)
                continue
            self._restore(a)
            if full:
                # capture on this segment (every kernel of the segment ran
                # eagerly at least once before, on an earlier segment)
                if descs is None and getattr(self, "_warm", False):
                    cg_par = s._par
                    base = s._step_desc(self._ws["beam_params"], None)
                    descs = []
                    for q in range(K):
                        c = _native.FitDesc.from_buffer_copy(base)
                        c.par = cg_par ^ (q & 1)
                        c.step_dev = B["ctr"].data_ptr()
                        descs.append(c)
                    # every kernel the graph holds has run before capture
                    _native.check(self.lib.wk_counter_add(
                        ctypes.c_void_p(B["ctr"].data_ptr()), 0,
                        ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
                        "wk_counter_add")
                    B["ctr"].fill_(a)
                    torch.cuda.synchronize(dev)
                    cg = torch.cuda.CUDAGraph()
                    cap = torch.cuda.Stream(dev)
                    cap.wait_stream(torch.cuda.current_stream(dev))
                    with torch.cuda.graph(cg, stream=cap):
                        self._segment(a, K, B, graph_descs=descs)
                    torch.cuda.current_stream(dev).wait_stream(cap)
                    s._par = cg_par
                    self._restore(a)
                    B["ctr"].fill_(a)
                    # capture ran nothing: replay for this segment as well
                    cg.replay()
                    s._par = cg_par ^ (K & 1)
                    continue
                self._warm = True
            self._segment(a, m, B)
        self._warm = False
        del cg
        s.check_status("ImpedanceDesign.backward")
        er = self.eps_r
        g_eps = B["gI"] * (-1.0 / (EPS_0 * er * er))
        return g_eps.cpu().numpy(), B["gS"].cpu().numpy()


class ImpedanceLoss(torch.autograd.Function):
    """L(eps_r, sigma) of an ImpedanceDesign as a differentiable torch op:
    forward runs the checkpointed forward pass, backward the adjoint."""

    @staticmethod
    def forward(ctx, eps_r, sigma, problem):
        problem.set_params(eps_r.detach().cpu().numpy(), sigma.detach().cpu().numpy())
        L = problem.forward(keep=True)
        ctx.problem = problem
        return torch.tensor(L, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        ge, gs = ctx.problem.backward()
        g = float(gout)
        return (torch.as_tensor(ge * g), torch.as_tensor(gs * g), None)
