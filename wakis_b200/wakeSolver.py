"""``WakeSolver``: wake potential and impedance from the Ez history, on the
device (upstream wakis/wakeSolver.py:19-870).

The constructor keeps upstream's parameters and defaults (22-208).  After
``SolverFIT3D.wakesolve`` the Ez history is a device tensor laid out
[window][k][step]; ``solve()`` runs

* ``calc_long_WP_3d`` / ``calc_long_WP`` -> ``wk_wake_potential``,
* ``calc_trans_WP``                     -> ``wk_trans_wake``,
* ``calc_long_Z`` / ``calc_trans_Z``    -> ``wk_dft_bins`` (direct DFT of the
  kept bins 0 <= f < fmax),

with the s axis, the key order of the history and the frequency axis formed
on the host by the same numpy expressions as upstream.
"""

import os

import numpy as np
import torch
from scipy.constants import c as c_light

from . import _native
from .logger import Logger


class WakeSolver:
    def __init__(self, wakelength=None, q=1e-9, sigmaz=1e-3, beta=1.0, xsource=0.0,
                 ysource=0.0, xtest=0.0, ytest=0.0, chargedist=None, ti=None, fmax=None,
                 compute_plane="both", skip_cells=0, add_space=None, Ez_file=None, save=True,
                 results_folder="results/", verbose=1, counter_moving=False):
        self.verbose = verbose
        self.q, self.sigmaz, self.beta = q, sigmaz, beta
        self.v = self.beta * c_light
        self.xsource, self.ysource = xsource, ysource
        self.xtest, self.ytest = xtest, ytest
        self.chargedist = chargedist
        self.fmax = self.v / (3.0 * self.sigmaz) if fmax is None else fmax
        self.skip_cells = skip_cells if add_space is None else add_space
        self.compute_plane = compute_plane
        self.counter_moving = counter_moving
        if ti is not None:
            self.ti = ti
        else:
            self.ti = 8.548921333333334 * self.sigmaz / (np.sqrt(self.beta) * self.v)
        self.Ez_file = Ez_file
        self.t = None
        self.xf = self.yf = self.zf = None
        self.wakelength = wakelength
        self.s = self.lambdas = self.WP = self.WP_3d = None
        self.n_transverse_cells = 1
        self.WPx = self.WPy = self.f = self.Z = self.Zx = self.Zy = self.lambdaf = None
        self.logger = Logger()
        self.save = save
        self.folder = results_folder if results_folder.endswith("/") else results_folder + "/"
        if self.save:
            os.makedirs(self.folder, exist_ok=True)
        self._hist = None
        self._stream = None
        self.logger.wakeSolver.update(dict(ti=self.ti, q=q, sigmaz=sigmaz, beta=beta,
                                           xsource=xsource, ysource=ysource, xtest=xtest,
                                           ytest=ytest, chargedist=chargedist,
                                           skip_cells=self.skip_cells,
                                           results_folder=self.folder))

    # ------------------------------------------------------------ history
    def set_history(self, hist, n_steps, one_d=False):
        """Attach the device Ez history [window][k][step] of n_steps steps."""
        if int(n_steps) > hist.shape[-1]:
            raise ValueError(f"history of {hist.shape[-1]} steps, n_steps={n_steps}")
        self._hist = hist
        self._hist_steps = int(n_steps)
        self._hist_1d = bool(one_d)
        self._stream = None

    @staticmethod
    def _key_order(n):
        """Step index of each history column in upstream's read order: the
        '#%05d' keys sorted as strings (wakeSolver.py:488-491).  The keys are
        the decimal digits of the step, zero-padded to 5: as strings they
        sort by the digits read as a fraction (value * 10^(D - length), D the
        longest length), a key before the longer keys it is a prefix of."""
        m = np.arange(n, dtype=np.int64)
        length = np.maximum(5, np.floor(np.log10(np.maximum(m, 1))).astype(np.int64) + 1)
        # guard the float log10 at powers of ten
        length = np.where(m >= 10 ** np.minimum(length, 18), length + 1, length)
        length = np.where((length > 5) & (m < 10 ** np.maximum(length - 1, 0)), length - 1,
                          length)
        D = int(length.max()) if n else 5
        scaled = m * (10 ** (D - length))
        return np.lexsort((length, scaled)).astype(np.int64)

    @classmethod
    def _key_positions(cls, n):
        """Position of each step's key in upstream's sorted key list (the
        inverse of _key_order); None when every key keeps its place
        (n <= 10^5)."""
        if n <= 100000:
            return None
        order = cls._key_order(n)
        pos = np.empty(n, dtype=np.int64)
        pos[order] = np.arange(n, dtype=np.int64)
        return pos

    # ------------------------------------------------- streamed history
    def stream_begin(self, n_steps, n_win, one_d, device):
        """Start a streamed integration of n_steps steps (the wake-potential
        sums are added chunk by chunk with ``stream_add`` while the solver
        steps, instead of keeping the whole [window][k][step] history).
        Needs the axes (t, xf, yf, zf, dz) and the wakelength set."""
        if one_d and self.skip_cells != 0:
            raise ValueError("could not broadcast input array: skip_cells with a 1-D history")
        nt, dt, zmin, zmax, z, s = self._axis()
        nt = min(nt, int(n_steps))
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)
        pos = self._key_positions(int(n_steps))
        st = {"n_win": n_win, "one_d": bool(one_d), "nt": nt, "dt": dt, "zmin": zmin,
              "zmax": zmax, "z": f64(z), "dz": f64(self.dz), "s": f64(s), "ns": len(s),
              "nz": len(z), "win": torch.arange(n_win, dtype=torch.int32, device=device),
              "pos": None if pos is None else torch.as_tensor(pos, device=device),
              "acc": torch.zeros((n_win, len(s)), dtype=torch.float64, device=device)}
        self._stream = st
        self._hist = None
        self._hist_1d = bool(one_d)
        self.s = s
        return st

    def stream_add(self, ring, step0, n_steps):
        """Add the steps step0 .. step0+n_steps-1 held in ring columns
        0 .. n_steps-1 ([window][k][column], the capture layout)."""
        st = self._stream
        lib = _native.lib()
        hdt = _native.WK_F64 if ring.dtype == torch.float64 else _native.WK_F32
        stream = torch.cuda.current_stream(ring.device).cuda_stream
        rc = lib.wk_wake_accumulate(
            ring.data_ptr(), hdt, ring.shape[-1], ring.shape[1], int(step0), int(n_steps),
            st["win"].data_ptr(), st["n_win"], st["z"].data_ptr(), st["dz"].data_ptr(), st["nz"],
            int(self.skip_cells), st["s"].data_ptr(), st["ns"],
            None if st["pos"] is None else st["pos"].data_ptr(), int(st["nt"]), float(self.v),
            float(st["zmin"]), float(st["zmax"]), float(self.t[0]), float(self.ti),
            float(st["dt"]), int(self.counter_moving), st["acc"].data_ptr(), stream)
        _native.check(rc, "wk_wake_accumulate")

    def _stream_wp(self, carry):
        st = self._stream
        lib = _native.lib()
        WP3d = torch.empty_like(st["acc"])
        stream = torch.cuda.current_stream(WP3d.device).cuda_stream
        rc = lib.wk_wake_finalize(st["acc"].data_ptr(), st["n_win"], st["ns"], int(carry),
                                  float(self.q * 1e12), WP3d.data_ptr(), stream)
        _native.check(rc, "wk_wake_finalize")
        return WP3d

    def _axis(self):
        nt = len(self.t)
        dt = self.t[2] - self.t[1]
        zmax, zmin = np.max(self.zf), np.min(self.zf)
        zz = slice(self.skip_cells, -self.skip_cells) if self.skip_cells != 0 else np.s_[:]
        z = self.zf[zz]
        if self.wakelength is not None:
            wakelength = self.wakelength
        else:
            wakelength = nt * dt * self.v - (zmax - zmin) - self.ti * self.v
            self.wakelength = wakelength
        s = np.arange(-self.ti * self.v, wakelength, dt * self.v)
        return nt, dt, zmin, zmax, z, s

    def _wp(self, n_win, carry):
        if getattr(self, "_stream", None) is not None:
            if self._stream["n_win"] != n_win:
                raise ValueError("the streamed history holds another window count")
            return self._stream_wp(carry)
        if self._hist is None:
            raise RuntimeError("no Ez history: run SolverFIT3D.wakesolve first")
        lib = _native.lib()
        nt, dt, zmin, zmax, z, s = self._axis()
        n_keys = self._hist_steps
        nt = min(nt, n_keys)
        dev = self._hist.device
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        zt, dzt, st = f64(z), f64(self.dz), f64(s)
        order = torch.as_tensor(self._key_order(n_keys), device=dev)
        win = torch.arange(n_win, dtype=torch.int32, device=dev)
        WP3d = torch.empty((n_win, len(s)), dtype=torch.float64, device=dev)
        hdt = _native.WK_F64 if self._hist.dtype == torch.float64 else _native.WK_F32
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.wk_wake_potential(
            self._hist.data_ptr(), hdt, self._hist.shape[-1], self._hist.shape[1],
            win.data_ptr(), n_win, int(carry), zt.data_ptr(), dzt.data_ptr(), len(z),
            int(self.skip_cells), st.data_ptr(), len(s), order.data_ptr(), int(nt),
            float(self.v), float(zmin), float(zmax), float(self.t[0]), float(self.ti),
            float(dt), float(self.q * 1e12), int(self.counter_moving), WP3d.data_ptr(), stream)
        _native.check(rc, "wk_wake_potential")
        self.s = s
        return WP3d

    # -------------------------------------------------------------- solve
    def solve(self, compute_plane=None, **kwargs):
        cp = (compute_plane or self.compute_plane).lower()
        for k, v in kwargs.items():
            setattr(self, k, v)
        if cp in ("both", "transverse"):
            self.calc_long_WP_3d()
            self.calc_trans_WP()
            self.calc_long_Z()
            self.calc_trans_Z()
        elif cp == "longitudinal":
            self.calc_long_WP()
            self.calc_long_Z()

    def calc_long_WP_3d(self, **kwargs):
        if self._hist_1d:
            raise ValueError("the Ez history holds the test line only (compute_plane="
                             "'longitudinal'); the 3d wake needs the 3x3 window")
        WP3d = self._wp(9, carry=True)
        self._WP3d_dev = WP3d
        self.WP_3d = WP3d.cpu().numpy().reshape(3, 3, -1)
        self.WP = self.WP_3d[1, 1, :]
        self._WP_dev = WP3d[4]

    def calc_long_WP(self, **kwargs):
        if not self._hist_1d:
            raise ValueError("calc_long_WP needs the history of compute_plane='longitudinal'")
        if self.skip_cells != 0:
            # upstream assigns the full Nz line into nz rows (wakeSolver.py:390-392)
            raise ValueError("could not broadcast input array: skip_cells with a 1-D history")
        WP = self._wp(1, carry=False)
        self._WP_dev = WP[0]
        self.WP = WP[0].cpu().numpy()

    # s axes longer than this take the O(ns) double-double scan instead of
    # the per-sample pairwise sums of upstream's np.sum (O(ns^2))
    TRANS_PAIRWISE_MAX = 65536

    def calc_trans_WP(self, **kwargs):
        lib = _native.lib()
        ds = self.s[2] - self.s[1]
        dxf, dyf = np.diff(self.xf), np.diff(self.yf)
        ns = len(self.s)
        dev = self._WP3d_dev.device
        WPx = torch.empty(ns, dtype=torch.float64, device=dev)
        WPy = torch.empty(ns, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if ns > self.TRANS_PAIRWISE_MAX or kwargs.get("scan", False):
            nb = int(lib.wk_trans_wake_scan_scratch_bytes(ns))
            scratch = torch.empty(max(nb, 16), dtype=torch.uint8, device=dev)
            rc = lib.wk_trans_wake_scan(self._WP3d_dev.data_ptr(), ns, float(ds),
                                        float(dxf[0] + dxf[1]), float(dyf[0] + dyf[1]),
                                        WPx.data_ptr(), WPy.data_ptr(), scratch.data_ptr(),
                                        scratch.numel(), stream)
            _native.check(rc, "wk_trans_wake_scan")
        else:
            rc = lib.wk_trans_wake(self._WP3d_dev.data_ptr(), ns, float(ds),
                                   float(dxf[0] + dxf[1]), float(dyf[0] + dyf[1]),
                                   WPx.data_ptr(), WPy.data_ptr(), stream)
            _native.check(rc, "wk_trans_wake")
        self._WPx_dev, self._WPy_dev = WPx, WPy
        self.WPx, self.WPy = WPx.cpu().numpy(), WPy.cpu().numpy()

    def calc_lambdas_analytic(self, **kwargs):
        self.lambdas = (1 / (self.sigmaz * np.sqrt(2 * np.pi))
                        * np.exp(-(self.s ** 2) / (2 * self.sigmaz ** 2)))

    def calc_lambdas(self, **kwargs):
        chargedist = self.chargedist
        if isinstance(chargedist, dict):
            keys = list(chargedist.keys())
            z, chargedist = chargedist[keys[0]], chargedist[keys[1]]
        elif len(self.zf) == len(chargedist):
            z = self.zf
        else:
            raise ValueError("Dimension error: check input dimensions")
        self.lambdas = np.interp(self.s, z, np.asarray(chargedist) / self.q)

    def _bins(self, signals, samples, fmax):
        """DFT bins 0 <= f < fmax of np.fft.fft(x, n=N) for host/device signals."""
        lib = _native.lib()
        ds = np.mean(self.s[1:] - self.s[:-1])
        fmax = self.fmax if fmax is None else fmax
        N = int((self.v / ds) // fmax * samples)
        ffft = np.fft.fftfreq(N, ds / self.v)
        mask = np.logical_and(ffft >= 0, ffft < fmax)
        nb = int(mask.sum())
        if nb and not mask[:nb].all():
            raise RuntimeError("kept DFT bins are not the leading bins")
        ns = len(self.s)
        dev = self._WP_dev.device
        x = torch.stack([torch.as_tensor(sg, dtype=torch.float64, device=dev) for sg in signals])
        x = x.contiguous()
        out = torch.empty((len(signals), nb, 2), dtype=torch.float64, device=dev)
        rc = lib.wk_dft_bins(x.data_ptr(), len(signals), ns, N, nb, out.data_ptr(),
                             torch.cuda.current_stream(dev).cuda_stream)
        _native.check(rc, "wk_dft_bins")
        return ds, ffft[mask], torch.view_as_complex(out)

    def calc_long_Z(self, samples=1001, fmax=None, **kwargs):
        if self.lambdas is None and self.chargedist is not None:
            self.calc_lambdas()
        elif self.lambdas is None:
            self.calc_lambdas_analytic()
        lam = torch.as_tensor(self.lambdas * self.v, dtype=torch.float64, device=self._WP_dev.device)
        ds, f, X = self._bins([lam, self._WP_dev * 1e12], samples, fmax)
        lambdaf = X[0] * ds
        WPf = X[1] * ds
        self.f = f
        self.Z = (-WPf / lambdaf).cpu().numpy()
        self.lambdaf = lambdaf.cpu().numpy()
        self._lambdaf_dev = lambdaf

    def calc_trans_Z(self, samples=1001, fmax=None):
        lam = torch.as_tensor(self.lambdas * self.v, dtype=torch.float64, device=self._WP_dev.device)
        ds, f, X = self._bins([lam, self._WPx_dev * 1e12, self._WPy_dev * 1e12], samples, fmax)
        lambdaf = X[0] * ds
        self.Zx = (1j * (X[1] * ds) / lambdaf).cpu().numpy()
        self.Zy = (1j * (X[2] * ds) / lambdaf).cpu().numpy()
        self.fx = self.fy = f

    # --------------------------------------------------- static FFT helpers
    @staticmethod
    def calc_impedance_from_wake(wake, s=None, t=None, fmax=None, samples=None, verbose=True):
        """Impedance of a wake function by FFT (upstream wakeSolver.py:
        1182-1250), on the host.  ``wake`` is the wake or a list [t, wake];
        the time axis may also come as ``s`` (m, t = s/c) or ``t`` (s).  With
        ``fmax`` the wake is first resampled on a 1/(2 fmax) grid, else fmax
        = 1/dt.  Returns [f, Z]: the bins 0 <= f < fmax of the DFT (2*samples
        points when ``samples`` is given) scaled by 2/len(wake)."""
        if type(wake) is list:
            t, wake = wake[0], wake[1]
        if s is not None:
            t = s / c_light
        elif t is None:
            raise AttributeError('Provide time data through parameter "t" [s] or "s" [m]')
        t = np.asarray(t)
        wake = np.asarray(wake)
        dt = np.mean(t[1:] - t[:-1])
        if fmax is not None:
            grid = np.arange(t.min(), t.max(), 1 / fmax / 2)
            wake = np.interp(grid, t, wake)
            dt = np.mean(grid[1:] - grid[:-1])
        else:
            fmax = 1 / dt
        spec = np.fft.fft(wake, n=2 * samples) if samples is not None else np.fft.fft(wake)
        freqs = np.fft.fftfreq(len(spec), dt)
        keep = np.logical_and(freqs >= 0, freqs < fmax)
        f = freqs[keep]
        Z = spec[keep] / len(wake) * 2
        if verbose:
            print(f"* Number of samples = {len(f)}")
            print(f"* Maximum frequency = {f.max()} Hz")
            print(f"* Maximum resolution = {np.mean(f[1:] - f[:-1])} Hz")
        return [f, Z]

    @staticmethod
    def calc_wake_from_impedance(impedance, f=None, tmax=None, samples=None, pad=0,
                                 verbose=True):
        """Wake function of an impedance (upstream wakeSolver.py:1252-1311),
        on the host.  ``impedance`` is Z or a list [f, Z] (a length-2 argument
        is read as the list, as upstream does).  With ``tmax`` Z is resampled
        on a 1/tmax frequency grid, else tmax = 1/df.  The wake is the real
        part of -FFT(Z) (``samples`` points) rolled back by one sample, on
        t = linspace(0, tmax, len(wake)); ``pad`` is accepted and unused, as
        upstream.  Returns [t, wake]."""
        if len(impedance) == 2:
            f, Z = impedance[0], impedance[1]
        elif f is None:
            raise AttributeError('Provide frequency data through parameter "f"')
        else:
            Z = impedance
        f = np.asarray(f)
        Z = np.asarray(Z)
        df = np.mean(f[1:] - f[:-1])
        if tmax is not None:
            Z = np.interp(np.arange(f.min(), f.max(), 1 / tmax), f, Z)
        else:
            tmax = 1 / df
        wake = np.roll(np.real(-1 * np.fft.fft(Z, n=samples)), -1)
        t = np.linspace(0, tmax, len(wake))
        if verbose:
            print(f"* Number of samples = {len(t)}")
            print(f"* Maximum time = {t.max()} s")
            print(f"* Maximum resolution = {np.mean(t[1:] - t[:-1])} s")
        return [t, wake]
