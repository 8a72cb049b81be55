"""Frequency-domain field monitor (upstream wakis/field_monitors.py).

``FieldMonitor(frequencies)`` accumulates, for every monitored frequency f,
sum_n E(t_n) exp(-2j pi f t_n) with t_n = n*dt over the whole grid
(upstream field_monitors.py:60-107).  The accumulators live on the device in
the flat field order; one kernel launch per ``update`` reads E once for all
frequencies (``wk_field_monitor``).  ``get_components`` returns
(n_freq, Nx, Ny, Nz) complex128 views indexed [f, i, j, k] as upstream's
arrays are.
"""

from typing import Sequence

import numpy as np
import torch

from . import _native


class FieldMonitor:
    def __init__(self, frequencies: Sequence[float]):
        self.frequencies = np.array(frequencies)
        self.time_index = 0
        self.dt = None
        self.shape = None
        self._acc = None
        self.xp = None
        self.Ex_acc = self.Ey_acc = self.Ez_acc = None

    def update(self, E, dt):
        """Add the snapshot of the Field E at t = time_index * dt."""
        if self.dt is None:
            self.dt = dt
            self.shape = (E.Nx, E.Ny, E.Nz)
            self.xp = getattr(E, "xp", torch)
            nf = len(self.frequencies)
            self._N = E.Nx * E.Ny * E.Nz
            self._acc = torch.zeros((nf, 3, self._N), dtype=torch.complex128,
                                    device=E.array.device)
            views = [self._acc[:, d].view(nf, E.Nz, E.Ny, E.Nx).permute(0, 3, 2, 1)
                     for d in range(3)]
            self.Ex_acc, self.Ey_acc, self.Ez_acc = views
        t = self.time_index * self.dt
        ph = np.exp(-2j * np.pi * self.frequencies * t)
        phases = torch.as_tensor(np.stack([ph.real, ph.imag], axis=1).ravel(),
                                 dtype=torch.float64, device=self._acc.device)
        arr = E.array
        dt_code = _native.WK_F64 if arr.dtype == torch.float64 else _native.WK_F32
        lib = _native.lib()
        rc = lib.wk_field_monitor(arr.data_ptr(), dt_code, self._N, phases.data_ptr(),
                                  len(self.frequencies), torch.view_as_real(self._acc).data_ptr(),
                                  torch.cuda.current_stream(self._acc.device).cuda_stream)
        _native.check(rc, "wk_field_monitor")
        self.time_index += 1

    def get_components(self):
        return {"Ex": self.Ex_acc, "Ey": self.Ey_acc, "Ez": self.Ez_acc}
