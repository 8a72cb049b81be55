"""The streamed wake integration (wakesolve(history="stream")) and the
O(ns) transverse scan, on the device.

The streamed form adds every chunk of captured steps into the wake-potential
sums as soon as the chunk completes, so a run needs memory for the s samples
only, not for the [window][k][step] history; its sums run in another order
than upstream's, so it is compared within the wake tolerance (1e-10) with
upstream's fixtures and with the full-history form (value-for-value
identical to upstream) of the same run.
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cases  # noqa: E402
from helpers import b200_wake_case, rel_err  # noqa: E402

WAKE_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("chunk", [256, 7])
@pytest.mark.parametrize("idx", range(len(cases.WAKE_CASES)))
def test_streamed_wakesolve_matches_upstream(idx, chunk, golden_dir, monkeypatch):
    from wakis_b200.solverFIT3D import SolverFIT3D
    monkeypatch.setattr(SolverFIT3D, "STREAM_CHUNK", chunk)
    g = np.load(os.path.join(golden_dir, "wake_cases.npz"))
    c = cases.WAKE_CASES[idx]
    s, w = b200_wake_case(c)
    s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"], history="stream")
    assert w._hist is None and w._stream is not None
    assert s.Nt == int(g[f"c{idx}_Nt"])
    names = ["WP", "Z"]
    if c["compute_plane"] == "both":
        names += ["WP_3d", "WPx", "WPy", "Zx", "Zy"]
    tol = WAKE_TOL if c["dtype"] == "float64" else 1e-5
    for n in names:
        assert rel_err(getattr(w, n), g[f"c{idx}_{n}"]) <= tol, (n, rel_err(getattr(w, n),
                                                                           g[f"c{idx}_{n}"]))


def _cavity_runs(wakelength, history_pair=("full", "stream")):
    from wakis_b200 import workloads
    out = []
    for h in history_pair:
        _, w, s = workloads.build_b200("cavity_40")
        s.wakesolve(wakelength=wakelength, history=h)
        out.append((s, w))
    return out


def test_streamed_equals_full_history_cavity_40():
    (sa, wa), (sb, wb) = _cavity_runs(0.5)
    assert sa.Nt == sb.Nt == 1896
    for n in ("WP", "WP_3d", "WPx", "WPy", "Z", "Zx", "Zy"):
        assert rel_err(getattr(wb, n), getattr(wa, n)) <= 1e-12, n


def test_streamed_equals_full_beyond_1e5_steps():
    """More than 10^5 steps: upstream's '#%05d' keys then sort out of step
    order and its sums read the steps at the sorted positions; the streamed
    form places each step at its key's position.  100,500 steps of the
    40x40x80 cavity, full history (0.6 GB) against streamed."""
    from wakis_b200 import workloads
    _, w0, s0 = workloads.build_b200("cavity_40")
    z = s0.z
    wl = (100500.5 * float(s0.dt) * w0.v) - w0.ti * w0.v - (z.max() - z.min())
    (sa, wa), (sb, wb) = _cavity_runs(wl)
    assert sa.Nt == sb.Nt and sa.Nt > 100000
    assert len(wa.s) > wa.TRANS_PAIRWISE_MAX        # the transverse scan runs in both
    for n in ("WP", "WP_3d", "WPx", "WPy", "Z"):
        assert rel_err(getattr(wb, n), getattr(wa, n)) <= 1e-12, n


def test_transverse_scan_equals_pairwise():
    """The O(ns) double-double scan against the per-sample pairwise sums
    (numpy's order) on the same WP_3d."""
    from wakis_b200 import workloads
    _, w, s = workloads.build_b200("cavity_40")
    s.wakesolve(wakelength=0.5)
    WPx, WPy = w.WPx.copy(), w.WPy.copy()
    w.calc_trans_WP(scan=True)
    assert rel_err(w.WPx, WPx) <= 1e-12 and rel_err(w.WPy, WPy) <= 1e-12
