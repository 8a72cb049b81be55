"""WakeSolver's static FFT helpers on the host (upstream
tests/test_004_wakes_and_impedances.py): a sinusoidal wake survives two
wake -> impedance -> wake round trips within 1, and both impedances peak at
the wake's amplitude and frequency."""

import numpy as np
import pytest

from wakis_b200.wakeSolver import WakeSolver as wk

FR, AMP = 0.5e9, 100.0


@pytest.fixture(scope="module")
def sin_wake():
    t = np.linspace(0, 100 * 1e-9, 3000)
    return t, AMP * np.sin(2 * np.pi * FR * t)


def test_sin_wake_round_trips(sin_wake):
    t, wake = sin_wake
    f, Z = wk.calc_impedance_from_wake([t, wake], verbose=False)
    tt, w2 = wk.calc_wake_from_impedance([f, Z], samples=3000, verbose=False)
    ff, Zz = wk.calc_impedance_from_wake([tt, w2], verbose=False)
    ttt, w3 = wk.calc_wake_from_impedance([ff, Zz], samples=3000, verbose=False)
    assert np.allclose(wake, w2, atol=1)
    assert np.allclose(wake, w3, atol=1)


def test_sin_impedance_peak(sin_wake):
    t, wake = sin_wake
    f, Z = wk.calc_impedance_from_wake([t, wake], verbose=False)
    tt, w2 = wk.calc_wake_from_impedance([f, Z], samples=3000, verbose=False)
    ff, Zz = wk.calc_impedance_from_wake([tt, w2], verbose=False)
    assert np.allclose(np.max(np.abs(Z)), AMP, atol=1)
    assert np.allclose(np.max(np.abs(Zz)), AMP, atol=1)
    assert np.allclose(f[np.argmax(Z)], FR, atol=1e6)
    assert np.allclose(ff[np.argmax(Zz)], FR, atol=1e6)


def test_time_axis_required():
    with pytest.raises(AttributeError):
        wk.calc_impedance_from_wake(np.ones(8))
    with pytest.raises(AttributeError):
        wk.calc_wake_from_impedance(np.ones(8))
