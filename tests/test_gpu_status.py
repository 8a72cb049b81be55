"""The status word of the TMA step kernels (device, through the C ABI).

Every mbarrier wait of the TMA step loops is bounded (a %globaltimer
deadline).  ``wk_fit_desc.wait_ns < 0`` makes the first wait of each block
give up at once, without any fault: the block records the timeout in the
status word, waits (with the default bound) for the tile loads it issued and
returns.  These tests run that path and check that the host sees it:
``wk_read_status`` returns WK_E_TIMEOUT, the Python calls that wait for the
device raise, and the context stays usable afterwards.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pair(prec):
    from wakis_b200 import workloads
    _, _, a = workloads.build_b200("cavity_40", precision=prec)
    _, _, b = workloads.build_b200("cavity_40", precision=prec)
    a.kernel = b.kernel = "tma"
    return a, b


@pytest.mark.parametrize("prec", [None, "fp32c"])
def test_timed_out_wait_is_reported_through_the_abi(prec):
    from wakis_b200 import _native
    a, _ = _pair(prec)
    lib = _native.lib()
    a._first_step()
    a._desc.wait_ns = -1
    d = a._step_desc()
    st = a._stream()
    assert lib.wk_fit_step(d, 1, 0, st) == 0
    a._par ^= 1
    rc = lib.wk_read_status(ctypes.c_void_p(a._status.data_ptr()), 1, st)
    assert rc == _native.WK_E_TIMEOUT
    assert b"gave up waiting" in lib.wk_last_error()
    # cleared by the read, and the next read of a clean run is WK_OK
    assert int(a._status.item()) == 0
    a._desc.wait_ns = 0
    assert lib.wk_fit_step(a._step_desc(), 1, 1, st) == 0
    a._par ^= 1
    assert lib.wk_read_status(ctypes.c_void_p(a._status.data_ptr()), 1, st) == 0


@pytest.mark.parametrize("prec", [None, "fp32c"])
def test_run_raises_on_timeout_and_context_stays_usable(prec):
    from wakis_b200.sources import Beam
    a, b = _pair(prec)
    a._desc.wait_ns = -1
    with pytest.raises(RuntimeError, match="gave up waiting"):
        a.run(3)
    assert int(a._status.item()) == 0
    # a fresh run on the same context, with the default bound, equals a
    # solver that never timed out
    a._desc.wait_ns = 0
    bp = Beam(q=1e-9, sigmaz=0.01, beta=1.0).params(a)
    for s in (a, b):
        s.reset_fields()
        s.step_0, s.nstep = True, 0
        s._advance(40, 0, beam=bp)
        s.check_status()
    if prec is None:
        assert np.array_equal(a.E.numpy(), b.E.numpy())
        assert np.array_equal(a.H.numpy(), b.H.numpy())
    else:
        for f in ("_E", "_H", "_Ec", "_Hc"):
            assert torch.equal(getattr(a, f)[a._par], getattr(b, f)[b._par])
    assert np.abs(b.E.numpy()).max() > 0


def test_wakesolve_raises_on_timeout():
    from wakis_b200 import workloads
    _, _, s = workloads.build_b200("cavity_40")
    s._desc.wait_ns = -1
    with pytest.raises(RuntimeError, match="wakesolve"):
        s.wakesolve(wakelength=0.01)
