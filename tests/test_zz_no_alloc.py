"""wk_trans_wake_scan_noalloc: the transverse-wake scan with its segment
sums in scratch built into the library, for callers that cannot give this
library device memory (their device memory is reserved by another
allocator or a fixed budget).  Checked through the C ABI against
wk_trans_wake_scan with caller scratch, on two calls in a row with
different inputs (the built-in scratch keeps the previous call's sums).

Collected last (file name), so that a run stopping at the first failure has
run every other test first; it needs nothing from the other tests.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _with_scratch(lib, wp, ns, ds, dx, dy, stream):
    nb = int(lib.wk_trans_wake_scan_scratch_bytes(ns))
    scratch = torch.empty(max(nb, 16), dtype=torch.uint8, device="cuda")
    wx = torch.empty(ns, dtype=torch.float64, device="cuda")
    wy = torch.empty_like(wx)
    rc = lib.wk_trans_wake_scan(wp.data_ptr(), ns, ds, dx, dy, wx.data_ptr(), wy.data_ptr(),
                                scratch.data_ptr(), scratch.numel(), stream)
    assert rc == 0, lib.wk_last_error()
    return wx, wy


def test_no_alloc_scan_equals_scan_with_caller_scratch():
    from wakis_b200 import _native
    lib = _native.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(5)
    for ns, ds, dx, dy in ((300000, 2.5e-4, 2.5e-3, 2.5e-3), (5000, 1e-3, 1e-3, 2e-3)):
        wp = torch.randn((9, ns), generator=g, dtype=torch.float64, device="cuda")
        ref_x, ref_y = _with_scratch(lib, wp, ns, ds, dx, dy, stream)
        wx = torch.full((ns,), float("nan"), dtype=torch.float64, device="cuda")
        wy = torch.full_like(wx, float("nan"))
        rc = lib.wk_trans_wake_scan_noalloc(wp.data_ptr(), ns, ds, dx, dy, wx.data_ptr(),
                                            wy.data_ptr(), stream)
        assert rc == 0, lib.wk_last_error()
        torch.cuda.synchronize()
        for got, ref in ((wx, ref_x), (wy, ref_y)):
            a, b = got.cpu().numpy(), ref.cpu().numpy()
            assert np.all(np.isfinite(a))
            assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b))


def test_no_alloc_scan_rejects_sizes_above_its_maximum():
    from wakis_b200 import _native
    lib = _native.lib()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.wk_trans_wake_scan_noalloc(x.data_ptr(), 2**31 - 1, 1.0, 1.0, 1.0, x.data_ptr(),
                                        x.data_ptr(), None)
    assert rc == 5            # WK_E_RANGE, nothing launched
    assert b"maximum" in lib.wk_last_error()
