"""ctypes binding of the C-ABI library ``libwakis_b200.so``.

The library is built in-tree (``wakis_b200/build.py``) and loaded from the
package directory.  There is no fallback: if the library is missing, every
entry point that needs it raises ``ImportError`` naming the build command.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwakis_b200.so")

WK_F64, WK_F32, WK_F32C = 0, 1, 2
WK_J_ZERO, WK_J_SIGMA_E, WK_J_ARRAY = 0, 1, 2
WK_KERNEL_AUTO, WK_KERNEL_CELL, WK_KERNEL_TWOPASS, WK_KERNEL_TMA = 0, 1, 4, 6
WK_BATCH_PERSISTENT, WK_BATCH_PHASES = 0, 1

_vp = ctypes.c_void_p
_i = ctypes.c_int
_ll = ctypes.c_longlong
_d = ctypes.c_double


class FitDesc(ctypes.Structure):
    """Mirror of ``wk_fit_desc`` in include/wakis_b200.h."""

    _fields_ = [
        ("Nx", _i), ("Ny", _i), ("Nz", _i), ("dtype", _i),
        ("E", _vp * 2), ("H", _vp * 2), ("par", _i), ("J", _vp),
        ("j_mode", _i), ("use_conductivity", _i),
        ("mat_id", _vp), ("id_bytes", _i), ("mat_table", _vp), ("n_mat", _i),
        ("Lx", _vp), ("Ly", _vp), ("Lz", _vp), ("tLx", _vp), ("tLy", _vp), ("tLz", _vp),
        ("iAx", _vp), ("iAy", _vp), ("iAz", _vp), ("itAx", _vp), ("itAy", _vp), ("itAz", _vp),
        ("pec_face", _i * 6), ("pmc_face", _i * 6), ("has_pec", _i), ("has_pmc", _i),
        ("h_sum_desc", _i), ("dt", _d), ("dt_is_f32", _i),
        ("beam_on", _i), ("ixs", _i), ("iys", _i),
        ("b_qv", _d), ("b_v", _d), ("b_s0", _d), ("b_c0", _d), ("b_two_sig2", _d),
        ("b_dx", _d), ("b_dy", _d), ("zc", _vp),
        ("line_on", _i), ("line_step0", _ll), ("line_nsteps", _ll), ("line", _vp),
        ("cap_on", _i), ("cap_i0", _i), ("cap_j0", _i), ("cap_ni", _i), ("cap_nj", _i),
        ("cap_nt", _ll), ("cap_step0", _ll), ("cap", _vp), ("status", _vp),
        ("kernel", _i), ("tile_rows", _i), ("tile_planes", _i),
        ("Ec", _vp * 2), ("Hc", _vp * 2),
        ("step_dev", _vp),
        ("faces_clean", _i),
        ("wait_ns", _ll),
        ("steps_per_launch", _i),
        ("comp_stencil", _i),
    ]


class BatchPlan(ctypes.Structure):
    """Mirror of ``wk_batch_plan`` in include/wakis_b200.h."""

    _fields_ = [
        ("workspace", _vp), ("workspace_bytes", _ll), ("n_inst", _i), ("n_items", _i * 2),
        ("grid", _i), ("smem", _i), ("variant", _i), ("device", _i), ("offsets", _ll * 4),
        ("n_parts", _i * 5), ("form", _i),
    ]


_SIGS = {
    "wk_version": (_i, []),
    "wk_last_error": (ctypes.c_char_p, []),
    "wk_zero_ghosts": (_i, [ctypes.POINTER(FitDesc), _vp]),
    "wk_fit_step": (_i, [ctypes.POINTER(FitDesc), _i, _ll, _vp]),
    "wk_fit_step_split": (_i, [ctypes.POINTER(FitDesc), _i, _ll, _vp]),
    "wk_fit_step_timed": (_i, [ctypes.POINTER(FitDesc), _i, _ll, _vp,
                               ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_i)]),
    "wk_sigma_e": (_i, [ctypes.POINTER(FitDesc), _vp, _vp]),
    "wk_counter_add": (_i, [_vp, _ll, _vp]),
    "wk_source_write": (_i, [_vp, _i, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp,
                             _ll, _vp, _ll, _vp]),
    "wk_batch_workspace_bytes": (_ll, [_vp, _i]),
    "wk_batch_prepare": (_i, [_vp, _i, _ll, _vp, _ll, ctypes.POINTER(BatchPlan), _vp]),
    "wk_batch_run": (_i, [ctypes.POINTER(BatchPlan), _i, _ll, _vp, _ll, _vp]),
    "wk_field_monitor": (_i, [_vp, _i, _ll, _vp, _i, _vp, _vp]),
    "wk_adj_h": (_i, [_i, _vp, _vp, _vp, _ll, _vp, _vp, ctypes.c_double, _vp, _vp, _vp]),
    "wk_adj_e": (_i, [_i, _vp, _vp, _vp, _ll, _vp, _vp, _vp, _vp, _vp]),
    "wk_adj_grad": (_i, [_i, _vp, _ll, _ll, _vp, _vp, _vp, _vp, _vp, _i, ctypes.c_double,
                         _vp, _vp, _vp]),
    "wk_adj_h_fit": (_i, [ctypes.POINTER(FitDesc), _i, _vp, _vp, _vp, _vp, _vp]),
    "wk_adj_e_fit": (_i, [ctypes.POINTER(FitDesc), _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "wk_adj_factors": (_i, [ctypes.POINTER(FitDesc), _i, _vp, _vp, _vp]),
    "wk_wake_potential": (_i, [_vp, _i, _ll, _i, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _i,
                               _vp, _ll, _d, _d, _d, _d, _d, _d, _d, _i, _vp, _vp]),
    "wk_trans_wake": (_i, [_vp, _i, _d, _d, _d, _vp, _vp, _vp]),
    "wk_dft_bins": (_i, [_vp, _i, _ll, _ll, _i, _vp, _vp]),
    "wk_read_status": (_i, [_vp, _i, _vp]),
    "wk_wake_accumulate": (_i, [_vp, _i, _ll, _i, _ll, _i, _vp, _i, _vp, _vp, _i, _i, _vp, _i,
                                _vp, _ll, _d, _d, _d, _d, _d, _d, _i, _vp, _vp]),
    "wk_wake_finalize": (_i, [_vp, _i, _i, _i, _d, _vp, _vp]),
    "wk_trans_wake_scan_scratch_bytes": (_ll, [_i]),
    "wk_trans_wake_scan": (_i, [_vp, _i, _d, _d, _d, _vp, _vp, _vp, _ll, _vp]),
    "wk_trans_wake_scan_noalloc": (_i, [_vp, _i, _d, _d, _d, _vp, _vp, _vp]),
}

EXPORTED = tuple(_SIGS)

_lib = None


def lib():
    """Load the library once; raise ImportError when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"wakis_b200 native library not found at {LIB_PATH}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`python -m wakis_b200.build`")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


class NativeError(RuntimeError):
    pass


WK_E_TIMEOUT = 7


def read_status(status, stream, what="step", reset=True):
    """Wait for `stream` and read the device status word ``status`` (a
    one-element int32 CUDA tensor) that the step kernels set when a tile
    load did not arrive within its wait bound; raise NativeError naming
    `what` when it is set (and clear it with ``reset``)."""
    rc = lib().wk_read_status(status.data_ptr(), int(bool(reset)), stream)
    if rc != 0:
        msg = lib().wk_last_error().decode(errors="replace")
        raise NativeError(f"{what}: {msg}")


def check(rc, what):
    """Map a non-zero ABI status to an exception carrying the library message."""
    if rc != 0:
        msg = lib().wk_last_error().decode(errors="replace")
        if rc > 0:
            raise ValueError(f"{what}: {msg} (status {rc})")
        raise NativeError(f"{what}: {msg} (CUDA error {-rc})")
