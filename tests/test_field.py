"""Field storage and indexing (upstream wakis/field.py) against fixtures
written by the upstream Field (tests/golden/field_cases.npz): component
matrices, |F|, tuple / integer / slice reads and writes, arithmetic with
scalars, flat arrays, (Nx, Ny, Nz) matrices and fields, compute_ijk.  The
field lives on the CPU here; every value must match bit for bit."""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cases  # noqa: E402


@pytest.fixture(scope="module")
def ref(golden_dir):
    return np.load(os.path.join(golden_dir, "field_cases.npz"))


def _field(arr):
    from wakis_b200.field import Field
    Nx, Ny, Nz = cases.FIELD_CASE["shape"]
    f = Field(Nx, Ny, Nz, use_gpu=False)
    f.fromarray(arr.copy())
    return f


def test_matrices_and_abs(ref):
    a, _, _, _ = cases.field_inputs()
    f = _field(a)
    for d in "xyz":
        assert np.array_equal(f.to_matrix(d).numpy(), ref[f"mat_{d}"])
    assert np.array_equal(f.get_abs(), ref["abs"])
    assert np.array_equal(f.get_abs(as_matrix=False), ref["abs_flat"])
    assert [f.compute_ijk(n) for n in cases.FIELD_IJK] == [tuple(r) for r in ref["ijk"]]


def test_reads(ref):
    a, _, _, _ = cases.field_inputs()
    f = _field(a)
    for name, key in cases.FIELD_READS:
        assert np.array_equal(np.asarray(f[key]), ref[name]), name


def test_writes(ref):
    a, _, m, _ = cases.field_inputs()
    f = _field(a)
    for key, val in cases.FIELD_WRITES:
        if isinstance(val, str) and val == "arange5":
            val = np.arange(5.0)
        elif isinstance(val, str) and val == "plane_y4":
            val = m[:, :, 4]
        f[key] = val
    assert np.array_equal(f.numpy(), ref["after_writes"])


def test_block_setters():
    a, b, m, _ = cases.field_inputs()
    f = _field(a)
    f.field_y = m                      # matrix: Fortran-order component
    f.field_z = b[:f.N]                # flat
    assert np.array_equal(f.to_matrix("y").numpy(), m)
    assert np.array_equal(f.field_z.numpy(), b[:f.N])


def test_arithmetic(ref):
    a, b, m, flat = cases.field_inputs()
    f, g = _field(a), _field(b)
    assert np.array_equal((f * 2.5).numpy(), ref["mul_scalar"])
    assert np.array_equal((f * m).numpy(), ref["mul_matrix"])
    assert np.array_equal((f * flat).numpy(), ref["mul_flat"])
    assert np.array_equal((f + g).numpy(), ref["add_field"])
    assert np.array_equal((f + m).numpy(), ref["add_matrix"])
    assert np.array_equal((f + flat).numpy(), ref["add_flat"])
