"""Host logic on the CPU: compact coefficients against the oracle's dense
material fields and sparse operators, the kernels' update formula (numpy
emulation) against the oracle's mat-vec step, geometry masks."""

import os
import tempfile

import numpy as np
import pytest

import cases
import stencil_emulator as emu
from helpers import oracle_step_case
from wakis_b200 import coefficients, geometry
from wakis_b200.gridFIT3D import GridFIT3D


def _coef(c):
    g = GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
    if c["solids"]:
        masks = cases.step_masks(c)
        for k, mat in c["solids"].items():
            g.add_solid(k, masks[k], mat)
    return coefficients.build(g, c["bc_low"], c["bc_high"], dtype=np.dtype(c["dtype"]).type,
                              bg=c["bg"], use_stl=bool(c["solids"]), use_sibc=False,
                              n_pml=c["n_pml"])


def _valid_cases():
    out = []
    for i, c in enumerate(cases.STEP_CASES):
        try:
            oracle_step_case(c)
        except ValueError:
            continue
        out.append(i)
    return out


VALID = _valid_cases()


@pytest.mark.parametrize("idx", VALID)
def test_coefficients_match_oracle(idx):
    c = cases.STEP_CASES[idx]
    o = oracle_step_case(c)
    k = _coef(c)
    assert k.dt == o.dt and type(k.dt) is type(o.dt)
    ie, im, sg = coefficients.dense_materials(k)
    assert np.array_equal(ie, o.ieps) and np.array_equal(im, o.imu)
    assert np.array_equal(sg, o.sigma)
    assert k.use_conductivity == o.use_conductivity
    assert k.h_sum_desc == ((o.pec_mask is not None) + (o.pmc_mask is not None) == 1)


@pytest.mark.parametrize("idx", VALID)
def test_emulated_step_is_bitwise_equal_to_oracle(idx):
    c = cases.STEP_CASES[idx]
    o = oracle_step_case(c)
    k = _coef(c)
    E0, H0 = cases.initial_fields(c, o.N)
    o.E[:], o.H[:] = E0, H0
    o.zero_ghosts()
    E, H = o.E.copy(), o.H.copy()
    J = np.zeros_like(E)
    o.step_0 = False
    for _ in range(3):
        Jin = o.J.copy()
        o.one_step()
        Hn = emu.h_update(k, E, H, k.dt)
        assert np.array_equal(Hn, o.H)
        En = emu.e_update(k, E, Hn, Jin, k.dt)
        assert np.array_equal(En, o.E)
        E, H = En, Hn


def test_abc_views_reference_semantics_documented():
    # both-ends ABC on one axis makes upstream drop the low-face snapshot;
    # the flags still fold the high-face metric copy (boundaries.py:152-181)
    pec, pmc, has_pec, has_pmc = coefficients.boundary_flags(["pec", "pec", "abc"],
                                                             ["pec", "pec", "abc"])
    assert pec == [0, 0, 0, 0, 1, 1] and has_pec and not has_pmc


def _cube_stl(path, lo, hi):
    # 12 triangles of an axis-aligned box, ASCII STL
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]])
    faces = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
             (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6), (3, 0, 4), (3, 4, 7)]
    with open(path, "w") as f:
        f.write("solid box\n")
        for a, b, cc in faces:
            f.write(" facet normal 0 0 0\n  outer loop\n")
            for p in (a, b, cc):
                f.write("   vertex %.9e %.9e %.9e\n" % tuple(v[p]))
            f.write("  endloop\n endfacet\n")
        f.write("endsolid box\n")


def test_stl_voxeliser_matches_analytic_box():
    x = np.linspace(-0.01, 0.01, 21)
    y = np.linspace(-0.01, 0.01, 17)
    z = np.linspace(-0.02, 0.02, 33)
    lo, hi = (-0.0043, -0.0051, -0.0077), (0.0061, 0.0037, 0.0093)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "box.stl")
        _cube_stl(p, lo, hi)
        m_stl = geometry.cell_mask(geometry.STLSolid(p), x, y, z)
    m_box = geometry.cell_mask(geometry.Box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]), x, y, z)
    assert m_stl.sum() > 0 and np.array_equal(m_stl, m_box)


def test_surface_mask_marks_both_sides_of_interface():
    m = np.zeros((6, 6, 6), bool)
    m[2:4, 2:4, 2:4] = True
    s = geometry.surface_mask(m)
    assert s[2, 2, 2] and s[1, 2, 2] and not s[0, 0, 0]


def test_lean_interior_formulas_equal_oracle():
    """The kernels' interior-cell formulas (one coefficient per metric,
    leading +0 dropped) give the oracle's values on interior cells."""
    c = dict(cases.STEP_CASES[2])
    c.update(shape=(9, 8, 10))
    for bc, mats in ((["pec"] * 3, c["solids"]), (["periodic"] * 3, {})):
        cc = dict(c, bc_low=bc, bc_high=bc, solids=mats)
        for dtype in ("float64", "float32"):
            cc["dtype"] = dtype
            o = oracle_step_case(cc)
            k = _coef(cc)
            E0, H0 = cases.initial_fields(cc, o.N)
            o.E[:], o.H[:] = E0, H0
            o.zero_ghosts()
            o.step_0 = False
            E, H, J = o.E.copy(), o.H.copy(), o.J.copy()
            o.one_step()
            N = o.N
            hc = emu.lean_cells(k.shape, "h")
            hx, hy, hz = emu.h_lean(k, E, H, k.dt, hc)
            assert hc.size > 0
            for d, v in enumerate((hx, hy, hz)):
                assert np.array_equal(v, o.H[d * N + hc])
            ec = emu.lean_cells(k.shape, "e")
            curl = emu.e_lean_curl(k, o.H, ec)
            t = k.table[k.ids.astype(np.int64)[ec]]
            for d in range(3):
                ieps = t[:, d]
                e_new = E[d * N + ec] + k.dt * (curl[d] - ieps * J[d * N + ec])
                assert np.array_equal(e_new, o.E[d * N + ec])


@pytest.mark.parametrize("idx", VALID)
def test_adjoint_operators_equal_oracle_matrices(idx):
    """The host assembly behind the adjoint kernels reproduces upstream's
    operators: A = dt * iDa iDmu C Ds and diag(ieps) B0 = iDeps itDa C^T tDs
    (the oracle's scipy matrices) on every valid step case."""
    from types import SimpleNamespace
    from wakis_b200.adjoint import assemble_operators
    c = cases.STEP_CASES[idx]
    o = oracle_step_case(c)
    k = _coef(c)
    nx, ny, nz = c["shape"]
    fake = SimpleNamespace(_coef=k, Nx=nx, Ny=ny, Nz=nz, dt=k.dt)
    A, B0 = assemble_operators(fake)
    dtA = (float(k.dt) * o.A.astype(np.float64)).toarray()
    Bo = o.B.astype(np.float64).toarray()
    ie = o.ieps.astype(np.float64)
    scale = np.max(np.abs(dtA)) or 1.0
    assert np.max(np.abs(A.toarray() - dtA)) <= 1e-6 * scale if c["dtype"] == "float32" \
        else np.max(np.abs(A.toarray() - dtA)) <= 1e-14 * scale
    B = ie[:, None] * B0.toarray()
    scale = np.max(np.abs(Bo)) or 1.0
    tol = 1e-6 if c["dtype"] == "float32" else 1e-14
    assert np.max(np.abs(B - Bo)) <= tol * scale


def test_key_order_matches_string_sort():
    """Upstream reads the Ez history in the order of its '#%05d' keys sorted
    as strings (wakeSolver.py:488-491); the vectorised order and its inverse
    (the position of each step) match Python's sort, past 10^5 and 10^6."""
    from wakis_b200.wakeSolver import WakeSolver
    for n in (0, 7, 99999, 100000, 100001, 234567, 1000011):
        ref = [int(k[1:]) for k in sorted("#" + str(i).zfill(5) for i in range(n))]
        order = WakeSolver._key_order(n)
        assert order.tolist() == ref
        pos = WakeSolver._key_positions(n)
        if n <= 100000:
            assert pos is None
        else:
            assert np.array_equal(order[pos], np.arange(n))


def test_batch_tile_policy():
    """The batched launches' tile-shape policy: the share of tile lanes that
    hold a cell, and the shape "fill" picks (32x16 only where it leaves
    fewer lanes idle than 64x8)."""
    from types import SimpleNamespace
    from wakis_b200 import batch
    assert batch.tile_fill(64, 8, 64) == 1.0
    assert batch.tile_fill(72, 72, 64) == pytest.approx(72 * 72 / (128 * 72))
    assert batch.tile_fill(72, 72, 32) == pytest.approx(72 * 72 / (96 * 80))
    rows = lambda nx, ny, pol: batch.tile_rows_for(SimpleNamespace(Nx=nx, Ny=ny), pol)
    assert rows(72, 72, "fill") == 16 and rows(128, 128, "fill") == 8
    assert rows(36, 24, "fill") == 8 and rows(32, 32, "fill") == 16
    assert rows(72, 72, "64x8") == 8 and rows(128, 128, "32x16") == 16
    with pytest.raises(ValueError):
        rows(64, 64, "16x32")
