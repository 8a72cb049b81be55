"""Device parity: the wakis_b200 kernels (through the C ABI) against the
oracle and the upstream fixtures.

Tolerances: FP64 fields after N steps within 1e-12 relative (max-abs error
over max-abs value, per field); wake potentials and impedances within 1e-10
relative in the same sense.  Runs that involve no exponential (no beam) are
required to be value-for-value identical to the oracle, which itself equals
upstream value for value (tests/test_oracle.py); with the fused beam the
only difference is CUDA's exp() against numpy's on the beam line.
"""

import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cases  # noqa: E402
from helpers import (b200_step_case, b200_wake_case, oracle_step_case,  # noqa: E402
                     oracle_wake_case, rel_err)
from oracle import fit as ofit  # noqa: E402
from oracle import wake as owake  # noqa: E402

FIELD_TOL = 1e-12
WAKE_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _valid(idx):
    try:
        oracle_step_case(cases.STEP_CASES[idx])
        return True
    except ValueError:
        return False


VALID = [i for i in range(len(cases.STEP_CASES)) if _valid(i)]


SCHEDULES = {"auto": ("auto", (0, 0)),
             "twopass": ("twopass", (0, 0)), "twopass2": ("twopass", (0, 2)),
             "twopass4": ("twopass", (0, 4)), "cell": ("cell", (0, 0)), "split": None}


@pytest.mark.parametrize("sched", list(SCHEDULES))
@pytest.mark.parametrize("idx", VALID)
def test_steps_without_beam_are_exact(idx, sched):
    c = cases.STEP_CASES[idx]
    o = oracle_step_case(c)
    s = b200_step_case(c)
    split = SCHEDULES[sched] is None
    if not split:
        s.kernel, s.tile = SCHEDULES[sched]
    assert s.dt == o.dt
    E0, H0 = cases.initial_fields(c, o.N)
    o.E[:], o.H[:] = E0, H0
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    for _ in range(c["steps"]):
        o.one_step()
    s._advance(c["steps"], 0, split=split)
    assert np.array_equal(s.E.numpy(), o.E)
    assert np.array_equal(s.H.numpy(), o.H)
    assert np.array_equal(s.J.numpy(), o.J)


@pytest.mark.parametrize("sched", ["auto", "twopass", "cell"])
@pytest.mark.parametrize("idx", VALID)
def test_steps_with_fused_beam_match_upstream(idx, sched, golden_dir):
    g = np.load(os.path.join(golden_dir, "step_cases.npz"))
    c = cases.STEP_CASES[idx]
    s = b200_step_case(c)
    s.kernel, s.tile = SCHEDULES[sched]
    E0, H0 = cases.initial_fields(c, s.N)
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    from wakis_b200.sources import Beam
    bp = Beam(**c["beam"]).params(s)
    s._advance(c["steps"], 0, beam=bp)
    tol = FIELD_TOL if c["dtype"] == "float64" else 1e-5
    for f in "EHJ":
        ref = g[f"c{idx}_{f}"]
        got = getattr(s, f).numpy()
        assert rel_err(got, ref) <= tol, (f, rel_err(got, ref))


def test_generic_beam_path_matches_fused():
    c = cases.STEP_CASES[2]   # conductive, PEC
    from wakis_b200.sources import Beam
    a = b200_step_case(c)
    b = b200_step_case(c)
    bm = Beam(**c["beam"])
    bp = Beam(**c["beam"]).params(a)
    for n in range(4):
        a._advance(1, n, beam=bp)
        bm.update(b, n * b.dt)
        b.one_step()
    assert rel_err(a.E.numpy(), b.E.numpy()) <= FIELD_TOL
    assert rel_err(a.J.numpy(), b.J.numpy()) <= FIELD_TOL


@pytest.mark.parametrize("idx", range(len(cases.WAKE_CASES)))
def test_wakesolve_matches_upstream(idx, golden_dir):
    g = np.load(os.path.join(golden_dir, "wake_cases.npz"))
    c = cases.WAKE_CASES[idx]
    s, w = b200_wake_case(c)
    s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"])
    assert s.Nt == int(g[f"c{idx}_Nt"])
    assert np.array_equal(w.s, g[f"c{idx}_s"]) and np.array_equal(w.f, g[f"c{idx}_f"])
    names = ["WP", "Z", "lambdaf"]
    if c["compute_plane"] == "both":
        names += ["WP_3d", "WPx", "WPy", "Zx", "Zy"]
    tol = WAKE_TOL if c["dtype"] == "float64" else 1e-5
    for n in names:
        assert rel_err(getattr(w, n), g[f"c{idx}_{n}"]) <= tol, (n, rel_err(getattr(w, n),
                                                                           g[f"c{idx}_{n}"]))
    assert rel_err(s.E.numpy()[2 * s.N:], g[f"c{idx}_Ez"]) <= (FIELD_TOL if c["dtype"] ==
                                                               "float64" else 1e-5)


def test_wake_kernels_exact_on_oracle_history():
    """Fed the oracle's own Ez history, the wake-potential and transverse
    kernels reproduce the oracle value for value (same order of every sum)."""
    c = cases.WAKE_CASES[0]
    so, wo = oracle_wake_case(c)
    owake.wakesolve(so, wo, c["wakelength"])
    s, w = b200_wake_case(c)
    keys = sorted(wo.hist)
    Nt = len(keys)
    hist = np.zeros((9, s.Nz, Nt))
    for n in range(Nt):
        hist[:, :, n] = wo.hist["#" + str(n).zfill(5)].reshape(9, s.Nz)
    w.xf, w.yf, w.zf, w.t = wo.xf, wo.yf, wo.zf, wo.t
    w.dx, w.dy, w.dz = wo.dx, wo.dy, wo.dz
    w.wakelength = c["wakelength"]
    w.set_history(torch.as_tensor(hist, device="cuda"), Nt)
    w.solve("both")
    assert np.array_equal(w.WP_3d, wo.WP_3d)
    assert np.array_equal(w.WPx, wo.WPx) and np.array_equal(w.WPy, wo.WPy)
    assert rel_err(w.Z, wo.Z) <= 1e-12 and rel_err(w.Zx, wo.Zx) <= 1e-12


def _test001_mask(x, y, z):
    from wakis_b200 import geometry
    shp = geometry.Box(-0.025, 0.025, -0.025, 0.025, -0.015, 0.015, tol=1e-12) | \
        geometry.Box(-0.0075, 0.0075, -0.0075, 0.0075, -1.0, 1.0, tol=1e-12)
    return geometry.cell_mask(shp, x, y, z)


def test_upstream_test001_regression_vectors(golden_dir):
    """Upstream tests/test_001_pec_cubic_cavity.py on the device (float32,
    50x50x150, 5184 steps) against its regression vectors and tolerances."""
    import wakis_b200 as wb
    gold = np.load(os.path.join(golden_dir, "upstream_test001.npz"))
    g = wb.GridFIT3D(-0.025, 0.025, -0.025, 0.025, -0.05, 0.05, 50, 50, 150, verbose=0)
    g.add_solid("cavity", _test001_mask(g.x, g.y, g.z), "vacuum")
    w = wb.WakeSolver(q=1e-9, sigmaz=18.5e-3, beta=1.0, save=False, skip_cells=12, verbose=0)
    s = wb.SolverFIT3D(g, w, bc_low=["pec"] * 3, bc_high=["pec"] * 3, use_stl=True, bg="pec",
                       dtype=np.float32, verbose=0)
    s.wakesolve(wakelength=1.0)
    assert s.Nt == 5184
    tol = float(gold["WP_tol"])
    assert np.allclose(w.WP[::50], gold["WP"], rtol=tol, atol=tol)
    assert np.cumsum(np.abs(w.WP))[-1] == pytest.approx(float(gold["WP_cumsum"]),
                                                        float(gold["WP_cumsum_rel"]))
    tz = float(gold["Z_tol"])
    for fn in (np.abs, np.real, np.imag):
        assert np.allclose(fn(w.Z)[::20], fn(gold["Z"]), rtol=tz, atol=tz)


def test_cavity_40_wakesolve_matches_oracle():
    """The 40x40x80 FP64 PEC cavity workload end to end (1896 steps)."""
    from wakis_b200 import workloads
    gb, wb_, sb = workloads.build_b200("cavity_40", dtype=np.float64)
    sp = workloads.spec("cavity_40")
    m = workloads.cavity_mask(gb.x, gb.y, gb.z)
    go = ofit.Grid(*workloads.BOUNDS, *sp["shape"], solids={"cavity": m},
                   materials={"cavity": "vacuum"})
    wo = owake.WakeOracle(**sp["wake"])
    so = ofit.Solver(go, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
                     dtype=np.float64, wake_fmax=wo.fmax)
    owake.wakesolve(so, wo, sp["wakelength"])
    sb.wakesolve(wakelength=sp["wakelength"])
    assert sb.Nt == so.Nt == 1896
    for f in "EH":
        assert rel_err(getattr(sb, f).numpy(), getattr(so, f)) <= FIELD_TOL, f
    for n in ("WP", "WP_3d", "WPx", "WPy", "Z", "Zx", "Zy"):
        assert rel_err(getattr(wb_, n), getattr(wo, n)) <= WAKE_TOL, n


@pytest.mark.parametrize("kernel,tile", [("twopass", (0, 0)),
                                         ("twopass", (0, 1)), ("twopass", (0, 4)),
                                         ("tma", (0, 0)), ("tma", (0, 3))])
def test_schedules_equal_cell_kernel_with_beam_and_capture(kernel, tile):
    """The TMA, two-pass and per-cell kernels give identical fields and Ez
    history (same arithmetic, different schedules)."""
    c = cases.WAKE_CASES[3]     # conductive background, PML, beta < 1
    a, wa = b200_wake_case(c)
    b, wb_ = b200_wake_case(c)
    a.kernel, a.tile = kernel, tile
    b.kernel = "cell"
    from wakis_b200.sources import Beam
    bp = Beam(q=1e-9, sigmaz=0.004, beta=0.7).params(a)
    ha = torch.zeros((9, a.Nz, 40), dtype=torch.float64, device="cuda")
    hb = torch.zeros_like(ha)
    a._advance(40, 0, beam=bp, capture=(ha, 5, 6, 3, 3))
    b._advance(40, 0, beam=bp, capture=(hb, 5, 6, 3, 3))
    assert np.array_equal(a.E.numpy(), b.E.numpy())
    assert np.array_equal(a.H.numpy(), b.H.numpy())
    assert torch.equal(ha, hb)


def _wake_errors(a, b):
    return {n: rel_err(getattr(a, n), getattr(b, n)) for n in ("WP", "WPx", "WPy", "Z", "Zx")}


@pytest.mark.parametrize("name", ["cavity_40", "lossy_small"])
def test_fp32c_wake_within_1e4_of_fp64(name):
    """FP32-compensated state: WP and |Z| within 1e-4 relative of the FP64
    run on the same grid (north-star accuracy bar); plain FP32 is reported
    beside it for context."""
    from wakis_b200 import workloads
    import wakis_b200 as wb
    if name == "cavity_40":
        runs = {}
        for prec in (None, "fp32c"):
            g, w, s = workloads.build_b200("cavity_40", dtype=np.float64, precision=prec)
            s.wakesolve(wakelength=workloads.spec("cavity_40")["wakelength"])
            runs[prec] = (s, w)
    else:   # conductive background + z-PML, beta < 1 (tests/cases WAKE_CASES[3])
        c = dict(cases.WAKE_CASES[3])
        runs = {}
        for prec in (None, "fp32c"):
            g = wb.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
            g.add_solid("cav", cases.wake_mask(c, g.x, g.y, g.z), c["material"])
            w = wb.WakeSolver(save=False, verbose=0, **c["wake"])
            s = wb.SolverFIT3D(g, w, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True,
                               bg=c["bg"], dtype=np.float64, verbose=0, precision=prec)
            s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"])
            runs[prec] = (s, w)
    err = _wake_errors(runs["fp32c"][1], runs[None][1])
    print(name, "fp32c vs fp64", err)
    assert err["WP"] <= 1e-4 and err["Z"] <= 1e-4
    assert rel_err(np.abs(runs["fp32c"][1].Z), np.abs(runs[None][1].Z)) <= 1e-4


TMA_GRIDS = [((16, 12, 20), "float64"), ((24, 16, 30), "float64"), ((32, 20, 26), "float32"),
             ((72, 18, 40), "float64")]


@pytest.mark.parametrize("rows", [8, 16])
@pytest.mark.parametrize("shape,dtype", TMA_GRIDS)
@pytest.mark.parametrize("bcs", [(["pec"] * 3, ["pec"] * 3),
                                 (["periodic", "pec", "pml"], ["periodic", "pec", "pml"]),
                                 (["pec", "pec", "abc"], ["pec", "pec", "abc"]),
                                 (["pec", "electric", "periodic"], ["pml", "pec", "periodic"]),
                                 (["pec", "pec", "pec"], ["pec", "pec", "abc"])])
def test_tma_kernel_exact_against_oracle(shape, dtype, bcs, rows):
    """TMA-staged fused kernel (interior) + shell, on 64x8 (rows 8) and
    32x16 tiles (rows 16): value-for-value equal to the oracle after
    several steps from random fields (no exponential)."""
    c = dict(cases.STEP_CASES[2])     # conductive materials on the case boxes
    c.update(shape=shape, dtype=dtype, bc_low=bcs[0], bc_high=bcs[1], steps=5, n_pml=3)
    o = oracle_step_case(c)
    s = b200_step_case(c)
    s.kernel, s.tile = "tma", (rows, 0)
    E0, H0 = cases.initial_fields(c, o.N)
    o.E[:], o.H[:] = E0, H0
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    for _ in range(c["steps"]):
        o.one_step()
    s._advance(c["steps"], 0)
    assert int(s._status.item()) == 0
    assert np.array_equal(s.E.numpy(), o.E)
    assert np.array_equal(s.H.numpy(), o.H)


@pytest.mark.parametrize("tile", [(0, 0), (0, 1), (0, 3), (0, 100)])
def test_tma_equals_twopass_with_beam_and_capture(tile):
    """40x40x80 PEC cavity workload, 60 steps with the fused beam and the Ez
    window capture: TMA kernel (several planes-per-block) equals two-pass."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    _, wa, a = workloads.build_b200("cavity_40")
    _, wb_, b = workloads.build_b200("cavity_40")
    a.kernel, a.tile = "tma", tile
    b.kernel = "twopass"
    bp = Beam(q=1e-9, sigmaz=0.01, beta=1.0).params(a)
    ha = torch.zeros((9, a.Nz, 60), dtype=torch.float64, device="cuda")
    hb = torch.zeros_like(ha)
    a._advance(60, 0, beam=bp, capture=(ha, 18, 18, 3, 3))
    b._advance(60, 0, beam=bp, capture=(hb, 18, 18, 3, 3))
    assert int(a._status.item()) == 0
    assert np.array_equal(a.E.numpy(), b.E.numpy())
    assert np.array_equal(a.H.numpy(), b.H.numpy())
    assert torch.equal(ha, hb)


def test_timed_step_matches_untimed():
    """wk_fit_step_timed: same state as wk_fit_step, one timed interior
    launch per step for the TMA schedule, positive time."""
    from wakis_b200 import workloads
    _, _, a = workloads.build_b200("cavity_40")
    _, _, b = workloads.build_b200("cavity_40")
    timing = []
    a._advance(12, 0, timing=timing)
    b._advance(12, 0)
    assert sum(t[1] for t in timing) == 12
    assert sum(t[0] for t in timing) > 0
    assert np.array_equal(a.E.numpy(), b.E.numpy())
    assert np.array_equal(a.H.numpy(), b.H.numpy())


def _decoded(s, fld):
    """FP32c state v + c of E or H as float64 numpy (flat 3N)."""
    v = (s._E if fld == "E" else s._H)[s._par].double()
    c = (s._Ec if fld == "E" else s._Hc)[s._par].double()
    return (v + c).cpu().numpy()


@pytest.mark.parametrize("tile", [(0, 0), (0, 3)])
def test_fp32c_tma_close_to_twopass(tile):
    """Compensated TMA kernel (float factors, packed f32x2 rows) against the
    compensated two-pass kernels (FP64-formed coefficients per cell): 150
    steps of the 40x40x80 cavity with beam and capture agree to ~1e-6
    relative; the status word stays 0."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    _, _, a = workloads.build_b200("cavity_40", precision="fp32c")
    _, _, b = workloads.build_b200("cavity_40", precision="fp32c")
    a.kernel, a.tile = "tma", tile
    b.kernel = "twopass"
    bp = Beam(q=1e-9, sigmaz=0.01, beta=1.0).params(a)
    ha = torch.zeros((9, a.Nz, 150), dtype=torch.float64, device="cuda")
    hb = torch.zeros_like(ha)
    a._advance(150, 0, beam=bp, capture=(ha, 18, 18, 3, 3))
    b._advance(150, 0, beam=bp, capture=(hb, 18, 18, 3, 3))
    assert int(a._status.item()) == 0
    for f in "EH":
        assert rel_err(_decoded(a, f), _decoded(b, f)) <= 2e-6
    assert rel_err(ha.cpu().numpy(), hb.cpu().numpy()) <= 2e-6


@pytest.mark.parametrize("shape", [(40, 40, 80), (36, 20, 30), (72, 44, 24)])
@pytest.mark.parametrize("bcs", [(["pec"] * 3, ["pec"] * 3),
                                 (["pec", "pec", "abc"], ["pec", "pec", "abc"]),
                                 (["periodic", "pec", "pml"], ["periodic", "pec", "pml"])])
def test_fp32c_tma_32x16_tiles_equal_64x8(bcs, shape):
    """The compensated TMA kernel on 32x16 tiles (wk_fit_desc.tile_rows =
    16, the default) gives the 64x8 tiles' (tile_rows = 8) fields,
    compensation words and Ez capture value for value: every cell runs the
    same rows, only the split of the grid into blocks differs (all three
    face modes; grids cut by both tile shapes; row pitch with and without
    TMA-loaded compensation words)."""
    from wakis_b200.sources import Beam
    c = dict(cases.STEP_CASES[2])
    c.update(shape=shape, dtype="float64", bc_low=bcs[0], bc_high=bcs[1], n_pml=3)
    runs = []
    for rows in (8, 16):
        s = b200_step_case(c, precision="fp32c")
        s.kernel, s.tile = "tma", (rows, 0)
        E0, H0 = cases.initial_fields(c, s.N)
        s.E.fromarray(E0)
        s.H.fromarray(H0)
        bp = Beam(q=1e-9, sigmaz=0.005, beta=1.0).params(s)
        h = torch.zeros((9, s.Nz, 40), dtype=torch.float64, device="cuda")
        s._advance(40, 0, beam=bp, capture=(h, s.Nx // 2 - 1, s.Ny // 2 - 1, 3, 3))
        assert int(s._status.item()) == 0
        bits = lambda t: t.view(torch.int16) if t.dtype == torch.bfloat16 else t
        runs.append([bits(t).cpu().numpy() for t in (s._E[s._par], s._H[s._par],
                                                      s._Ec[s._par], s._Hc[s._par], h)])
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(16, 12, 20), (20, 12, 20)])
@pytest.mark.parametrize("bcs", [(["pec"] * 3, ["pec"] * 3),
                                 (["periodic", "pec", "pml"], ["periodic", "pec", "pml"])])
def test_fp32c_tma_fields_close_to_oracle(bcs, shape):
    """Compensated TMA path from random fields on a 16x12x20 grid (row pitch
    Nx % 8 == 0: compensation words staged by TMA) and a 20x12x20 grid
    (per-thread loads) with conductive materials: E and H after 8 steps
    within 1e-5 relative of the FP64 oracle."""
    c = dict(cases.STEP_CASES[2])
    c.update(shape=shape, dtype="float64", bc_low=bcs[0], bc_high=bcs[1], steps=8,
             n_pml=3)
    o = oracle_step_case(c)
    s = b200_step_case(c, precision="fp32c")
    s.kernel = "tma"
    E0, H0 = cases.initial_fields(c, o.N)
    o.E[:], o.H[:] = E0, H0
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    for _ in range(c["steps"]):
        o.one_step()
    s._advance(c["steps"], 0)
    assert int(s._status.item()) == 0
    assert rel_err(_decoded(s, "E"), o.E) <= 1e-5
    assert rel_err(_decoded(s, "H"), o.H) <= 1e-5


@pytest.mark.parametrize("idx", [2, 5])
def test_fp32c_compensated_stencil_tracks_fp64(idx):
    """The compensated stencil (comp_stencil: every neighbour value read as
    v + c, increments formed with error-free float transformations) keeps
    the FP32c state on the FP64 oracle's trajectory: from random
    float-exact fields on a 16x12x20 grid, E and H after 8 steps
    (conductive materials, PML faces) within 1e-8 relative and at least
    twice as close as with the float stencil.  (Over the thousands of steps
    of a wake or adjoint run the gap grows: the float stencil's increments
    carry a float rounding every step; see the adjoint gradient test.)"""
    c = dict(cases.STEP_CASES[idx])
    c.update(shape=(16, 12, 20), dtype="float64", steps=8, n_pml=3)
    o = oracle_step_case(c)
    # float-exact initial fields: writing the state sets v = float(value), c = 0
    E0, H0 = (f.astype(np.float32).astype(np.float64) for f in cases.initial_fields(c, o.N))
    o.E[:], o.H[:] = E0, H0
    for _ in range(c["steps"]):
        o.one_step()
    err = {}
    for cst in (False, True):
        s = b200_step_case(c, precision="fp32c")
        s.kernel = "twopass"
        s.comp_stencil = cst
        s.E.fromarray(E0)
        s.H.fromarray(H0)
        s._advance(c["steps"], 0)
        err[cst] = max(rel_err(_decoded(s, "E"), o.E), rel_err(_decoded(s, "H"), o.H))
    assert err[True] <= 1e-8, err
    assert err[True] * 2 <= err[False], err


def _small_pillboxes(precision=None):
    from wakis_b200 import batch
    ps = [dict(R=0.020, L=0.030, beta=0.9, sigma=1e4), dict(R=0.026, L=0.036, beta=0.6, sigma=3e5),
          dict(R=0.022, L=0.040, beta=1.0, sigma=2e3)]
    return [batch.build_pillbox(**q, cell=2e-3, precision=precision) for q in ps]


def test_batched_graph_equals_individual_wakesolve():
    """Three uneven pillboxes stepped in one replayed CUDA graph (device step
    counter, 4 streams) give the same WP and Z, value for value, as separate
    wakesolve runs of the same instances."""
    from wakis_b200 import batch
    inst = _small_pillboxes()
    b = batch.BatchedWakeSolve([x[2] for x in inst], 601, streams=4)
    b.run()
    solo = _small_pillboxes()
    for (g, w, s), (g2, w2, s2) in zip(inst, solo):
        wl = batch.BatchedWakeSolve.wakelength_for(s2, 601)
        s2.wakesolve(wakelength=wl)
        assert s2.Nt == 601
        assert int(s._status.item()) == 0
        assert np.array_equal(np.asarray(w.WP), np.asarray(w2.WP))
        assert np.array_equal(np.asarray(w.Z), np.asarray(w2.Z))
        assert np.array_equal(s.E.numpy(), s2.E.numpy())


def test_batched_fp32c_close_to_fp64():
    """The same batch in FP32c: WP and |Z| of every instance within 1e-4 of
    the FP64 batch."""
    from wakis_b200 import batch
    a = _small_pillboxes("fp32c")
    b = _small_pillboxes()
    batch.BatchedWakeSolve([x[2] for x in a], 600, streams=2).run()
    batch.BatchedWakeSolve([x[2] for x in b], 600, streams=2).run()
    for (_, wa, _), (_, wb_, _) in zip(a, b):
        assert rel_err(np.asarray(wa.WP), np.asarray(wb_.WP)) <= 1e-4
        assert rel_err(np.abs(np.asarray(wa.Z)), np.abs(np.asarray(wb_.Z))) <= 1e-4


def _design_problem(dtype, n_steps=800, adjoint_dtype=None, precision=None,
                    operators="stencil", comp_stencil=False):
    """cavity_40 geometry with an 8x8x8-cell design region at the centre,
    PEC walls (dt not clamped), FP32, FP64 or FP32-compensated (with the
    float or the compensated stencil)."""
    from wakis_b200 import workloads
    from wakis_b200.adjoint import ImpedanceDesign
    _, _, s = workloads.build_b200("cavity_40", dtype=dtype, precision=precision)
    s.comp_stencil = comp_stencil
    m = np.zeros((s.Nx, s.Ny, s.Nz), bool)
    m[16:24, 16:24, 36:44] = True
    return ImpedanceDesign(s, m, f_band=(0.5e9, 3e9), n_steps=n_steps, segment=30,
                           adjoint_dtype=adjoint_dtype, operators=operators)


@pytest.mark.parametrize("dtype,prec", [(np.float64, None), (np.float32, None),
                                        (np.float64, "fp32c")])
def test_adjoint_graph_replay_equals_step_by_step(dtype, prec):
    """The backward pass with the full segments replayed from one captured
    CUDA graph gives the gradient of the step-by-step backward pass value
    for value (same kernels in the same order; 400 steps, segments of 30)."""
    rng = np.random.default_rng(4)
    er = rng.uniform(1.0, 10.0, 512)
    sg = rng.uniform(0.0, 10.0, 512)
    p = _design_problem(dtype, n_steps=400, precision=prec)
    p.set_params(er, sg)
    p.forward()
    ge1, gs1 = p.backward(graph=False)
    ge2, gs2 = p.backward(graph=True)
    assert np.abs(ge1).max() > 0
    assert np.array_equal(ge1, ge2) and np.array_equal(gs1, gs2)


@pytest.mark.parametrize("dtype,adt", [(np.float64, None), (np.float32, None),
                                       (np.float32, np.float64)])
def test_adjoint_stencil_transposes_equal_csr(dtype, adt):
    """The matrix-free transposes (wk_adj_h_fit / wk_adj_e_fit, stencils over
    the compact coefficient tables) give the gradient of the CSR products of
    the host-assembled A^T, B0^T to rounding (same parameters, 300 steps)."""
    rng = np.random.default_rng(2)
    er = rng.uniform(1.0, 10.0, 512)
    sg = rng.uniform(0.0, 10.0, 512)
    out = {}
    for op in ("csr", "stencil"):
        p = _design_problem(dtype, n_steps=300, adjoint_dtype=adt, operators=op)
        p.set_params(er, sg)
        p.forward()
        out[op] = p.backward()
    tol = 1e-10 if (adt or dtype) == np.float64 else 1e-4
    for a, b in zip(out["stencil"], out["csr"]):
        assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b))


@pytest.mark.parametrize("adt", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(7, 5, 9), (37, 13, 11), (64, 16, 10), (33, 9, 17)])
@pytest.mark.parametrize("idx", VALID[::5])
def test_adjoint_tiled_transposes_equal_per_cell(idx, shape, adt):
    """The z-marching tiled transposes (the default of wk_adj_h_fit /
    wk_adj_e_fit), with the cell factors from the tables or from
    wk_adj_factors, equal the one-thread-per-cell kernels value for value,
    in place, with and without the decay factor, on grids whose edges cut
    the 32x8 tiles (the flat-offset neighbours past a row or plane end) and
    on every face mix of the step cases."""
    import ctypes
    from wakis_b200 import _native
    c = dict(cases.STEP_CASES[idx], shape=shape)
    s = b200_step_case(c)
    base = _native.FitDesc.from_buffer_copy(s._sync_desc())
    N = s.N
    rng = np.random.default_rng(idx + sum(shape))
    tdt = torch.float64 if adt == np.float64 else torch.float32
    wk = _native.WK_F64 if adt == np.float64 else _native.WK_F32
    mk = lambda lo, hi: torch.tensor(rng.uniform(lo, hi, 3 * N), dtype=tdt, device="cuda")
    lamE, lamH, decay = mk(-1, 1), mk(-1, 1), mk(0.5, 1)
    lib = _native.lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    fu, fw = torch.empty_like(lamE), torch.empty_like(lamE)
    _native.check(lib.wk_adj_factors(base, wk, ptr(fu), ptr(fw), st), "wk_adj_factors")
    out = {}
    for kern, fac in ((_native.WK_KERNEL_CELL, False), (_native.WK_KERNEL_AUTO, False),
                      (_native.WK_KERNEL_AUTO, True)):
        d = _native.FitDesc.from_buffer_copy(base)
        d.kernel = kern
        pu, pw = (ptr(fu), ptr(fw)) if fac else (None, None)
        h, e, e2 = lamH.clone(), lamE.clone(), lamE.clone()
        _native.check(lib.wk_adj_h_fit(d, wk, pu, ptr(lamE), ptr(h), ptr(h), st),
                      "wk_adj_h_fit")
        _native.check(lib.wk_adj_e_fit(d, wk, pw, ptr(h), ptr(e), ptr(decay), ptr(e), st),
                      "wk_adj_e_fit")
        _native.check(lib.wk_adj_e_fit(d, wk, pw, ptr(lamH), ptr(e2), None, ptr(e2), st),
                      "wk_adj_e_fit")
        out[(kern, fac)] = [t.cpu().numpy() for t in (h, e, e2)]
    ref = out[(_native.WK_KERNEL_CELL, False)]
    for key in ((_native.WK_KERNEL_AUTO, False), (_native.WK_KERNEL_AUTO, True)):
        for a, b in zip(out[key], ref):
            assert np.array_equal(a, b), key
            assert np.any(a != 0)


def test_adjoint_operators_match_step_kernels():
    """A and B0 assembled on the host reproduce the step kernels: from
    random (E, H) one FP64 step equals H - A E, E + dt ieps (B0 H')."""
    from wakis_b200 import workloads
    from wakis_b200.adjoint import assemble_operators
    _, _, s = workloads.build_b200("cavity_40")
    A, B0 = assemble_operators(s)
    rng = np.random.default_rng(3)
    E0 = rng.standard_normal(3 * s.N)
    H0 = rng.standard_normal(3 * s.N)
    s._first_step()
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    E0, H0 = s.E.numpy().copy(), s.H.numpy().copy()     # ghosts as the kernel sees them
    s._advance(1, 0)
    H1 = H0 - A @ E0
    ie = s.ieps.numpy()
    E1 = E0 + float(s.dt) * ie * (B0 @ H1)
    assert rel_err(s.H.numpy(), H1) <= 1e-13
    assert rel_err(s.E.numpy(), E1) <= 1e-13


@pytest.mark.parametrize("dtype,prec,adt,tol,cst", [
    (np.float64, None, None, 1e-5, False), (np.float64, "fp32c", None, 1e-5, False),
    (np.float64, "fp32c", np.float32, 1e-5, False), (np.float64, "fp32c", None, 1e-5, True),
    (np.float32, None, None, 5e-2, False), (np.float32, None, np.float64, 5e-2, False)])
def test_adjoint_gradient_matches_central_differences(dtype, prec, adt, tol, cst):
    """dL/d(eps_r, sigma) of L = int_{0.5}^{3 GHz} |Z|^2 df from the adjoint
    against central finite differences of FP64 forward runs along 4 random
    directions of the 1024 parameters: within 1e-5 with the FP64 adjoint
    after an FP64 or FP32-compensated forward, and with a float32 adjoint
    state after the compensated forward; the plain float32 forward (either
    adjoint dtype) within a few per cent, the accuracy of its float state
    over 800 steps."""
    rng = np.random.default_rng(1)
    nd = 512
    er = rng.uniform(1.0, 10.0, nd)
    sg = rng.uniform(0.0, 10.0, nd)
    p = _design_problem(dtype, adjoint_dtype=adt, precision=prec, comp_stencil=cst)
    p.set_params(er, sg)
    L = p.forward()
    ge, gs = p.backward()
    assert L > 0 and np.all(np.isfinite(ge)) and np.all(np.isfinite(gs))
    q = _design_problem(np.float64)

    def central(v_e, v_s, h):
        q.set_params(er + h * v_e, sg + h * v_s)
        lp = q.forward(keep=False)
        q.set_params(er - h * v_e, sg - h * v_s)
        lm = q.forward(keep=False)
        return (lp - lm) / (2.0 * h)

    for t in range(4):
        ve = rng.standard_normal(nd)
        vs = rng.standard_normal(nd)
        # Richardson extrapolation of two central differences: O(h^4)
        fd = (4.0 * central(ve, vs, 5e-4) - central(ve, vs, 1e-3)) / 3.0
        ad = ge @ ve + gs @ vs
        print("adjoint", dtype.__name__, prec, adt, t, abs(ad - fd) / abs(fd))
        assert abs(ad - fd) <= tol * abs(fd), (t, ad, fd)


@pytest.mark.parametrize("idx", range(len(cases.SOURCE_CASES)))
def test_emsolve_sources_match_upstream(idx, golden_dir):
    """emsolve driven by PlaneWave / WavePacket / Dipole / Pulse (E, H and J
    hard sources) reproduces upstream's E, H, J after Nt steps."""
    import wakis_b200 as wb
    c = cases.SOURCE_CASES[idx]
    ref = np.load(os.path.join(golden_dir, "source_cases.npz"))
    g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
    s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0, bg="vacuum",
                       use_stl=False, use_sibc=False)
    assert s.dt == ref[f"c{idx}_dt"]
    src = getattr(wb.sources, c["kind"])(**c["kw"])
    s.emsolve(c["Nt"], source=src)
    for f in "EHJ":
        got = getattr(s, f).numpy()
        want = ref[f"c{idx}_{f}"]
        assert rel_err(got, want) <= 1e-12, (f, rel_err(got, want))


@pytest.mark.parametrize("idx", range(len(cases.SOURCE_CASES)))
def test_emsolve_device_sources_equal_update(idx):
    """emsolve with the source values tabulated once and written on the
    device before each step (wk_source_write; step by step, and replayed
    from a captured CUDA graph with a device step counter) equals emsolve
    through the source's update() value for value (E, H, J), with a vacuum
    and with a conductive background."""
    import wakis_b200 as wb
    c = cases.SOURCE_CASES[idx]
    for bg in ("vacuum", [1.0, 1.0, 5.0]):
        out = {}
        for mode in ("graph", "eager", "update"):
            g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
            s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                               bg=bg, use_stl=False, use_sibc=False)
            src = getattr(wb.sources, c["kind"])(**c["kw"])
            s.emsolve(c["Nt"], source=src, device_sources=mode != "update",
                      graph=mode == "graph")
            out[mode] = [getattr(s, f).numpy() for f in "EHJ"]
        for mode in ("graph", "eager"):
            for a, b in zip(out[mode], out["update"]):
                assert np.array_equal(a, b), (bg, mode)


def test_emsolve_device_sources_fp32c():
    """The device-written sources with the compensated state (a point
    source on E in a PEC box): the written cells carry the source value to
    ~32 bits (float + compensation word), and the run stays within 1e-6 of
    the FP64 one."""
    import wakis_b200 as wb
    c = cases.SOURCE_CASES[2]
    res = {}
    for prec in (None, "fp32c"):
        g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
        s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                           bg="vacuum", use_stl=False, use_sibc=False, precision=prec)
        s.emsolve(c["Nt"], source=getattr(wb.sources, c["kind"])(**c["kw"]))
        res[prec] = (_decoded(s, "E"), _decoded(s, "H")) if prec else (s.E.numpy(), s.H.numpy())
    for a, b in zip(res["fp32c"], res[None]):
        assert rel_err(a, b) <= 1e-6


def _const_field(Nx, Ny, Nz, values):
    from wakis_b200.field import Field
    f = Field(Nx, Ny, Nz, dtype=float, device="cuda")
    for c, v in zip("xyz", values):
        f.from_matrix(np.full((Nx, Ny, Nz), v), c)
    return f


def test_field_monitor_upstream_semantics():
    """Upstream tests/test_012_field_monitors.py on the device: initial state,
    first update, zero-frequency accumulation, alternating phase."""
    from wakis_b200.field_monitors import FieldMonitor
    m = FieldMonitor([1.0e9, 2.0e9])
    assert m.time_index == 0 and m.dt is None and m.shape is None and m.xp is None
    assert m.get_components()["Ex"] is None
    f = _const_field(2, 2, 2, (1.0, 2.0, 3.0))
    m = FieldMonitor([0.0])
    m.update(f, 1e-9)
    c = m.get_components()
    assert m.dt == 1e-9 and m.shape == (2, 2, 2) and m.time_index == 1 and m.xp is f.xp
    for k, v in zip(("Ex", "Ey", "Ez"), (1.0, 2.0, 3.0)):
        assert c[k].shape == (1, 2, 2, 2) and c[k].is_complex()
        assert torch.allclose(c[k][0].real, torch.full((2, 2, 2), v, dtype=torch.float64,
                                                        device="cuda"))
    f = _const_field(2, 2, 2, (1.0, 0.0, 0.0))
    m = FieldMonitor([0.0])
    for _ in range(5):
        m.update(f, 0.1)
    c = m.get_components()
    assert torch.allclose(c["Ex"][0].real, torch.full((2, 2, 2), 5.0, dtype=torch.float64,
                                                       device="cuda"))
    assert float(c["Ey"].abs().max()) == 0.0
    f = _const_field(1, 1, 1, (1.0, 0.0, 0.0))
    m = FieldMonitor([0.5])
    for _ in range(4):
        m.update(f, 1.0)
    assert float(m.get_components()["Ex"][0].abs().max()) <= 1e-12


def test_field_monitor_equals_numpy_dft_during_emsolve():
    """Monitor updated from an emsolve callback (Dipole source, 3
    frequencies) equals the numpy running DFT of the same E snapshots."""
    import wakis_b200 as wb
    from wakis_b200.field_monitors import FieldMonitor
    c = cases.SOURCE_CASES[2]
    g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
    s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0, bg="vacuum",
                       use_stl=False, use_sibc=False)
    freqs = np.array([1e9, 4e9, 9e9])
    m = FieldMonitor(freqs)
    ref = {k: np.zeros((3,) + c["shape"], complex) for k in "xyz"}
    n = [0]

    def cb(solver, t):
        m.update(solver.E, solver.dt)
        ph = np.exp(-2j * np.pi * freqs * (n[0] * solver.dt))
        for k in "xyz":
            E = solver.E.to_matrix(k).cpu().numpy()
            for i in range(3):
                ref[k][i] += E * ph[i]
        n[0] += 1

    s.emsolve(30, source=wb.sources.Dipole(field="Ez", nodes=5), callback=cb)
    got = m.get_components()
    for k in "xyz":
        assert np.array_equal(got["E" + k].cpu().numpy(), ref[k])


@pytest.mark.parametrize("name,shape,prec", [("cavity_40", None, None),
                                             ("lossy_256", (64, 64, 128), None),
                                             ("lossy_256", (64, 64, 128), "fp32c")])
def test_clean_faces_skip_equals_masked_step(name, shape, prec):
    """With fields written only by the steps, the tangential E on the PEC
    faces stays +0 and the full-domain kernels skip the H-row column masks
    (faces_clean).  The same 300 steps (beam, Ez capture) after E is
    rewritten with its own zero values (which marks the faces as not clean,
    so every mask is applied) give the same fields and history value for
    value."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec(name)
    runs = []
    for dirty in (False, True):
        _, _, s = workloads.build_b200(name, shape=shape, precision=prec)
        if dirty:
            s._first_step()
            s.E.fromarray(np.zeros(3 * s.N))
            assert not s._faces_clean
        else:
            assert s._faces_clean
        bp = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
                  ).params(s)
        ixt = int(np.abs(s.x).argmin())
        iyt = int(np.abs(s.y).argmin())
        hist = torch.zeros((9, s.Nz, 300), dtype=s._cap_dtype, device="cuda")
        s._advance(300, 0, beam=bp, capture=(hist, ixt - 1, iyt - 1, 3, 3))
        assert int(s._status.item()) == 0
        assert s._faces_clean == (not dirty)
        E = s.E.numpy() if prec is None else _decoded(s, "E")
        H = s.H.numpy() if prec is None else _decoded(s, "H")
        runs.append((E, H, hist.cpu().numpy()))
    assert np.abs(runs[0][0]).max() > 0
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


def _full_size_pair(kernels):
    from wakis_b200 import workloads
    out = []
    for k in kernels:
        _, _, s = workloads.build_b200("lossy_256")
        s.kernel = k
        out.append(s)
    return out


def test_full_size_tma_equals_twopass():
    """lossy_256 at its benchmark size (256x256x512): the full-domain TMA
    step equals the two-pass step value for value, from random fields (H-row
    face masks applied) and from zero fields with the fused beam and the Ez
    capture (faces clean, masks skipped), 8 steps each."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    a, b = _full_size_pair(["tma", "twopass"])
    g = torch.Generator(device="cuda").manual_seed(7)
    E0 = torch.randn(3 * a.N, generator=g, device="cuda", dtype=torch.float64)
    H0 = torch.randn(3 * a.N, generator=g, device="cuda", dtype=torch.float64)
    for s in (a, b):
        s._first_step()
        s.E.fromarray(E0)
        s.H.fromarray(H0)
        s._advance(8, 0)
    assert int(a._status.item()) == 0
    assert torch.equal(a.E.array, b.E.array) and torch.equal(a.H.array, b.H.array)
    sp = workloads.spec("lossy_256")
    bp = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
              ).params(a)
    hists = []
    for s in (a, b):
        s.reset_fields()
        s.step_0, s.nstep = True, 0
        h = torch.zeros((9, s.Nz, 8), dtype=torch.float64, device="cuda")
        s._advance(8, 0, beam=bp, capture=(h, 127, 127, 3, 3))
        hists.append(h)
    assert a._faces_clean
    assert torch.equal(a.E.array, b.E.array) and torch.equal(a.H.array, b.H.array)
    assert torch.equal(hists[0], hists[1])


def test_full_size_step_is_linear():
    """At the benchmark size, 8 source-free steps from 2x a random state give
    exactly twice the steps from the state (scaling by a power of two is
    exact in every product and sum of the update)."""
    a, b = _full_size_pair(["auto", "auto"])
    g = torch.Generator(device="cuda").manual_seed(8)
    E0 = torch.randn(3 * a.N, generator=g, device="cuda", dtype=torch.float64)
    H0 = torch.randn(3 * a.N, generator=g, device="cuda", dtype=torch.float64)
    for s, f in ((a, 1.0), (b, 2.0)):
        s._first_step()
        s.E.fromarray(E0 * f)
        s.H.fromarray(H0 * f)
        s._advance(8, 0)
    assert torch.equal(b.E.array, 2.0 * a.E.array)
    assert torch.equal(b.H.array, 2.0 * a.H.array)


def test_adjoint_gradient_matches_oracle_finite_differences():
    """The FP64 adjoint gradient against central differences of the oracle
    (the CPU restatement of upstream's solver, a fresh solver per
    evaluation): cavity_40 with a 16^3 design region of per-cell eps_r in
    [1, 10] and sigma in [0, 5] S/m (below the relaxation clamp, so every
    evaluation keeps the CFL time step), 800 steps; loss and its
    post-processing as ImpedanceDesign.loss_from_history.  Two random
    directions, Richardson-extrapolated, within 1e-5."""
    import os as _os

    from wakis_b200 import workloads
    from wakis_b200.adjoint import ImpedanceDesign
    from scipy.constants import epsilon_0 as EPS0
    _, _, s = workloads.build_b200("cavity_40")
    m = np.zeros((s.Nx, s.Ny, s.Nz), bool)
    m[12:28, 12:28, 32:48] = True
    p = ImpedanceDesign(s, m, f_band=(0.5e9, 3e9), n_steps=800, segment=30)
    rng = np.random.default_rng(11)
    nd = int(m.sum())
    er = rng.uniform(1.0, 10.0, nd)
    sg = rng.uniform(0.0, 5.0, nd)
    p.set_params(er, sg)
    L = p.forward()
    ge, gs = p.backward()
    sp = workloads.spec("cavity_40")
    cells = np.flatnonzero(m.ravel(order="F"))
    g0 = ofit.Grid(*workloads.BOUNDS, *sp["shape"])
    cav = workloads.cavity_mask(g0.x, g0.y, g0.z)

    def oracle_loss(e_r, sig):
        g = ofit.Grid(*workloads.BOUNDS, *sp["shape"], solids={"cavity": cav, "design": m},
                      materials={"cavity": "vacuum", "design": [1.0, 1.0, 1.0]})
        wo = owake.WakeOracle(**sp["wake"])
        so = ofit.Solver(g, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True,
                         bg=sp["bg"], dtype=np.float64, wake_fmax=wo.fmax)
        assert so.dt == s.dt
        so.set_threads(_os.cpu_count() or 1)
        N = so.N
        for d in range(3):
            so.ieps[d * N + cells] = 1.0 / (e_r * EPS0)
            so.sigma[d * N + cells] = sig
        so.update_tensors()
        so.zero_ghosts()
        beam = ofit.Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource",
                                                         "ysource")})
        ixt = int(np.abs(so.x - sp["wake"]["xtest"]).argmin())
        iyt = int(np.abs(so.y - sp["wake"]["ytest"]).argmin())
        hist = np.zeros((so.Nz, p.n_steps))
        ez = lambda: ofit.comp_view(so.E, 2, so.shape)
        for n in range(p.n_steps):
            beam.update(so, n * so.dt)
            hist[:, n] = ez()[ixt, iyt, :]
            so.one_step()
        return float(p.loss_from_history(torch.as_tensor(hist, device="cuda")).item())

    assert abs(oracle_loss(er, sg) - L) <= 1e-10 * abs(L)
    for t in range(2):
        ve = rng.standard_normal(nd)
        vs = rng.standard_normal(nd)

        def central(h):
            return (oracle_loss(er + h * ve, sg + h * vs)
                    - oracle_loss(er - h * ve, sg - h * vs)) / (2.0 * h)

        fd = (4.0 * central(5e-4) - central(1e-3)) / 3.0
        ad = ge @ ve + gs @ vs
        print("adjoint vs oracle FD", t, abs(ad - fd) / abs(fd))
        assert abs(ad - fd) <= 1e-5 * abs(fd), (t, ad, fd)
