"""Device parity on the benchmarked lossy-wall geometry, on the surface-
impedance (SIBC) pillbox wall and on emsolve with ABC faces.

* The lossy workload (the benchmark's geometry: sigma = 1e4 S/m background,
  dt at the relaxation clamp, 10-cell z-PML, cavity + pipe) is built by the
  same builder as the benchmark (``workloads.build_b200('lossy_256',
  shape=...)``) and stepped on the default path (full-domain TMA kernel,
  clean-face mask skipping while the faces stay clean).  It is compared with
  upstream fixtures (``tests/golden/lossy_cases.npz``) and, at 64x64x128 and
  96x96x192, with the oracle over 200 steps with the beam and the Ez capture.
* The lossy geometry's wake integration (the kernels of WakeSolver.solve on
  the device history) against the oracle's on its own history.
* SIBC: the pillbox wall of the batched form (upstream's surface-impedance
  branch, the same surface mask on both sides) against upstream fixtures,
  through a single solver and through the batched CUDA-graph run.
* ABC: emsolve with ABC faces against upstream, with its CPU snapshot
  semantics (use_gpu=False) and its GPU ones (use_gpu=True).

Tolerances: FP64 fields within 1e-12 relative, WP/Z within 1e-10 (the only
difference being CUDA's exp() against numpy's on the beam line); FP32 within
1e-5.
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cases  # noqa: E402
from helpers import (b200_lossy_case, b200_sibc_case, oracle_lossy_case,  # noqa: E402
                     oracle_sibc_case, rel_err)
from oracle import fit as ofit  # noqa: E402
from oracle import wake as owake  # noqa: E402

FIELD_TOL = 1e-12
WAKE_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _threads(so):
    so.set_threads(os.cpu_count() or 1)
    return so


# ------------------------------------------------------------ lossy geometry
@pytest.mark.parametrize("idx", range(len(cases.LOSSY_CASES)))
def test_lossy_geometry_matches_upstream(idx, golden_dir):
    from wakis_b200.sources import Beam
    g = np.load(os.path.join(golden_dir, "lossy_cases.npz"))
    c = cases.LOSSY_CASES[idx]
    _, _, s = b200_lossy_case(c)
    assert s.dt == g[f"c{idx}_dt"]
    if c["init"] == "random":
        E0, H0 = cases.case_fields(c, s.N)
        s.E.fromarray(E0)
        s.H.fromarray(H0)
    else:
        assert s._faces_clean
    s._advance(c["steps"], 0, beam=Beam(**c["beam"]).params(s))
    s.check_status()
    tol = FIELD_TOL if c["dtype"] == "float64" else 1e-5
    for f in "EHJ":
        got, want = getattr(s, f).numpy(), g[f"c{idx}_{f}"]
        assert rel_err(got, want) <= tol, (f, rel_err(got, want))


def _short_beam(sp):
    """The workload's beam with ti = 2 sigma_z / v: the bunch is at the
    upstream end of the grid from the first step (the workload's own ti puts
    it 8.5 sigma_z outside, where 200 steps of 8.85e-16 s carry it 0.05 mm)."""
    kw = {k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
    kw["ti"] = 2.0 * kw["sigmaz"] / (kw["beta"] * 299792458.0)
    return kw


def _oracle_lossy(shape):
    c = dict(cases.LOSSY_CASES[0])
    c.update(shape=shape)
    return _threads(oracle_lossy_case(c)), c


@pytest.mark.parametrize("shape", [(64, 64, 128), (96, 96, 192)])
def test_lossy_default_path_matches_oracle(shape):
    """200 steps of the benchmark step (fused beam, 3x3 Ez capture, full-
    domain TMA kernel with clean faces) from zero fields: E, H, J and the
    captured Ez history against the oracle."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    so, c = _oracle_lossy(shape)
    _, _, s = workloads.build_b200("lossy_256", shape=shape)
    assert s.dt == so.dt
    assert s._faces_clean
    bkw = _short_beam(sp)
    n = 200
    ixt = int(np.abs(s.x).argmin())
    iyt = int(np.abs(s.y).argmin())
    hist = torch.zeros((9, s.Nz, n), dtype=torch.float64, device="cuda")
    s._advance(n, 0, beam=Beam(**bkw).params(s), capture=(hist, ixt - 1, iyt - 1, 3, 3))
    s.check_status()
    assert s._faces_clean
    beam = ofit.Beam(**bkw)
    ohist = np.zeros((3, 3, so.Nz, n))
    ez = lambda: ofit.comp_view(so.E, 2, so.shape)
    for m in range(n):
        beam.update(so, m * so.dt)
        ohist[..., m] = ez()[ixt - 1:ixt + 2, iyt - 1:iyt + 2, :]
        so.one_step()
    for f in "EHJ":
        want = getattr(so, f)
        assert np.abs(want).max() > 0, f
        assert rel_err(getattr(s, f).numpy(), want) <= FIELD_TOL, f
    assert rel_err(hist.cpu().numpy().reshape(3, 3, so.Nz, n), ohist) <= FIELD_TOL


def test_lossy_random_fields_match_oracle():
    """From seeded random fields (every face mask applied, every coefficient
    of the lossy geometry exercised), 30 steps with the beam at 64x64x128."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    so, c = _oracle_lossy((64, 64, 128))
    _, _, s = workloads.build_b200("lossy_256", shape=(64, 64, 128))
    E0, H0 = cases.initial_fields(c, so.N)
    so.E[:], so.H[:] = E0, H0
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    bkw = _short_beam(sp)
    s._advance(30, 0, beam=Beam(**bkw).params(s))
    s.check_status()
    beam = ofit.Beam(**bkw)
    for m in range(30):
        beam.update(so, m * so.dt)
        so.one_step()
    for f in "EHJ":
        assert rel_err(getattr(s, f).numpy(), getattr(so, f)) <= FIELD_TOL, f


def test_lossy_fp32c_close_to_oracle():
    """The compensated FP32 state on the lossy geometry (default path), 200
    steps with the beam: E and H within 1e-5 of the FP64 oracle."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    so, c = _oracle_lossy((64, 64, 128))
    _, _, s = workloads.build_b200("lossy_256", shape=(64, 64, 128), precision="fp32c")
    bkw = _short_beam(sp)
    s._advance(200, 0, beam=Beam(**bkw).params(s))
    s.check_status()
    beam = ofit.Beam(**bkw)
    for m in range(200):
        beam.update(so, m * so.dt)
        so.one_step()
    for f, buf, cw in (("E", s._E, s._Ec), ("H", s._H, s._Hc)):
        got = (buf[s._par].double() + cw[s._par].double()).cpu().numpy()
        assert rel_err(got, getattr(so, f)) <= 1e-5, f


def test_lossy_wake_integration_matches_oracle():
    """WakeSolver.solve on the device (WP_3d, WP, WPx, WPy, Z, Zx, Zy) on
    the lossy geometry at 64x64x128 from 300 steps of history, against the
    oracle's integration of its own history (both read only the steps that
    exist: int(ts/dt) < steps; the time axis is that of the full run)."""
    import wakis_b200 as wb
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    shape, n, wl = (64, 64, 128), 300, 0.002
    bkw = _short_beam(sp)
    wkw = dict(sp["wake"])
    wkw["ti"] = bkw["ti"]
    so, c = _oracle_lossy(shape)
    _, _, s = workloads.build_b200("lossy_256", shape=shape)
    ixt = int(np.abs(s.x).argmin())
    iyt = int(np.abs(s.y).argmin())
    xx, yy = slice(ixt - 1, ixt + 2), slice(iyt - 1, iyt + 2)
    wo = owake.WakeOracle(**wkw)
    w = wb.WakeSolver(save=False, verbose=0, **wkw)
    z = so.z
    Nt = int(((wl + wo.ti * wo.v + (z.max() - z.min())) / wo.v) / so.dt)
    for ww, sv in ((wo, so), (w, s)):
        ww.wakelength = wl
        ww.xf, ww.yf, ww.zf = sv.x[xx], sv.y[yy], sv.z
        ww.dx, ww.dy, ww.dz = sv.dx, sv.dy, sv.grid.dz
        ww.t = np.arange(0, Nt * sv.dt, sv.dt)
    beam = ofit.Beam(**bkw)
    ez = lambda: ofit.comp_view(so.E, 2, so.shape)
    wo.hist = {}
    for m in range(n):
        beam.update(so, m * so.dt)
        wo.hist["#" + str(m).zfill(5)] = np.array(ez()[xx, yy, :])
        so.one_step()
    wo.solve("both")
    hist = torch.zeros((9, s.Nz, n), dtype=torch.float64, device="cuda")
    s._advance(n, 0, beam=Beam(**bkw).params(s), capture=(hist, ixt - 1, iyt - 1, 3, 3))
    s.check_status()
    w.set_history(hist, n_steps=n)
    w.solve("both")
    assert np.array_equal(w.s, wo.s)
    assert np.abs(wo.WP).max() > 0
    for name in ("WP_3d", "WP", "WPx", "WPy", "Z", "Zx", "Zy"):
        assert rel_err(getattr(w, name), getattr(wo, name)) <= WAKE_TOL, name


# ---------------------------------------------------------------------- SIBC
def test_sibc_step_matches_upstream(golden_dir):
    from wakis_b200.sources import Beam
    g = np.load(os.path.join(golden_dir, "sibc_cases.npz"))
    c = cases.SIBC_CASES[0]
    s = b200_sibc_case(c)
    assert s.dt == g["c0_dt"]
    assert np.array_equal(s.ieps.numpy(), g["c0_ieps"])
    assert np.array_equal(s.sigma.numpy(), g["c0_sigma"])
    E0, H0 = cases.initial_fields(c, s.N)
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    s._advance(c["steps"], 0, beam=Beam(**c["beam"]).params(s))
    s.check_status()
    for f in "EHJ":
        assert rel_err(getattr(s, f).numpy(), g[f"c0_{f}"]) <= FIELD_TOL, f


def _sibc_wake_check(w, s, g, idx=1):
    assert s.Nt == int(g[f"c{idx}_Nt"])
    assert np.array_equal(w.s, g[f"c{idx}_s"]) and np.array_equal(w.f, g[f"c{idx}_f"])
    for n in ("WP", "WP_3d", "WPx", "WPy", "Z", "Zx", "Zy", "lambdaf"):
        assert rel_err(getattr(w, n), g[f"c{idx}_{n}"]) <= WAKE_TOL, n
    assert rel_err(s.E.numpy()[2 * s.N:], g[f"c{idx}_Ez"]) <= FIELD_TOL


def test_sibc_wakesolve_matches_upstream(golden_dir):
    import wakis_b200 as wb
    g = np.load(os.path.join(golden_dir, "sibc_cases.npz"))
    c = cases.SIBC_CASES[1]
    w = wb.WakeSolver(save=False, verbose=0, **c["wake"])
    s = b200_sibc_case(c, wake=w)
    assert s.dt == g["c1_dt"]
    s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"])
    _sibc_wake_check(w, s, g)


def test_sibc_pillbox_in_batched_run_matches_upstream(golden_dir):
    """The SIBC pillbox as one instance of the batched form (the step graph
    replayed with the device step counter), next to a second, different
    instance: the instance's WP/Z equal upstream's wakesolve."""
    import wakis_b200 as wb
    from wakis_b200 import batch
    g = np.load(os.path.join(golden_dir, "sibc_cases.npz"))
    c = cases.SIBC_CASES[1]
    w = wb.WakeSolver(save=False, verbose=0, **c["wake"])
    s = b200_sibc_case(c, wake=w)
    other = batch.build_pillbox(R=0.026, L=0.040, beta=0.7, sigma=3e5, cell=2e-3)[2]
    Nt = int(g["c1_Nt"])
    b = batch.BatchedWakeSolve([s, other], Nt, streams=2)
    b.run()
    # the batch sets each wakelength from the step count (same Nt, another
    # s axis end): integrate the same history on the case's wakelength
    # (the bunch profile is formed again on that axis)
    w.wakelength = c["wakelength"]
    w.lambdas = None
    w.solve("both")
    _sibc_wake_check(w, s, g)


# ----------------------------------------------------------------------- ABC
@pytest.mark.parametrize("idx", range(len(cases.ABC_SOURCE_CASES)))
def test_emsolve_abc_matches_upstream(idx, golden_dir):
    import wakis_b200 as wb
    ref = np.load(os.path.join(golden_dir, "abc_cases.npz"))
    c = cases.ABC_SOURCE_CASES[idx]
    g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
    s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0, bg="vacuum",
                       use_stl=False, use_sibc=False, use_gpu=c["abc_copies"])
    assert s.activate_abc
    assert s.dt == ref[f"c{idx}_dt"]
    src = getattr(wb.sources, c["kind"])(**c["kw"])
    s.emsolve(c["Nt"], source=src)
    for f in "EHJ":
        got, want = getattr(s, f).numpy(), ref[f"c{idx}_{f}"]
        assert rel_err(got, want) <= FIELD_TOL, (f, rel_err(got, want))


def test_abc_on_both_sides_of_an_axis_raises_like_upstream():
    """Upstream keeps one snapshot dict per axis, so ABC on both z faces
    loses the low face's entries and update_abc raises KeyError."""
    import wakis_b200 as wb
    g = wb.GridFIT3D(*cases.SOURCE_BOUNDS, 16, 16, 24, verbose=0)
    s = wb.SolverFIT3D(g, bc_low=["pec", "pec", "abc"], bc_high=["pec", "pec", "abc"],
                       verbose=0, bg="vacuum", use_stl=False, use_sibc=False)
    with pytest.raises(KeyError):
        s.emsolve(2, source=wb.sources.Dipole(field="Ez", nodes=5))


# ------------------------------------------------------- temporal blocking
@pytest.mark.parametrize("shape,dtype,tile", [((64, 64, 128), np.float64, 0),
                                              ((64, 64, 128), np.float64, 3),
                                              ((72, 40, 52), np.float64, 7),
                                              ((72, 40, 52), np.float64, 1),
                                              ((64, 64, 128), np.float32, 0),
                                              ((136, 24, 33), np.float32, 5)])
def test_two_steps_per_launch_equal_one(shape, dtype, tile):
    """k_tma2 (two steps per launch, overlapped tiles) against k_tma (one
    step per launch) on the lossy geometry: 42 steps with the fused beam and
    the Ez capture give the same fields and history value for value (the
    first step runs alone, then ten pairs of two-step launches and one
    single step)."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    out = []
    for spl in (2, 1):
        _, _, s = workloads.build_b200("lossy_256", shape=shape, dtype=dtype)
        s.steps_per_launch = spl
        s.tile = (0, tile)
        ixt = int(np.abs(s.x).argmin())
        iyt = int(np.abs(s.y).argmin())
        hist = torch.zeros((9, s.Nz, 42), dtype=s._cap_dtype, device="cuda")
        timing = []
        s._advance(42, 0, beam=Beam(**_short_beam(sp)).params(s),
                   capture=(hist, ixt - 1, iyt - 1, 3, 3), timing=timing)
        s.check_status()
        out.append((s.E.numpy(), s.H.numpy(), s.J.numpy(), hist.cpu().numpy(),
                    sum(t[1] for t in timing)))
    a, b = out
    assert a[4] == 1 + 20 + 1 and b[4] == 42      # launches: the pairs ran as k_tma2
    assert np.abs(b[0]).max() > 0
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_two_steps_per_launch_non_conductive():
    """J = 0 (vacuum in a PEC box, every face PEC) with the fused beam: the
    two-step kernel equals the one-step kernel (40 steps)."""
    import wakis_b200 as wb
    from wakis_b200.sources import Beam
    c = cases.WAKE_CASES[0]
    out = []
    for spl in (2, 1):
        g = wb.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
        g.add_solid("cav", cases.wake_mask(c, g.x, g.y, g.z), c["material"])
        s = wb.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], use_stl=True,
                           bg=c["bg"], verbose=0)
        assert not s.use_conductivity
        s.steps_per_launch = spl
        s._advance(40, 0, beam=Beam(q=1e-9, sigmaz=0.004, beta=1.0, ti=0.0).params(s))
        s.check_status()
        out.append((s.E.numpy(), s.H.numpy()))
    assert np.abs(out[1][0]).max() > 0
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_two_steps_per_launch_matches_oracle():
    """Two steps per launch (steps_per_launch = 2) on the lossy geometry at
    64x64x128 from seeded random fields with clean faces: the face entries
    of the random E are zeroed first, then the faces are marked clean; 40
    steps against the oracle within 1e-12."""
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec("lossy_256")
    so, c = _oracle_lossy((64, 64, 128))
    _, _, s = workloads.build_b200("lossy_256", shape=(64, 64, 128))
    E0, H0 = cases.initial_fields(c, so.N)
    # tangential E on every face set to +0 (the state a wakesolve keeps)
    Nx, Ny, Nz = so.shape
    for d in range(3):
        v = E0[d * so.N:(d + 1) * so.N].reshape(Nz, Ny, Nx)
        if d != 0:
            v[:, :, 0] = 0.0
            v[:, :, -1] = 0.0
        if d != 1:
            v[:, 0, :] = 0.0
            v[:, -1, :] = 0.0
        if d != 2:
            v[0] = 0.0
            v[-1] = 0.0
    so.E[:], so.H[:] = E0, H0
    s.E.fromarray(E0)
    s.H.fromarray(H0)
    s._faces_clean = True
    s.steps_per_launch = 2
    bkw = _short_beam(sp)
    timing = []
    s._advance(40, 0, beam=Beam(**bkw).params(s), timing=timing)
    s.check_status()
    assert sum(t[1] for t in timing) < 40
    beam = ofit.Beam(**bkw)
    for m in range(40):
        beam.update(so, m * so.dt)
        so.one_step()
    for f in "EHJ":
        assert rel_err(getattr(s, f).numpy(), getattr(so, f)) <= FIELD_TOL, f
