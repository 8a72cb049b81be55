"""The oracle (CPU restatement of upstream) against the golden fixtures made
from the upstream package and against upstream's own regression vectors."""

import json
import os

import numpy as np
import pytest

import cases
from helpers import oracle_step_case, oracle_wake_case
from oracle import fit as ofit
from oracle import wake as owake


@pytest.fixture(scope="module")
def step_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "step_cases.npz"))


@pytest.fixture(scope="module")
def wake_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "wake_cases.npz"))


@pytest.mark.parametrize("idx", range(len(cases.STEP_CASES)))
def test_oracle_steps_match_upstream(idx, step_golden):
    c = cases.STEP_CASES[idx]
    meta = {m["index"]: m for m in json.loads(str(step_golden["meta"]))}[idx]
    if meta.get("error"):
        with pytest.raises(ValueError):
            oracle_step_case(c)
        return
    s = oracle_step_case(c)
    assert s.dt == step_golden[f"c{idx}_dt"]
    for f in ("ieps", "imu", "sigma"):
        assert np.array_equal(getattr(s, f), step_golden[f"c{idx}_{f}"]), f
    E0, H0 = cases.initial_fields(c, s.N)
    s.E[:], s.H[:] = E0, H0
    beam = ofit.Beam(**c["beam"])
    for n in range(c["steps"]):
        beam.update(s, n * s.dt)
        s.one_step()
    for f in "EHJ":
        assert np.array_equal(getattr(s, f), step_golden[f"c{idx}_{f}"]), f


@pytest.mark.parametrize("idx", range(len(cases.WAKE_CASES)))
def test_oracle_wake_matches_upstream(idx, wake_golden):
    c = cases.WAKE_CASES[idx]
    s, w = oracle_wake_case(c)
    Nt = owake.wakesolve(s, w, c["wakelength"], compute_plane=c["compute_plane"])
    assert Nt == int(wake_golden[f"c{idx}_Nt"])
    names = ["s", "WP", "Z", "f", "lambdas", "lambdaf"]
    if c["compute_plane"] == "both":
        names += ["WP_3d", "WPx", "WPy", "Zx", "Zy"]
    for n in names:
        assert np.array_equal(getattr(w, n), wake_golden[f"c{idx}_{n}"]), n
    assert np.array_equal(s.E[2 * s.N:], wake_golden[f"c{idx}_Ez"])


def _test001_mask():
    """Upstream tests/test_001: 50x50x150 over the STL bounds, PEC
    background, vacuum cavity = box |x|,|y| <= 25 mm, |z| <= 15 mm plus a
    square pipe |x|,|y| <= 7.5 mm (the vertices of tests/stl/
    001_cubic_cavity.stl), cells inside when any corner is inside."""
    g0 = ofit.Grid(-0.025, 0.025, -0.025, 0.025, -0.05, 0.05, 50, 50, 150)
    X, Y, Z = np.meshgrid(g0.x, g0.y, g0.z, indexing="ij")
    tol = 1e-12
    inside = (((np.abs(X) <= 0.025 + tol) & (np.abs(Y) <= 0.025 + tol) & (np.abs(Z) <= 0.015 + tol))
              | ((np.abs(X) <= 0.0075 + tol) & (np.abs(Y) <= 0.0075 + tol)))
    m = np.zeros((50, 50, 150), bool)
    for a in (0, 1):
        for b in (0, 1):
            for cc in (0, 1):
                m |= inside[a:a + 50, b:b + 50, cc:cc + 150]
    return m


@pytest.mark.slow
def test_oracle_reproduces_upstream_test001(golden_dir):
    gold = np.load(os.path.join(golden_dir, "upstream_test001.npz"))
    m = _test001_mask()
    g = ofit.Grid(-0.025, 0.025, -0.025, 0.025, -0.05, 0.05, 50, 50, 150,
                  solids={"cavity": m}, materials={"cavity": "vacuum"})
    w = owake.WakeOracle(q=1e-9, sigmaz=18.5e-3, beta=1.0, skip_cells=12)
    s = ofit.Solver(g, bc_low=["pec"] * 3, bc_high=["pec"] * 3, use_stl=True, bg="pec",
                    dtype=np.float32, wake_fmax=w.fmax)
    owake.wakesolve(s, w, 1.0)
    tol = float(gold["WP_tol"])
    assert np.allclose(w.WP[::50], gold["WP"], rtol=tol, atol=tol)
    assert np.cumsum(np.abs(w.WP))[-1] == pytest.approx(float(gold["WP_cumsum"]),
                                                        float(gold["WP_cumsum_rel"]))
    tz = float(gold["Z_tol"])
    for fn in (np.abs, np.real, np.imag):
        assert np.allclose(fn(w.Z)[::20], fn(gold["Z"]), rtol=tz, atol=tz)
    assert np.cumsum(np.abs(w.Z))[-1] == pytest.approx(float(gold["Z_cumsum"]),
                                                       float(gold["Z_cumsum_rel"]))


@pytest.fixture(scope="module")
def lossy_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "lossy_cases.npz"))


@pytest.fixture(scope="module")
def sibc_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "sibc_cases.npz"))


@pytest.mark.parametrize("idx", range(len(cases.LOSSY_CASES)))
def test_oracle_lossy_geometry_matches_upstream(idx, lossy_golden):
    """The lossy-wall workload geometry (sigma = 1e4 S/m background, dt at
    the relaxation clamp, 10-cell z-PML, cavity + pipe, beam): the oracle
    equals upstream value for value."""
    from helpers import oracle_lossy_case
    c = cases.LOSSY_CASES[idx]
    s = oracle_lossy_case(c)
    assert s.dt == lossy_golden[f"c{idx}_dt"]
    E0, H0 = cases.case_fields(c, s.N)
    s.E[:], s.H[:] = E0, H0
    beam = ofit.Beam(**c["beam"])
    for n in range(c["steps"]):
        beam.update(s, n * s.dt)
        s.one_step()
    for f in "EHJ":
        assert np.abs(lossy_golden[f"c{idx}_{f}"]).max() > 0, f
        assert np.array_equal(getattr(s, f), lossy_golden[f"c{idx}_{f}"]), f


def test_oracle_sibc_step_matches_upstream(sibc_golden):
    """Surface-impedance wall (upstream's SIBC branch with the same surface
    mask injected): materials, dt and fields after steps value for value."""
    from helpers import oracle_sibc_case
    idx = 0
    c = cases.SIBC_CASES[idx]
    s = oracle_sibc_case(c)
    assert s.dt == sibc_golden[f"c{idx}_dt"]
    assert np.array_equal(s.ieps, sibc_golden[f"c{idx}_ieps"])
    assert np.array_equal(s.sigma, sibc_golden[f"c{idx}_sigma"])
    E0, H0 = cases.initial_fields(c, s.N)
    s.E[:], s.H[:] = E0, H0
    beam = ofit.Beam(**c["beam"])
    for n in range(c["steps"]):
        beam.update(s, n * s.dt)
        s.one_step()
    for f in "EHJ":
        assert np.array_equal(getattr(s, f), sibc_golden[f"c{idx}_{f}"]), f


def test_oracle_sibc_wake_matches_upstream(sibc_golden):
    from helpers import oracle_sibc_case
    idx = 1
    c = cases.SIBC_CASES[idx]
    w = owake.WakeOracle(**c["wake"])
    s = oracle_sibc_case(c, wake=w)
    assert s.dt == sibc_golden[f"c{idx}_dt"]
    Nt = owake.wakesolve(s, w, c["wakelength"], compute_plane=c["compute_plane"])
    assert Nt == int(sibc_golden[f"c{idx}_Nt"])
    for n in ["s", "WP", "Z", "f", "lambdaf", "WP_3d", "WPx", "WPy", "Zx", "Zy"]:
        assert np.array_equal(getattr(w, n), sibc_golden[f"c{idx}_{n}"]), n
    assert np.array_equal(s.E[2 * s.N:], sibc_golden[f"c{idx}_Ez"])
