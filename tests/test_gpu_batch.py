"""The batched form over one device work list (wk_batch_prepare /
wk_batch_run, wakis_b200.batch with launch="batched"), as one persistent
cooperative launch or as one launch per list and step: every instance equals
its own wakesolve value for value, and the bounded waits of the persistent
launch (tile loads, waits for an instance's earlier work) end it with the
status word set instead of hanging.

Upstream runs one wakesolve per geometry (wakis/routines.py:231-482); the
batched launches must reproduce each of them exactly: their tiles run the
block work of the one-grid FP32-compensated kernel and its boundary planes the
same shell rows, so the arithmetic of every cell is the same.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pillboxes(precision="fp32c"):
    """Three uneven pillboxes at 2 mm cells (x/y PEC, z ABC: the four
    z-boundary planes take the shell rows); transverse sizes 28, 32, 28
    cells, so one instance has its compensation words loaded by TMA and two
    by per-thread loads."""
    from wakis_b200 import batch
    ps = [dict(R=0.020, L=0.030, beta=0.9, sigma=1e4), dict(R=0.026, L=0.036, beta=0.6, sigma=3e5),
          dict(R=0.022, L=0.040, beta=1.0, sigma=2e3)]
    return [batch.build_pillbox(**q, cell=2e-3, precision=precision) for q in ps]


def _lossy(shapes):
    """The benchmark's geometry and faces (conductive walls, 10-cell z-PML:
    every face PEC-masked, one phase per step) with a 10 S/m background, so
    that the relaxation clamp keeps dt large enough for a few hundred steps
    to carry the bunch through the domain; FP32-compensated."""
    import wakis_b200 as wb
    from wakis_b200 import workloads
    out = []
    for shp in shapes:
        g = wb.GridFIT3D(*workloads.BOUNDS, *shp, verbose=0)
        g.add_solid("cavity", workloads.cavity_mask(g.x, g.y, g.z), "vacuum")
        w = wb.WakeSolver(q=1e-9, sigmaz=5e-3, beta=1.0, save=False, verbose=0)
        s = wb.SolverFIT3D(g, w, bc_low=["pec", "pec", "pml"], bc_high=["pec", "pec", "pml"],
                           use_stl=True, bg=[1.0, 1.0, 10.0], n_pml=10, verbose=0,
                           precision="fp32c")
        out.append((g, w, s))
    return out


def _solo(inst, n_steps):
    from wakis_b200 import batch
    for g, w, s in inst:
        s.wakesolve(wakelength=batch.BatchedWakeSolve.wakelength_for(s, n_steps))
        assert s.Nt == n_steps
    return inst


def _same(a, b):
    for (_, w, s), (_, w2, s2) in zip(a, b):
        assert int(s._status.item()) == 0
        for f in "EH":
            assert np.array_equal(getattr(s, f).numpy(), getattr(s2, f).numpy()), f
        assert np.array_equal(np.asarray(w.WP), np.asarray(w2.WP))
        assert np.array_equal(np.asarray(w.Z), np.asarray(w2.Z))
        assert np.array_equal(np.asarray(w.WPx), np.asarray(w2.WPx))


@pytest.mark.parametrize("form", ["persistent", "phases"])
def test_batch_equals_individual_wakesolve(form):
    """Pillboxes (two phases per step), autotuned planes per item, graph
    replays of 97-step chunks plus a tail."""
    from wakis_b200 import batch
    inst = _pillboxes()
    b = batch.BatchedWakeSolve([x[2] for x in inst], 601, launch="batched", chunk=97, form=form)
    tm = b.run()
    assert tm["launch"] == "batched" and b.tuned["form"] == form
    assert b.tuned["planes_per_item"] in batch.BATCH_KC_CANDIDATES
    assert b.tuned["launches"] == 7
    _same(inst, _solo(_pillboxes(), 601))


@pytest.mark.parametrize("form", ["persistent", "phases"])
def test_batch_32x16_tiles_equal_individual_wakesolve(form):
    """The pillboxes on 32x16 tiles (28- and 32-cell planes: tiles cut by
    the grid edge in x and in y, compensation words by TMA and by
    per-thread loads), autotuned planes per item."""
    from wakis_b200 import batch
    inst = _pillboxes()
    b = batch.BatchedWakeSolve([x[2] for x in inst], 601, launch="batched", chunk=97, form=form,
                               tiles="32x16")
    b.run()
    assert b.tuned["tile_policy"] == "32x16" and b.tuned["tiles_32x16"] == 3
    _same(inst, _solo(_pillboxes(), 601))


@pytest.mark.parametrize("tiles", ["64x8", "fill", "32x16"])
@pytest.mark.parametrize("form", ["persistent", "phases"])
def test_batch_all_faces_masked(form, tiles):
    """Conductive walls with z-PML on two grid shapes (one phase per step,
    one instance with TMA-loaded compensation words and one without) in one
    chunk with fixed planes per item; with tiles="fill" one instance runs
    on 32x16 tiles and the other on 64x8 tiles in the same launch."""
    from wakis_b200 import batch
    shapes = [(32, 32, 64), (36, 24, 56)]
    inst = _lossy(shapes)
    for _, _, s in inst:
        s.tile = (0, 16)
    b = batch.BatchedWakeSolve([x[2] for x in inst], 500, launch="batched", tune=False,
                               chunk=1000, form=form, tiles=tiles)
    b.run()
    rows = [s.tile[0] for _, _, s in inst]
    assert rows == {"64x8": [8, 8], "fill": [16, 8], "32x16": [16, 16]}[tiles]
    _same(inst, _solo(_lossy(shapes), 500))


def test_batch_rejects_mixed_instances():
    """An FP64 instance cannot join the batched launches."""
    from wakis_b200 import batch
    a = _pillboxes()[:1] + _pillboxes(precision=None)[:1]
    assert not batch.batched_ok([x[2] for x in a])
    with pytest.raises(ValueError):
        batch.BatchedWakeSolve([x[2] for x in a], 100, launch="batched")


def _plan(inst, wait_ns=0):
    from wakis_b200 import _native, batch
    descs = []
    for _, _, s in inst:
        s._first_step()
        d = _native.FitDesc.from_buffer_copy(s._step_desc())
        d.wait_ns = wait_ns
        descs.append(d)
    return batch.BatchPlan([x[2] for x in inst], descs, t_ref=0)


def test_persistent_tile_wait_timeout_sets_status():
    """Tile loads whose waits give up at once (wait_ns < 0) end the launch:
    the instance's status word is set, the other blocks leave at the next
    barrier, and the context steps correctly afterwards."""
    inst = _pillboxes()
    plan = _plan(inst, wait_ns=-1)
    plan.run(3, 0)
    torch.cuda.synchronize()
    assert sum(int(s._status.item()) for _, _, s in inst) >= 1
    with pytest.raises(RuntimeError):
        for _, _, s in inst:
            s.check_status("timeout test")
    for _, _, s in inst:
        s._status.zero_()
        s.reset_fields()
    ok = _plan(inst)
    ok.run(2, 0)
    torch.cuda.synchronize()
    assert all(int(s._status.item()) == 0 for _, _, s in inst)


def test_persistent_dependency_wait_timeout_sets_status():
    """Dependency waits bounded by 1 ns give up (items of step 1 claimed
    before their instance's step 0 is done): the status word of an instance
    is set, every block leaves, and the context steps correctly afterwards."""
    inst = _pillboxes()
    plan = _plan(inst)
    plan.run(4, 0, wait_ns=1)
    torch.cuda.synchronize()
    assert sum(int(s._status.item()) for _, _, s in inst) >= 1
    for _, _, s in inst:
        s._status.zero_()
        s.reset_fields()
    ok = _plan(inst)
    ok.run(2, 0)
    torch.cuda.synchronize()
    assert all(int(s._status.item()) == 0 for _, _, s in inst)
