"""z-slab decomposition (wakis_b200/slab.py).

On the CPU: the kernels' update formula (numpy emulation) stepped slab by
slab with the sliced coefficient sets and the ghost-plane exchange equals the
single-domain emulation bit for bit, for every step case (PEC, PMC, PML,
periodic and ABC faces, conductive materials) and 2 or 3 slabs, in one
process and as two gloo ranks exchanging through torch.distributed.  On the
GPU: ``SlabWakeSolve`` with 2 and 3 slabs in one process against the
single-domain ``wakesolve``.
"""

import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import cases
import stencil_emulator as emu
from helpers import oracle_step_case
from wakis_b200 import coefficients, slab
from wakis_b200.sources import Beam
from wakis_b200.gridFIT3D import GridFIT3D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


class _EmuSlab:
    """A slab stepped by the numpy emulation of the kernels, holding its
    state like a solver (two ping-pong buffers per field, live index _par),
    so that slab.LocalExchange / slab.DistExchange operate on it."""

    def __init__(self, coef, E, H, sigma):
        self.coef = coef
        self.Nx, self.Ny, self.Nz = coef.shape
        self.precision = None
        self._E = [torch.from_numpy(E.copy()), torch.from_numpy(E.copy())]
        self._H = [torch.from_numpy(H.copy()), torch.from_numpy(H.copy())]
        self._par = 0
        self.sigma = sigma

    def step(self):
        E, H = self._E[self._par].numpy(), self._H[self._par].numpy()
        Hn = emu.h_update(self.coef, E, H, self.coef.dt)
        En = emu.e_update(self.coef, E, Hn, self.sigma * E, self.coef.dt)
        self._par ^= 1
        self._E[self._par].copy_(torch.from_numpy(En))
        self._H[self._par].copy_(torch.from_numpy(Hn))


def _local(a, shape, lo, hi):
    Nx, Ny, Nz = shape
    return np.ascontiguousarray(a.reshape(3, Nz, Nx * Ny)[:, lo:hi].reshape(-1))


def _single_domain(k, E, H, sigma, steps):
    for _ in range(steps):
        Hn = emu.h_update(k, E, H, k.dt)
        E = emu.e_update(k, E, Hn, sigma * E, k.dt)
        H = Hn
    return E, H


def _owned(so, s, shape):
    Nx, Ny, _ = shape
    E = so._E[so._par].numpy().reshape(3, so.Nz, Nx * Ny)[:, s.k0 - s.lo:s.k1 - s.lo]
    H = so._H[so._par].numpy().reshape(3, so.Nz, Nx * Ny)[:, s.k0 - s.lo:s.k1 - s.lo]
    return E, H


def test_partition_and_layout():
    assert slab.partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    lay = slab.layout(20, 3)
    assert [(s.k0, s.k1, s.lo, s.hi) for s in lay] == [(0, 7, 0, 9), (7, 14, 5, 16),
                                                       (14, 20, 12, 20)]
    with pytest.raises(ValueError):
        slab.partition(3, 4)
    lay = slab.layout(20, 3, depth=4)
    assert [(s.k0, s.k1, s.lo, s.hi, s.depth) for s in lay] == [
        (0, 7, 0, 12, 4), (7, 14, 2, 19, 4), (14, 20, 9, 20, 4)]
    with pytest.raises(ValueError):
        slab.layout(20, 3, depth=7)


def test_side_streams_only_for_several_cuda_slabs():
    """Slabs get their own streams only when one process holds two or more
    of them on CUDA devices; otherwise advance() runs them in turn on the
    current stream (no stream is created on a host without a GPU)."""
    from types import SimpleNamespace
    cpu = {r: SimpleNamespace(device=torch.device("cpu")) for r in range(3)}
    assert slab.side_streams(cpu, [0, 1, 2]) is None
    one = {0: SimpleNamespace(device=torch.device("cuda", 0))}
    assert slab.side_streams(one, [0]) is None
    calls = []
    fake = {r: SimpleNamespace(_advance=lambda c, n0, beam=None, capture=None, r=r:
                               calls.append((r, c, n0, capture))) for r in range(2)}
    slab.advance(fake, [0, 1], 4, 8, captures={0: "c0", 1: "c1"})
    assert calls == [(0, 4, 8, "c0"), (1, 4, 8, "c1")]


@pytest.mark.parametrize("n,depth", [(2, 1), (3, 1), (2, 2), (2, 4), (3, 3)])
@pytest.mark.parametrize("idx", VALID)
def test_emulated_slabs_equal_single_domain(idx, n, depth):
    """Slabs with `depth` ghost planes per side, exchanging every `depth`
    steps: after 4 steps the owned planes equal the single domain."""
    c = cases.STEP_CASES[idx]
    k = _coef(c)
    shape = k.shape
    Nx, Ny, Nz = shape
    N = Nx * Ny * Nz
    E0, H0 = cases.initial_fields(c, N)
    E0, H0 = E0.astype(k.dtype), H0.astype(k.dtype)
    sigma = coefficients.dense_materials(k)[2].astype(k.dtype)
    Eg, Hg = _single_domain(k, E0, H0, sigma, 4)
    lay = slab.layout(Nz, n, depth)
    solvers = {}
    for s in lay:
        ks = slab.slice_coefficients(k, s.lo, s.hi)
        solvers[s.index] = _EmuSlab(ks, _local(E0, shape, s.lo, s.hi),
                                    _local(H0, shape, s.lo, s.hi),
                                    _local(sigma, shape, s.lo, s.hi))
    ex = slab.LocalExchange()
    done = 0
    while done < 4:
        blk = min(depth, 4 - done)
        for _ in range(blk):
            for s in lay:
                solvers[s.index].step()
        ex(lay, solvers)
        done += blk
    Eg3 = Eg.reshape(3, Nz, Nx * Ny)
    Hg3 = Hg.reshape(3, Nz, Nx * Ny)
    for s in lay:
        E, H = _owned(solvers[s.index], s, shape)
        assert np.array_equal(E, Eg3[:, s.k0:s.k1]), (idx, n, s)
        assert np.array_equal(H, Hg3[:, s.k0:s.k1]), (idx, n, s)


def test_internal_faces_mask_only_the_padding():
    c = dict(cases.STEP_CASES[0])
    c.update(bc_low=["pec", "pmc", "pec"], bc_high=["pec", "pec", "pmc"])
    k = _coef(c)
    lay = slab.layout(k.shape[2], 2)
    lo_slab = slab.slice_coefficients(k, lay[0].lo, lay[0].hi)
    hi_slab = slab.slice_coefficients(k, lay[1].lo, lay[1].hi)
    assert lo_slab.pec_face[4] == k.pec_face[4] and lo_slab.pec_face[5] == 0
    assert hi_slab.pec_face[4] == 0 and hi_slab.pec_face[5] == k.pec_face[5]
    assert hi_slab.pmc_face[5] == k.pmc_face[5] and hi_slab.pmc_face[4] == 1
    assert lo_slab.h_sum_desc == k.h_sum_desc and hi_slab.has_pec
    assert lo_slab.shape == (k.shape[0], k.shape[1], lay[0].hi)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, idx, out, depth=1):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        c = cases.STEP_CASES[idx]
        k = _coef(c)
        shape = k.shape
        Nx, Ny, Nz = shape
        E0, H0 = cases.initial_fields(c, Nx * Ny * Nz)
        E0, H0 = E0.astype(k.dtype), H0.astype(k.dtype)
        sigma = coefficients.dense_materials(k)[2].astype(k.dtype)
        lay = slab.layout(Nz, ws, depth)
        s = lay[rank]
        so = _EmuSlab(slab.slice_coefficients(k, s.lo, s.hi), _local(E0, shape, s.lo, s.hi),
                      _local(H0, shape, s.lo, s.hi), _local(sigma, shape, s.lo, s.hi))
        ex = slab.DistExchange()
        done = 0
        while done < 4:
            blk = min(depth, 4 - done)
            for _ in range(blk):
                so.step()
            ex(lay, {rank: so})
            done += blk
        E, H = _owned(so, s, shape)
        out.put((rank, E.copy(), H.copy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("idx,depth", [(VALID[0], 1), (VALID[1], 1), (VALID[2], 1),
                                       (VALID[2], 2), (VALID[4], 4)])
def test_two_gloo_ranks_equal_single_domain(idx, depth):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, idx, q, depth))
             for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, E, H = q.get(timeout=180)
        got[r] = (E, H)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c = cases.STEP_CASES[idx]
    k = _coef(c)
    Nx, Ny, Nz = k.shape
    E0, H0 = cases.initial_fields(c, Nx * Ny * Nz)
    sigma = coefficients.dense_materials(k)[2].astype(k.dtype)
    Eg, Hg = _single_domain(k, E0.astype(k.dtype), H0.astype(k.dtype), sigma, 4)
    lay = slab.layout(Nz, 2, depth)
    for s in lay:
        E, H = got[s.index]
        assert np.array_equal(E, Eg.reshape(3, Nz, -1)[:, s.k0:s.k1])
        assert np.array_equal(H, Hg.reshape(3, Nz, -1)[:, s.k0:s.k1])


def _cavity_args():
    from wakis_b200 import workloads
    sp = workloads.spec("cavity_40")
    g = GridFIT3D(*workloads.BOUNDS, *sp["shape"], verbose=0)
    g.add_solid("cavity", workloads.cavity_mask(g.x, g.y, g.z), "vacuum")
    kw = dict(bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
              n_pml=sp["n_pml"])
    return g, sp, kw


@pytest.mark.gpu
@pytest.mark.parametrize("n,depth", [(2, 1), (3, 1), (2, 4)])
def test_slab_wakesolve_equals_single_domain(n, depth):
    """cavity_40 (PEC x/y, ABC z, beam and 3x3 Ez capture, 1896 steps) split
    into n z-slabs on one GPU: fields, WP and Z value for value equal to the
    single-domain wakesolve."""
    import wakis_b200 as wb
    g, sp, kw = _cavity_args()
    w1 = wb.WakeSolver(save=False, verbose=0, **sp["wake"])
    s1 = wb.SolverFIT3D(g, w1, verbose=0, **kw)
    s1.wakesolve(wakelength=sp["wakelength"])
    w2 = wb.WakeSolver(save=False, verbose=0, **sp["wake"])
    sw = slab.SlabWakeSolve(g, w2, n_slabs=n, depth=depth, **kw)
    sw.wakesolve(wakelength=sp["wakelength"])
    assert sw.Nt == s1.Nt
    for so in sw.solvers.values():
        assert int(so._status.item()) == 0
    E, H = sw.fields()
    assert np.array_equal(E, s1.E.numpy().astype(np.float64))
    assert np.array_equal(H, s1.H.numpy().astype(np.float64))
    for name in ("WP", "WPx", "WPy", "Z", "Zx", "Zy"):
        assert np.array_equal(np.asarray(getattr(w2, name)), np.asarray(getattr(w1, name))), name


@pytest.mark.gpu
def test_slab_wakesolve_fp32c_close_to_single_domain():
    """The same split in FP32c: the ghost planes of a slab go through the
    compensated shell kernels (FP64-formed coefficients per cell) where the
    single domain uses the compensated TMA kernel (float factor rows), so the
    results agree to the compensated state's accuracy, not bit for bit."""
    import wakis_b200 as wb
    g, sp, kw = _cavity_args()
    w1 = wb.WakeSolver(save=False, verbose=0, **sp["wake"])
    s1 = wb.SolverFIT3D(g, w1, verbose=0, precision="fp32c", **kw)
    s1.wakesolve(wakelength=sp["wakelength"])
    w2 = wb.WakeSolver(save=False, verbose=0, **sp["wake"])
    sw = slab.SlabWakeSolve(g, w2, n_slabs=2, precision="fp32c", **kw)
    sw.wakesolve(wakelength=sp["wakelength"])
    rel = lambda a, b: np.max(np.abs(a - b)) / np.max(np.abs(b))
    assert rel(np.asarray(w2.WP), np.asarray(w1.WP)) <= 1e-5
    assert rel(np.abs(np.asarray(w2.Z)), np.abs(np.asarray(w1.Z))) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("name,shape,n,depth", [("cavity_40", (24, 24, 40), 2, 1),
                                                ("lossy_256", (32, 32, 48), 3, 1),
                                                ("lossy_256", (32, 32, 48), 3, 4)])
def test_stacked_chain_built_per_slab_equals_single_domain(name, shape, n, depth):
    """The weak-scaling workload of the slab decomposition: a chain of n
    workload blocks along z.  Each slab built on its own (the chain's edges
    for its planes, masks evaluated locally, internal ends without mask or
    PML), stepped with the fused beam and the ghost exchange, equals the
    single-domain chain value for value after 300 steps (with 4 ghost planes
    per side and steps_per_launch = 2 the lossy slabs run their steps two
    per launch between exchanges every 4 steps)."""
    from wakis_b200 import workloads
    _, w, s1 = workloads.build_stacked(name, n, shape=shape)
    lay = slab.layout(s1.Nz, n, depth)
    solvers = {sl.index: workloads.build_stacked(name, n, shape=shape,
                                                 planes=(sl.lo, sl.hi))[2] for sl in lay}
    for so in solvers.values():
        assert so.dt == s1.dt
        so.steps_per_launch = 2 if depth >= 4 else 0
    sp = workloads.spec(name)
    bp = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
              ).params(s1)
    steps = 300
    s1._advance(steps, 0, beam=bp)
    ex = slab.LocalExchange()
    for k in range(0, steps, depth):
        c = min(depth, steps - k)
        for so in solvers.values():
            so._advance(c, k, beam=bp)
        ex(lay, solvers)
    nxy = s1.Nx * s1.Ny
    Eg = s1.E.numpy().reshape(3, s1.Nz, nxy)
    Hg = s1.H.numpy().reshape(3, s1.Nz, nxy)
    assert np.abs(Eg).max() > 0
    for sl in lay:
        so = solvers[sl.index]
        E = so.E.numpy().reshape(3, so.Nz, nxy)[:, sl.k0 - sl.lo:sl.k1 - sl.lo]
        H = so.H.numpy().reshape(3, so.Nz, nxy)[:, sl.k0 - sl.lo:sl.k1 - sl.lo]
        assert np.array_equal(E, Eg[:, sl.k0:sl.k1]), sl
        assert np.array_equal(H, Hg[:, sl.k0:sl.k1]), sl
