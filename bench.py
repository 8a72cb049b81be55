"""Throughput of the FIT leap-frog wake stepper on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload lossy_256|cavity_40] [--dtype float64|float32]

A step is one wakesolve step over the whole grid: Gaussian beam current on
the beam line, capture of the 3x3 Ez window around the test line, H
half-step and E half-step (one fused kernel launch).  Default workload:
256x256x512 cells (33.5 M) FP64, lossy-wall cavity with pipe, 10-cell PML at
both z ends (``wakis_b200.workloads.lossy_256``).  The state (4 x 805 MB
ping-pong buffers) is far larger than L2, so no L2 flush is needed.

value  = cells x steps / device time of the K timed steps (CUDA events,
         max over ranks), in Gcell-steps/s, whole job.
e2e    = the same through SolverFIT3D.run_with_io: every step copies the
         beam-line current host->device and the captured Ez window
         device->host (pinned buffers), wall clock around the K steps.
Multi-GPU (torchrun): a chain of N workload blocks along z, one per rank
(weak scaling), exchanging --slab-depth ghost planes with the neighbouring
ranks every --slab-depth steps through NCCL point-to-point messages
(wakis_b200/slab.py); --decomp replicas instead runs independent replicas
(no data-path collective).  --slabs K splits the workload into K z-slabs on
one GPU.

--impl reference times the CPU oracle (a restatement of upstream's scipy
solver) on the host cores with all threads, rank 0 only: the workload's own
grid when the host has the memory for its sparse operators, else the same
geometry at 128x128x256; at most about 2 minutes of timed steps.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = {"float64": 96, "float32": 48, "fp32c": 48}
METRIC = "Gcell-steps/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic(workload, dtype, schedule, cells):
    """DRAM bytes (read + write) per launch of the interior kernel over
    `cells` cells: the bytes per cell of the committed ncu summary
    profiles/traffic.json (one launch on a smaller grid of the same
    workload) times the cells, if the summary holds this case."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        e = t.get(f"{workload}:{dtype}:{schedule}")
        if e is None:
            return None
        per_cell = (e["read_bytes_small"] + e["write_bytes_small"]) / e["cells_small"]
        return int(round(per_cell * cells))
    except Exception:
        return None


class RegionClocks:
    """SM clock and clock-event reasons read through NVML every 2 ms by a
    thread, from start() to stop(): the samples of the timed region itself
    (read-only queries; None when NVML is unavailable)."""

    def __init__(self, uuid, device_index):
        self.samples, self.reasons, self.smax = [], set(), None
        self.h, self.t, self.run = None, None, False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            h = None
            if uuid:
                u = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
                try:
                    h = pynvml.nvmlDeviceGetHandleByUUID(u)
                except Exception:
                    h = None
            if h is None:
                h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.h = h
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.h = None

    def _poll(self):
        nv = self.nv
        names = {nv.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 nv.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwPowerCap: "sw_power_cap"}
        while self.run:
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for b, nm in names.items():
                    if bits & b:
                        self.reasons.add(nm)
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        if self.h is None:
            return
        import threading
        self.run = True
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def stop(self):
        if self.t is None:
            return None
        self.run = False
        self.t.join(timeout=5)
        if not self.samples:
            return None
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "source": "NVML, every 2 ms inside the timed region"}


class Clocks:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 8 or (self.uuid and self.uuid not in c[0]):
                continue
            try:
                sm.append(float(c[1]))
                smax.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(vals, ws, device=None):
    """Element-wise max of a list of floats over all ranks, one all_reduce
    (every rank calls it at the same point)."""
    if ws <= 1:
        return [float(v) for v in vals]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def _status_ok(solver):
    """True when no step kernel of `solver` timed out since the last check
    (reads and clears its device status word)."""
    try:
        solver.check_status("bench")
        return True
    except RuntimeError as e:
        print(str(e), file=sys.stderr, flush=True)
        return False


def _ref_sample(args, sp):
    """Grid of the reference arm: the workload's own grid (or --shape) when
    the host has the memory for the oracle's sparse operators there (about
    1.4 kB per cell at the peak of their assembly, measured at 128x128x256),
    else 128x128x256."""
    full = tuple(int(v) for v in args.shape.split("x")) if args.shape else tuple(sp["shape"])
    need = 1.4e3 * float(np.prod(full)) * 1.5
    try:
        import psutil
        avail = float(psutil.virtual_memory().available)
    except Exception:
        avail = 0.0
    if avail >= need:
        return full, True, avail
    return (128, 128, 256), False, avail


def run_reference(args):
    """CPU oracle on the host cores: Gcell-steps/s of upstream's scipy
    algorithm (same geometry; the workload's own grid when the host memory
    allows, else a 128x128x256 sample)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from oracle import fit as ofit
    from wakis_b200 import workloads
    sp = workloads.spec(args.workload)
    sample, same, avail = _ref_sample(args, sp)
    t_init = time.perf_counter()
    g0 = ofit.Grid(*workloads.BOUNDS, *sample)
    m = workloads.cavity_mask(g0.x, g0.y, g0.z)
    g = ofit.Grid(*workloads.BOUNDS, *sample, solids={"cavity": m}, materials={"cavity": "vacuum"})
    so = ofit.Solver(g, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
                     dtype=np.float32 if args.dtype == "float32" else np.float64,
                     n_pml=sp["n_pml"])
    t_init = time.perf_counter() - t_init
    cores = os.cpu_count() or 1
    so.set_threads(cores)
    beam = ofit.Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")})
    for n in range(args.warmup):
        beam.update(so, n * so.dt)
        so.one_step()
    # K steps, or fewer when they would take more than ~2 minutes
    t0 = time.perf_counter()
    done = 0
    for n in range(args.warmup, args.warmup + args.steps):
        beam.update(so, n * so.dt)
        so.one_step()
        done += 1
        if time.perf_counter() - t0 > 120.0:
            break
    t = time.perf_counter() - t0
    value = so.N * done / t / 1e9
    line = {"metric": METRIC, "value": value, "unit": "Gcell-steps/s", "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * t / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.dtype == "float32" else "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload,
                       "cells": int(np.prod([int(v) for v in args.shape.split("x")]
                                            if args.shape else sp["shape"])),
                       "sample_cells": so.N, "grid": list(sample), "same_grid": same,
                       "host_mem_available_gb": round(avail / 1e9, 1),
                       "init_s": round(t_init, 1)},
            "cpu_baseline": {"value": value, "unit": "Gcell-steps/s", "cores": cores,
                             "kind": "port",
                             "sample": f"oracle (scipy CSR, {cores} threads) on the "
                                       f"{args.workload} geometry at "
                                       f"{sample[0]}x{sample[1]}x{sample[2]}, "
                                       f"{done} steps with beam"},
            "e2e": {"value": value, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_accuracy(args):
    """FP32-compensated against FP64 on one grid (rank 0 only): one JSON
    line with the relative errors of WP, WPx, WPy, |Z|, Re Z, Im Z, |Zx| and
    the Gcell-steps/s of both whole wakesolve runs (CUDA events)."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    from wakis_b200 import workloads
    name = args.workload if args.workload != "lossy_256" else "precision_448"
    shape = tuple(int(v) for v in args.shape.split("x")) if args.shape else None
    r = workloads.precision_compare(name, shape=shape, wakelength=args.wakelength)
    line = {"metric": "FP32c vs FP64 relative error (max|a-b|/max|b|)", "workload": name,
            "grid": list(shape or workloads.spec(name)["shape"]), "wakelength": r["wakelength"],
            "errors": r["errors"], "fp64": r["fp64"], "fp32c": r["fp32c"],
            "speed_ratio": r["fp32c"]["gcell_steps_per_s"] / r["fp64"]["gcell_steps_per_s"],
            "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_batch(args):
    """Batched form (rank 0 only): `--batch` pillbox cavities stepped in one
    captured CUDA graph (wakis_b200.batch), FP32c unless --dtype says
    otherwise; aggregate Gcell-steps/s over all instances."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    from wakis_b200 import batch
    params = batch.pillbox_params(args.batch, seed=0)
    prec = None if args.dtype in ("float64", "float32") else "fp32c"
    dt = np.float32 if args.dtype == "float32" else np.float64

    def run(precision, dtype):
        t0 = time.perf_counter()
        built = [batch.build_pillbox(**q, precision=precision, dtype=dtype,
                                     multiple=args.batch_multiple) for q in params]
        t_build = time.perf_counter() - t0
        b = batch.BatchedWakeSolve([x[2] for x in built], args.batch_steps,
                                   launch=args.batch_launch if precision else "graph",
                                   form=args.batch_form, tiles=args.batch_tiles)
        t1 = time.perf_counter()
        tm = b.run()
        t_run = time.perf_counter() - t1
        res = [(np.array(x[1].WP), np.array(x[1].Z)) for x in built]
        shapes = [(x[2].Nx, x[2].Ny, x[2].Nz) for x in built]
        tuned = dict(b.tuned)
        del built, b
        torch.cuda.empty_cache()
        return tm, res, shapes, t_build, t_run, tuned

    tm, res, shapes, t_build, t_run, tuned = run(prec, dt)
    cells = tm["cells"]
    line = {"metric": METRIC, "value": tm["gcell_steps_per_s"], "unit": "Gcell-steps/s",
            "n_gpus": 1, "steps": args.batch_steps, "warmup": 0,
            "ms_per_step": tm["ms"] / args.batch_steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"float64": "f64", "float32": "f32"}.get(args.dtype, "f32+bf16 comp"),
            "data": "synthetic",
            "config": {"workload": f"batch_{args.batch}_pillboxes_seed0", "instances": args.batch,
                       "cells_total": cells, "grids_min": min(shapes), "grids_max": max(shapes),
                       "transverse_multiple": args.batch_multiple,
                       "launch": tm["launch"],
                       "graph": ("device work list over all instances (wk_batch_run), a chunk "
                                 "of steps captured once and replayed" if tm["launch"] == "batched"
                                 else "2 steps of every instance per replay, 8 streams"),
                       "tuned": tuned},
            "e2e": {"value": cells * args.batch_steps / t_run / 1e9, "unit": "Gcell-steps/s",
                    "note": "wall clock of the batched run incl. the wake integration",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "build_s": t_build}
    if args.batch_compare and prec == "fp32c":
        tm64, res64, _, _, _, _ = run(None, np.float64)

        def rel(a, b):
            den = np.max(np.abs(b))
            return float(np.max(np.abs(a - b)) / den) if den else 0.0

        ewp = [rel(a[0], b[0]) for a, b in zip(res, res64)]
        ez = [rel(np.abs(a[1]), np.abs(b[1])) for a, b in zip(res, res64)]
        line["per_instance_error_vs_fp64"] = {"WP_max": max(ewp), "absZ_max": max(ez),
                                              "WP": ewp, "absZ": ez}
        line["fp64_value"] = tm64["gcell_steps_per_s"]
    print(json.dumps(line), flush=True)


def run_adjoint(args):
    """Differentiation form (rank 0 only).  The cavity_40 geometry on
    128x128x256 cells (PEC walls) with a central 64^3 design region of
    per-cell eps_r ~ U[1, 10] and sigma ~ U[0, --adjoint-sigma-max] S/m (seed
    1; 1e3 as the configuration states); loss = int_{0.5}^{3 GHz} |Z_par|^2
    df; forward + adjoint in FP64, FP32, and the FP32-compensated forward
    (per-cell materials: the two-pass kernels) with the float stencil or the
    compensated stencil (comp_stencil: neighbour values v + c, increments
    formed with error-free float transformations), each with an FP64 or
    FP32 adjoint, with sqrt(N)-step checkpoints; 16 random directions
    checked against central differences of FP64 forward runs
    (Richardson-extrapolated from steps 1e-3 and 5e-4 along the direction).
    The time step is upstream's for the seeded parameters: the CFL step,
    clamped to the smallest relaxation time eps_0 eps_r / sigma of the design
    cells (solverFIT3D.py:301-310), fixed for every evaluation."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    from wakis_b200 import workloads
    from wakis_b200.adjoint import ImpedanceDesign
    shape = tuple(int(v) for v in args.shape.split("x")) if args.shape else (128, 128, 256)
    rng = np.random.default_rng(1)
    smax = float(args.adjoint_sigma_max)
    dt_fixed = [None]

    def problem(dtype, precision=None, adjoint_dtype=None, comp_stencil=False):
        _, _, s = workloads.build_b200("cavity_40", dtype=dtype, shape=shape,
                                       precision=precision, dt=dt_fixed[0])
        s.comp_stencil = comp_stencil
        m = np.zeros(shape, bool)
        c = [n // 2 for n in shape]
        h = [min(32, n // 4) for n in shape]
        m[c[0] - h[0]:c[0] + h[0], c[1] - h[1]:c[1] + h[1], c[2] - h[2]:c[2] + h[2]] = True
        return (ImpedanceDesign(s, m, n_steps=nsteps, adjoint_dtype=adjoint_dtype),
                int(m.sum()))

    runs = {}
    forms = (("f64", np.float64, None, None, False), ("f32", np.float32, None, None, False),
             ("fp32c", np.float64, "fp32c", None, False),
             ("fp32c_adj32", np.float64, "fp32c", np.float32, False),
             ("fp32c_cs", np.float64, "fp32c", None, True),
             ("fp32c_cs_adj32", np.float64, "fp32c", np.float32, True))
    # the seeded parameters and upstream's time step for them
    _, _, s_cfl = workloads.build_b200("cavity_40", shape=shape)
    dt_cfl = float(s_cfl.dt)
    del s_cfl
    m0 = np.zeros(shape, bool)
    c0 = [n // 2 for n in shape]
    h0 = [min(32, n // 4) for n in shape]
    m0[c0[0] - h0[0]:c0[0] + h0[0], c0[1] - h0[1]:c0[1] + h0[1], c0[2] - h0[2]:c0[2] + h0[2]] = True
    nd0 = int(m0.sum())
    er = rng.uniform(1.0, 10.0, nd0)
    sg = rng.uniform(0.0, smax, nd0)
    pos = sg > 0
    tau = (er[pos] * 8.8541878128e-12) / sg[pos]
    dt_fixed[0] = min(dt_cfl, float(tau.min())) if pos.any() else dt_cfl
    # steps: as given, else 4000 (the configuration) or, when the clamp
    # shortens dt so much that 4000 steps do not carry the bunch through the
    # domain, the steps for 2000 wake samples behind it
    nsteps = args.adjoint_steps
    if nsteps <= 0:
        sp = workloads.spec("cavity_40")
        v = 299792458.0 * sp["wake"]["beta"]
        span = workloads.BOUNDS[5] - workloads.BOUNDS[4]
        ti_v = 8.548921333333334 * sp["wake"]["sigmaz"]
        need = int(np.ceil((span + ti_v + 2000 * v * dt_fixed[0]) / (v * dt_fixed[0])))
        nsteps = max(4000, need) if dt_fixed[0] < dt_cfl else 4000
    if args.adjoint_forms:
        keep = args.adjoint_forms.split(",")
        unknown = sorted(set(keep) - {f[0] for f in forms})
        if unknown or "f64" not in keep:
            raise SystemExit(f"--adjoint-forms: unknown {unknown} (f64 is required: its forward "
                             f"runs give the finite differences)")
        forms = tuple(f for f in forms if f[0] in keep)
    for name, dt_, prec, adt, cst in forms:
        t0 = time.perf_counter()
        prob, nd = problem(dt_, prec, adt, cst)
        t_setup = time.perf_counter() - t0
        prob.set_params(er, sg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = prob.forward()
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        ge, gs = prob.backward()
        torch.cuda.synchronize()
        t_bwd = time.perf_counter() - t0
        N = prob.s.N
        runs[name] = dict(L=L, ge=ge, gs=gs, forward_s=t_fwd, backward_s=t_bwd,
                          setup_s=t_setup)
        if name != "f64":
            del prob
            torch.cuda.empty_cache()
        else:
            p64 = prob
            p64.ckpt = {}      # only its forward runs are needed from here on
            torch.cuda.empty_cache()
    errs = {name: [] for name in runs}

    def central(v_e, v_s, h):
        p64.set_params(er + h * v_e, sg + h * v_s)
        lp = p64.forward(keep=False)
        p64.set_params(er - h * v_e, sg - h * v_s)
        lm = p64.forward(keep=False)
        return (lp - lm) / (2.0 * h)

    for _ in range(args.adjoint_directions):
        ve = rng.standard_normal(nd)
        vs = rng.standard_normal(nd)
        # Richardson extrapolation of central differences at h and h/2: O(h^4)
        fd = (4.0 * central(ve, vs, 5e-4) - central(ve, vs, 1e-3)) / 3.0
        for name, r in runs.items():
            ad = float(r["ge"] @ ve) + float(r["gs"] @ vs)
            errs[name].append(abs(ad - fd) / abs(fd) if fd else abs(ad))
    line = {"metric": "adjoint gradient vs central differences (relative)", "grid": list(shape),
            "design_cells": nd, "steps": nsteps, "data": "synthetic",
            "sigma_range": [0.0, smax], "eps_r_range": [1.0, 10.0],
            "dt": dt_fixed[0], "dt_cfl": dt_cfl,
            "dt_policy": "CFL step clamped to the smallest eps_0 eps_r / sigma of the seeded "
                         "design cells (upstream's clamp), fixed for every evaluation",
            "fd": "FP64 forward runs, Richardson-extrapolated central differences"}
    for name, r in runs.items():
        line[name] = {"loss": r["L"],
                      "grad_rel_err_max": max(errs[name]) if errs[name] else None,
                      "grad_rel_err": errs[name], "forward_s": r["forward_s"],
                      "backward_s": r["backward_s"], "setup_s": r["setup_s"],
                      "forward_gcell_steps_per_s": N * nsteps / r["forward_s"] / 1e9,
                      "adjoint_gcell_steps_per_s": N * nsteps / r["backward_s"] / 1e9}
    print(json.dumps(line), flush=True)


def run_slab(args):
    """z-slab decomposition (wakis_b200/slab.py).  With --slabs K (one GPU):
    the workload split into K z-slabs in this process, ghost planes copied on
    the device after every step; the rate against the single-domain run is
    the cost of the ghost planes and the exchange.  Under torchrun with
    --decomp slab: a chain of N workload blocks along z, one block per rank
    (weak scaling), ghost planes exchanged with the neighbouring ranks through
    NCCL point-to-point messages every step; value = all cells x steps / max
    over ranks of the CUDA-event time."""
    import datetime
    from types import SimpleNamespace

    import torch
    import torch.distributed as dist

    from wakis_b200 import slab, workloads
    from wakis_b200.sources import Beam
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    sp = workloads.spec(args.workload)
    shape = tuple(int(v) for v in args.shape.split("x")) if args.shape else sp["shape"]
    dtype = np.float64 if args.dtype == "fp32c" else np.dtype(args.dtype).type
    precision = "fp32c" if args.dtype == "fp32c" else None
    if ws > 1:
        n_blocks, n, mine, ex = ws, ws, [rank], slab.DistExchange()
    else:
        n_blocks, n, mine, ex = 1, max(args.slabs, 1), list(range(max(args.slabs, 1))), \
            slab.LocalExchange()
    x, y, z = workloads.stacked_edges(args.workload, n_blocks, shape)
    Nx, Ny, Nz = len(x) - 1, len(y) - 1, len(z) - 1
    N = Nx * Ny * Nz
    lay = slab.layout(Nz, n, args.slab_depth)
    solvers = {r: workloads.build_stacked(args.workload, n_blocks, shape=shape,
                                          planes=(lay[r].lo, lay[r].hi), dtype=dtype,
                                          precision=precision, device=dev)[2] for r in mine}
    dts = [float(so.dt) for so in solvers.values()]
    if ws > 1:
        allg = [None] * ws
        dist.all_gather_object(allg, dts)
        dts = [v for part in allg for v in part]
    if len(set(dts)) != 1:
        raise RuntimeError(f"slabs disagree on the time step: {sorted(set(dts))}")
    so0 = solvers[mine[0]]
    cen = lambda e: e[:-1] + np.diff(e) / 2
    view = SimpleNamespace(x=cen(x), y=cen(y), z=cen(z), dx=np.diff(x), dy=np.diff(y))
    beam = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")})
    bp = beam.params(view)
    ixt = int(np.abs(view.x - sp["wake"]["xtest"]).argmin())
    iyt = int(np.abs(view.y - sp["wake"]["ytest"]).argmin())
    total = args.warmup + args.steps
    caps = {r: (torch.zeros((9, solvers[r].Nz, total), dtype=solvers[r]._cap_dtype, device=dev),
                ixt - 1, iyt - 1, 3, 3) for r in mine}

    G = lay[0].depth
    streams = slab.side_streams(solvers, mine)

    def steps(n0, k):
        m = n0
        while m < n0 + k:
            c = min(G, n0 + k - m)
            slab.advance(solvers, mine, c, m, bp, caps, streams)
            ex(lay, solvers)
            m += c

    def barrier():
        if ws > 1:
            dist.barrier()

    steps(0, args.warmup)
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clk = Clocks(uuid)
    rclk = RegionClocks(uuid, local)
    time.sleep(0.3)
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    rclk.start()
    e0.record(st)
    steps(args.warmup, args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    region_clocks = rclk.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    # step kernels per slab and step (one timed step per slab)
    launches = 0
    for r in mine:
        tm = []
        solvers[r]._advance(1, total, timing=tm)
        launches += sum(t[1] for t in tm)
    ex(lay, solvers)
    launches *= args.steps
    # end to end: per step and slab the beam line of its planes from pinned
    # host memory and its 3x3 Ez window back (SolverFIT3D.run_with_io), then
    # the exchange
    t_line = lambda m: (beam.q * beam.v * beam.profile(view, m * so0.dt) / view.dx[bp[0]]
                        / view.dy[bp[1]])
    step0 = total + 1
    lines = np.stack([t_line(m) for m in range(step0, step0 + args.steps)]).astype(
        np.float64 if args.dtype == "fp32c" else dtype)
    jz = {r: torch.from_numpy(np.ascontiguousarray(lines[:, lay[r].lo:lay[r].hi])).pin_memory()
          for r in mine}
    ez = {r: torch.empty((args.steps, 9, solvers[r].Nz), dtype=solvers[r]._cap_dtype
                         ).pin_memory() for r in mine}
    main = torch.cuda.current_stream(dev)
    # warm-up of the I/O path (its device staging buffers are allocated on
    # the first call, on the stream of the call), one exchange block
    nw = min(G, args.steps)
    for r in mine:
        if streams:
            streams[r].wait_stream(main)
        with torch.cuda.stream(streams[r] if streams else main):
            solvers[r].run_with_io(jz[r][:nw].clone().pin_memory(),
                                   torch.empty_like(ez[r][:nw]).pin_memory(), step0=step0)
        if streams:
            main.wait_stream(streams[r])
    ex(lay, solvers)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m in range(0, args.steps, G):
        c = min(G, args.steps - m)
        for r in mine:
            if streams:
                streams[r].wait_stream(main)
            with torch.cuda.stream(streams[r] if streams else main):
                solvers[r].run_with_io(jz[r][m:m + c], ez[r][m:m + c], step0=step0 + m,
                                       wait=False)
        if streams:
            for r in mine:
                main.wait_stream(streams[r])
        ex(lay, solvers)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    for r in mine:
        solvers[r].check_status("bench (slabs, end to end)")
    clocks = region_clocks or clk.stop()
    if region_clocks is not None:
        clk.stop()
    ms, t_e2e = max_over_ranks([ms, t_e2e], ws, dev)
    if rank == 0:
        bpc = BYTES_PER_CELL[args.dtype]
        peak, src = _peaks()
        per_gpu = bpc * (N / ws) / (ms / 1e3 / args.steps) / 1e9
        line = {
            "metric": METRIC, "value": N * args.steps / (ms / 1e3) / 1e9,
            "unit": "Gcell-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"float64": "f64", "float32": "f32",
                      "fp32c": "f32+bf16 comp (factors formed in f64)"}[args.dtype],
            "data": "synthetic",
            "config": {"workload": f"{args.workload} chain of {n_blocks} block(s) along z",
                       "cells": N, "grid": [Nx, Ny, Nz],
                       "parallelism": f"zslab{ws}" if ws > 1 else f"zslab{n}-on-1gpu",
                       "slabs": [[s.k0, s.k1] for s in lay],
                       "exchange": "NCCL point-to-point" if ws > 1 else "device copies",
                       "ghost_depth": G,
                       "slab_streams": "one per slab" if streams else "current stream",
                       "l2": "state above L2, no flush",
                       "step": "fused beam + Ez 3x3 capture + H and E half-steps + ghost "
                               "exchange"},
            "roofline": {"bound": "hbm", "achieved": per_gpu, "peak": peak, "unit": "GB/s",
                         "frac": per_gpu / peak, "peak_source": src, "bytes_per_cell_step": bpc,
                         "kernel": "whole step per GPU (owned cells; ghost and padding "
                                   "planes and the exchange are overhead)",
                         "traffic": None},
            "e2e": {"value": N * args.steps / t_e2e / 1e9, "unit": "Gcell-steps/s",
                    "h2d_bytes_per_step": int(sum(jz[r][0].numel() * jz[r].element_size()
                                                  for r in mine)) * ws,
                    "d2h_bytes_per_step": int(sum(ez[r][0].numel() * ez[r].element_size()
                                                  for r in mine)) * ws},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def precision_leg(args, dev, fp64_value):
    """The FP32-compensated state on the same workload and grid in the same
    run (rank 0, N=1): device-timed rate of K steps (same warm-up, beam and
    capture as the FP64 line), the roofline of its step kernel at 48 B per
    cell-step, and the WP / Z errors of a whole FP32c wakesolve against the
    FP64 one on the precision workload at 112x112x224 with a 0.3 m wake
    (``workloads.precision_compare``)."""
    import torch
    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec(args.workload)
    shape = tuple(int(v) for v in args.shape.split("x")) if args.shape else None
    g, w, s = workloads.build_b200(args.workload, dtype=np.float64, shape=shape,
                                   precision="fp32c")
    N = s.N
    bp = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
              ).params(s)
    ixt = int(np.abs(s.x - w.xtest).argmin())
    iyt = int(np.abs(s.y - w.ytest).argmin())
    total = args.warmup + args.steps
    hist = torch.zeros((9, s.Nz, total + args.steps), dtype=s._cap_dtype, device=dev)
    cap = (hist, ixt - 1, iyt - 1, 3, 3)
    s._advance(args.warmup, 0, beam=bp, capture=cap)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s._advance(args.steps, args.warmup, beam=bp, capture=cap)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if not _status_ok(s):
        return {"error": "a step kernel timed out in the FP32c timed region"}
    timing = []
    s._advance(args.steps, total, beam=bp, capture=cap, timing=timing)
    ms_int = sum(t[0] for t in timing)
    n_int = sum(t[1] for t in timing)
    del g, w, s, hist
    torch.cuda.empty_cache()
    value = N * args.steps / (ms / 1e3) / 1e9
    peak, src = _peaks()
    bpc = BYTES_PER_CELL["fp32c"]
    achieved = bpc * N * args.steps / (ms_int / 1e3) / 1e9 if ms_int > 0 else None
    out = {"value": value, "unit": "Gcell-steps/s", "ms_per_step": ms / args.steps,
           "vs_fp64": value / fp64_value,
           "dtype": "f32 state + bf16 compensation words; update factors formed in f64, rounded to f32",
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved else None, "peak_source": src,
                        "bytes_per_cell_step": bpc,
                        "kernel": f"k_tma_comp: {n_int} launches, "
                                  f"{ms_int / max(args.steps, 1):.4f} ms per step",
                        "traffic": _traffic(args.workload, "fp32c", "tma", N)},
           "gpu_launches": args.steps}
    # accuracy of a whole wakesolve, FP32c against FP64 on one grid
    acc_shape, acc_wl = (112, 112, 224), 0.3
    r = workloads.precision_compare("precision_448", shape=acc_shape, wakelength=acc_wl)
    out["accuracy"] = {"workload": f"precision_448 geometry at {acc_shape[0]}x{acc_shape[1]}"
                                   f"x{acc_shape[2]}, wakelength {acc_wl} m",
                       "steps": r["fp64"]["steps"],
                       "relative_errors_vs_fp64": r["errors"],
                       "bar": 1e-4,
                       "within_bar": bool(r["errors"]["WP"] <= 1e-4
                                          and r["errors"]["absZ"] <= 1e-4),
                       "wakesolve_rate_fp64": r["fp64"]["gcell_steps_per_s"],
                       "wakesolve_rate_fp32c": r["fp32c"]["gcell_steps_per_s"]}
    return out


def cpu_baseline(args, budget_s=20.0):
    """Single-thread oracle on a bounded sample (rank 0, N=1 only)."""
    from oracle import fit as ofit
    from wakis_b200 import workloads
    sample = (96, 96, 192)
    sp = workloads.spec(args.workload)
    g0 = ofit.Grid(*workloads.BOUNDS, *sample)
    m = workloads.cavity_mask(g0.x, g0.y, g0.z)
    g = ofit.Grid(*workloads.BOUNDS, *sample, solids={"cavity": m}, materials={"cavity": "vacuum"})
    so = ofit.Solver(g, bc_low=sp["bc_low"], bc_high=sp["bc_high"], use_stl=True, bg=sp["bg"],
                     dtype=np.dtype(args.dtype).type, n_pml=sp["n_pml"])
    beam = ofit.Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")})
    beam.update(so, 0.0)
    so.one_step()
    n, t0 = 0, time.perf_counter()
    while True:
        n += 1
        beam.update(so, n * so.dt)
        so.one_step()
        if time.perf_counter() - t0 > budget_s / 2 or n >= 50:
            break
    t = time.perf_counter() - t0
    return {"value": so.N * n / t / 1e9, "unit": "Gcell-steps/s", "cores": 1, "kind": "port",
            "sample": f"oracle (scipy CSR, 1 thread) on the {args.workload} geometry at "
                      f"96x96x192, {n} steps with beam"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200,
                    help="timed steps (200 FP64 steps at 256x256x512 take about 0.12 s, long enough for\n                    several clock samples inside the timed region)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="lossy_256")
    ap.add_argument("--dtype", default="float64", choices=["float64", "float32", "fp32c"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision-leg", action="store_true",
                    help="skip the FP32-compensated leg of the default FP64 run")
    ap.add_argument("--kernel", default="auto", choices=["auto", "tma", "twopass", "cell", "split"])
    ap.add_argument("--tile", default="0x0", help="rows x planes per block (0 = auto)")
    ap.add_argument("--steps-per-launch", type=int, default=0, choices=[0, 1, 2],
                    help="2: two steps per launch (temporal blocking) where it applies; "
                         "1: one step per launch; 0: the library's default (one)")
    ap.add_argument("--shape", default=None,
                    help="override the grid, e.g. 128x128x256 (profiling runs)")
    ap.add_argument("--accuracy", action="store_true",
                    help="FP32c vs FP64 wakesolve on the same grid (default workload "
                         "precision_448): relative WP / Z errors and both rates")
    ap.add_argument("--wakelength", type=float, default=None)
    ap.add_argument("--batch", type=int, default=0,
                    help="batched form: this many random pillbox cavities (seed 0) in "
                         "one captured CUDA graph, FP32c, --batch-steps steps each")
    ap.add_argument("--batch-steps", type=int, default=4000)
    ap.add_argument("--batch-launch", default="auto", choices=["auto", "batched", "graph"],
                    help="batched form: the device work list over all instances "
                         "(wk_batch_run), or a graph of per-instance launches")
    ap.add_argument("--batch-form", default="auto", choices=["auto", "persistent", "phases"],
                    help="batched launch form (auto: chosen by the autotuner)")
    ap.add_argument("--batch-tiles", default="auto", choices=["auto", "64x8", "fill", "32x16"],
                    help="tile shapes of the batched launch (auto: chosen by the autotuner; "
                         "fill: per instance, the shape with fewer idle lanes)")
    ap.add_argument("--batch-multiple", type=int, default=8,
                    help="batched form: transverse cell counts rounded up to this multiple")
    ap.add_argument("--adjoint", action="store_true",
                    help="differentiation form: 128x128x256 cavity with a 64^3 design region, "
                         "FP64 / FP32 / FP32-compensated forward + adjoint (4000 steps), "
                         "gradient checked on 16 random "
                         "directions against central differences of FP64 forward runs")
    ap.add_argument("--adjoint-steps", type=int, default=0,
                    help="steps of the differentiation form (0: 4000, or enough for the wake "
                         "when the relaxation clamp shortens dt)")
    ap.add_argument("--adjoint-forms", default="",
                    help="comma-separated subset of the adjoint forms (f64, f32, fp32c, "
                         "fp32c_adj32, fp32c_cs, fp32c_cs_adj32; default all)")
    ap.add_argument("--adjoint-directions", type=int, default=16,
                    help="random directions checked against central differences")
    ap.add_argument("--adjoint-sigma-max", type=float, default=1e3,
                    help="design-cell sigma ~ U[0, this] S/m (1e3: the configuration)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="z-slab decomposition on one GPU: the workload split into this many "
                         "z-slabs in one process (ghost planes copied every step)")
    ap.add_argument("--decomp", default="slab", choices=["replicas", "slab"],
                    help="with torchrun (N > 1): one block of a chain of N workload blocks per "
                         "rank with the z-slab ghost exchange over NCCL (default), or "
                         "independent replicas")
    ap.add_argument("--slab-depth", type=int, default=4,
                    help="z-slab ghost planes per side = steps between exchanges (fewer, "
                         "larger messages as it grows)")
    ap.add_argument("--batch-compare", action="store_true",
                    help="also run the batch in FP64 and report per-instance WP/|Z| errors")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        run_reference(args)
        return
    if args.accuracy:
        run_accuracy(args)
        return
    if args.batch:
        run_batch(args)
        return
    if args.adjoint:
        run_adjoint(args)
        return
    if args.slabs > 1 or (args.decomp == "slab" and int(os.environ.get("WORLD_SIZE", "1")) > 1):
        run_slab(args)
        return

    import torch
    import torch.distributed as dist

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    from wakis_b200 import workloads
    from wakis_b200.sources import Beam
    sp = workloads.spec(args.workload)
    dtype = np.float64 if args.dtype == "fp32c" else np.dtype(args.dtype).type
    shape = tuple(int(v) for v in args.shape.split("x")) if args.shape else None
    g, w, s = workloads.build_b200(args.workload, dtype=dtype, shape=shape,
                                   precision="fp32c" if args.dtype == "fp32c" else None)
    N = s.N
    split = args.kernel == "split"
    s.kernel = "auto" if split else args.kernel
    s.tile = tuple(int(v) for v in args.tile.split("x"))
    s.steps_per_launch = args.steps_per_launch
    bp = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")}
              ).params(s)
    ixt = int(np.abs(s.x - w.xtest).argmin())
    iyt = int(np.abs(s.y - w.ytest).argmin())
    total = args.warmup + args.steps
    hist = torch.zeros((9, s.Nz, total + args.steps), dtype=s._cap_dtype, device=dev)
    cap = (hist, ixt - 1, iyt - 1, 3, 3)

    def barrier():
        if ws > 1:
            dist.barrier()

    # warm-up (includes the first-step ghost zeroing)
    s._advance(args.warmup, 0, beam=bp, capture=cap, split=split)
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clk = Clocks(uuid)
    rclk = RegionClocks(uuid, local)
    time.sleep(0.3)
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    rclk.start()
    e0.record(st)
    s._advance(args.steps, args.warmup, beam=bp, capture=cap, split=split)
    e1.record(st)
    torch.cuda.synchronize()
    region_clocks = rclk.stop()
    # the status word of the step kernels: a timed-out tile load leaves the
    # steps incomplete, and then no rate is reported
    status_ok = _status_ok(s)
    barrier()
    ms = e0.elapsed_time(e1)
    # interior-kernel time of the same K steps, CUDA events around each
    # interior launch (wk_fit_step_timed), for the roofline of that kernel
    timing = []
    s._advance(args.steps, args.warmup + args.steps, beam=bp, capture=cap, timing=timing)
    ms_int = sum(t[0] for t in timing)
    n_int = sum(t[1] for t in timing)
    # kernels launched per step: TMA 1 (every face PEC-masked) or 1 interior
    # + 2 shell launches, two-pass 2 interior + 2 shell launches; the other
    # schedules launch a fixed set
    fixed = {"split": 4, "cell": 1}
    # the TMA schedule needs no shell launch when every face is PEC-masked;
    # with --steps-per-launch 2 it runs pairs of steps as one launch (k_tma2),
    # so fewer interior launches than steps
    pec_faces = all(b.lower() in ("pec", "electric", "pml") for b in s.bc_low + s.bc_high)
    two_step = pec_faces and 0 < n_int < args.steps
    n_per = 1 if two_step else n_int // max(args.steps, 1)
    tma_per_step = 1 if pec_faces else 3
    per_step = fixed.get(args.kernel, {1: tma_per_step, 2: 4}.get(n_per, 2 * n_per))
    # step kernels launched in the timed region
    launches = n_int if two_step else args.steps * per_step
    # cells the TMA / interior kernel updates: the whole grid when every face
    # is PEC-masked, all of x and y when the x/y faces are, else the interior
    # without the two-cell shell
    xy_pec = all(b.lower() in ("pec", "electric", "pml")
                 for b in s.bc_low[:2] + s.bc_high[:2])
    if n_per == 1 and per_step == 1:
        interior = N
    elif n_per == 1 and xy_pec:
        interior = s.Nx * s.Ny * (s.Nz - 4)
    else:
        interior = (s.Nx - 4) * (s.Ny - 4) * (s.Nz - 4)
    schedule = "tma2" if two_step else {1: "tma", 2: "twopass"}.get(n_per, args.kernel)

    # end to end through the public API: per-step H2D line current, D2H window
    prof = Beam(**{k: sp["wake"][k] for k in ("q", "sigmaz", "beta", "xsource", "ysource")})
    lines = np.stack([(prof.q * prof.v * prof.profile(s, n * s.dt) / s.dx[bp[0]] / s.dy[bp[1]])
                      for n in range(total + args.steps, total + 2 * args.steps)])
    lines = lines.astype(np.float64 if args.dtype == "fp32c" else dtype)
    jz = torch.from_numpy(lines).pin_memory()
    ez = torch.empty((args.steps, 9, s.Nz), dtype=s._cap_dtype).pin_memory()
    # warm-up of the I/O path (its device staging buffers are allocated on
    # the first call), on copies of the first chunk
    nw = min(4, args.steps)
    s.run_with_io(jz[:nw].clone().pin_memory(), torch.empty_like(ez[:nw]).pin_memory(),
                  step0=total + args.steps)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.run_with_io(jz, ez, step0=total + args.steps)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    clocks = region_clocks or clk.stop()
    if region_clocks is not None:
        clk.stop()
    # device times and the end-to-end wall time: max over ranks (and the
    # status flags: any rank that timed out voids the run)
    ms, ms_int, t_e2e, bad = max_over_ranks([ms, ms_int, t_e2e, 0.0 if status_ok else 1.0],
                                            ws, dev)
    if bad:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "error": "a step kernel timed out waiting for "
                              "a tile load in the timed region; no rate reported"}), flush=True)
        if ws > 1:
            dist.destroy_process_group()
        sys.exit(3)

    if rank == 0:
        value = N * args.steps * ws / (ms / 1e3) / 1e9
        bpc = BYTES_PER_CELL[args.dtype]
        peak, src = _peaks()
        step_gbs = bpc * N / (ms / 1e3 / args.steps) / 1e9
        if n_int > 0 and ms_int > 0:
            # algorithmic bytes of the interior cells of the timed steps over
            # the summed interior-kernel time
            achieved = bpc * interior * args.steps / (ms_int / 1e3) / 1e9
            kernel_note = (f"interior kernel(s) of the {schedule} schedule: {n_int} launches, "
                           f"{ms_int / args.steps:.4f} ms per step, {bpc} B x {interior} "
                           f"cells per step")
        else:
            achieved = step_gbs
            kernel_note = "whole step (no separate interior kernel)"
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"float64": "f64", "float32": "f32", "fp32c": "f32+bf16 comp (factors formed in f64)"}[
                args.dtype], "data": "synthetic",
            "config": {"workload": args.workload, "cells": N, "grid": [s.Nx, s.Ny, s.Nz],
                       "parallelism": f"replicas{ws}" if ws > 1 else "single",
                       "l2": "state %.0f MB > L2, no flush" % (
                           4 * 3 * N * s._E[0].element_size() / 1e6),
                       "step": "fused beam + Ez 3x3 capture + H and E half-steps",
                       "kernel": args.kernel, "schedule": schedule, "tile": args.tile,
                       "steps_per_launch": 2 if two_step else 1},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": src,
                         "bytes_per_cell_step": bpc, "kernel": kernel_note,
                         "traffic": _traffic(args.workload, args.dtype, schedule, interior),
                         "step_achieved": step_gbs, "step_frac": step_gbs / peak},
            "e2e": {"value": N * args.steps * ws / t_e2e / 1e9, "unit": "Gcell-steps/s",
                    "h2d_bytes_per_step": int(jz[0].numel() * jz.element_size()),
                    "d2h_bytes_per_step": int(ez[0].numel() * ez.element_size())},
            "gpu_launches": launches,
            "clocks": clocks,
            "status_word": 0,
        }
        if ws == 1 and args.dtype == "float64" and not args.no_precision_leg:
            del g, w, s, hist, cap
            torch.cuda.empty_cache()
            line["fp32c"] = precision_leg(args, dev, value)
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
