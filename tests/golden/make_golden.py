"""Generate the golden fixtures under tests/golden/ from the upstream Wakis
package (pure Python, loaded through ``refshim``).

Run on a machine that has the upstream source tree, naming its root in
``WAKIS_UPSTREAM``:

    WAKIS_UPSTREAM=<upstream tree> python tests/golden/make_golden.py [step|wake|source|test001|...]

Outputs (all small, committed):

* ``upstream_test001.npz``  regression vectors of upstream
  ``tests/test_001_pec_cubic_cavity.py`` (WP[::50], Z[::20], cumsum targets
  and tolerances), extracted from that file's source with ``ast``.
* ``step_cases.npz``  fields E, H, J after a few ``one_step`` calls of the
  upstream solver on tiny grids, for a matrix of boundary conditions,
  materials and dtypes, from seeded random initial fields, with a Gaussian
  beam driving Jz.
* ``wake_cases.npz``  WP, WP_3d, WPx, WPy, Z, Zx, Zy, f, s of upstream
  ``wakesolve`` + ``WakeSolver.solve`` on small cavities.
* ``source_cases.npz``  E, H, J after upstream ``emsolve`` driven by each
  hard source (PlaneWave, WavePacket, Dipole, Pulse) on a small vacuum box.
* ``lossy_cases.npz``  E, H, J after ``one_step`` calls with the beam on the
  lossy-wall workload geometry (sigma = 1e4 S/m background, z-PML) at small
  sizes.
* ``sibc_cases.npz``  a pillbox whose wall takes upstream's surface-impedance
  branch (the surface mask injected, see ``cases.SIBC_CASES``): fields after
  a few steps, and a full ``wakesolve`` + ``WakeSolver.solve``.
* ``abc_cases.npz``  E, H, J after ``emsolve`` with ABC faces, with upstream's
  CPU snapshot semantics and with copied snapshots (its GPU semantics).
* ``field_cases.npz``  upstream ``Field`` storage, indexing, assignment and
  arithmetic on a small random field (``cases.FIELD_*``).

The case definitions live in ``tests/cases.py`` so that the tests rebuild the
same inputs without the upstream package.
"""

import ast
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import refshim  # noqa: E402
import cases  # noqa: E402


def upstream_test001():
    path = os.path.join(refshim.UPSTREAM, "tests", "test_001_pec_cubic_cavity.py")
    tree = ast.parse(open(path).read())
    vals = {}
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            t = node.targets[0]
            if isinstance(t, ast.Name) and t.id in ("WP", "Z"):
                call = node.value
                arr = ast.literal_eval(call.args[0])
                vals[t.id] = np.array(arr[0] if isinstance(arr, tuple) else arr)
    # cumsum targets: pytest.approx(<value>, <rel>) calls
    approx = []
    for node in ast.walk(tree):
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute)
                and node.func.attr == "approx"):
            approx.append([ast.literal_eval(a) for a in node.args])
    assert len(approx) == 2 and "WP" in vals and "Z" in vals
    np.savez(os.path.join(HERE, "upstream_test001.npz"), WP=vals["WP"], Z=vals["Z"],
             WP_cumsum=approx[0][0], WP_cumsum_rel=approx[0][1],
             Z_cumsum=approx[1][0], Z_cumsum_rel=approx[1][1],
             WP_tol=50e-6, Z_tol=50e-5)
    print("upstream_test001.npz:", len(vals["WP"]), "WP samples,", len(vals["Z"]), "Z samples")


def step_cases(wakis):
    out = {}
    meta = []
    for idx, c in enumerate(cases.STEP_CASES):
        g = wakis.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
        masks = cases.step_masks(c)
        use_stl = bool(c["solids"])
        if use_stl:
            refshim.inject_solids(g, {k: masks[k] for k in c["solids"]}, c["solids"])
        try:
            s = wakis.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                                  dtype=np.dtype(c["dtype"]).type, bg=c["bg"],
                                  n_pml=c["n_pml"], use_stl=use_stl, use_sibc=False)
        except ValueError as e:
            meta.append({"index": idx, "error": "ValueError", "msg": str(e)})
            continue
        E0, H0 = cases.initial_fields(c, s.N)
        s.E.fromarray(E0.copy())
        s.H.fromarray(H0.copy())
        beam = wakis.sources.Beam(**c["beam"]) if c["beam"] else None
        for n in range(c["steps"]):
            if beam is not None:
                beam.update(s, n * s.dt)
            s.one_step()
        for f in "EHJ":
            out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
        for f in ("ieps", "imu", "sigma"):
            out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
        out[f"c{idx}_dt"] = np.array(s.dt)
        meta.append({"index": idx, "use_conductivity": bool(s.use_conductivity)})
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "step_cases.npz"), **out)
    print("step_cases.npz:", len(cases.STEP_CASES), "cases")


def wake_cases(wakis):
    out = {}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            for idx, c in enumerate(cases.WAKE_CASES):
                g = wakis.GridFIT3D(*c["bounds"], *c["shape"], verbose=0)
                m = cases.wake_mask(c, g.x, g.y, g.z)
                refshim.inject_solids(g, {"cav": m}, {"cav": c["material"]})
                w = wakis.WakeSolver(save=False, verbose=0, **c["wake"])
                s = wakis.SolverFIT3D(g, w, bc_low=c["bc_low"], bc_high=c["bc_high"],
                                      use_stl=True, bg=c["bg"], verbose=0,
                                      dtype=np.dtype(c["dtype"]).type)
                s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"])
                names = ["s", "WP", "Z", "f", "lambdas", "lambdaf"]
                if c["compute_plane"] == "both":
                    names += ["WP_3d", "WPx", "WPy", "Zx", "Zy"]
                for n in names:
                    out[f"c{idx}_{n}"] = np.asarray(getattr(w, n))
                out[f"c{idx}_Nt"] = np.array(s.Nt)
                out[f"c{idx}_dt"] = np.array(s.dt)
                out[f"c{idx}_Ez"] = s.E.toarray()[2 * s.N:].copy()
        finally:
            os.chdir(cwd)
    np.savez_compressed(os.path.join(HERE, "wake_cases.npz"), **out)
    print("wake_cases.npz:", len(cases.WAKE_CASES), "cases")


def source_cases(wakis):
    out = {}
    for idx, c in enumerate(cases.SOURCE_CASES):
        g = wakis.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
        s = wakis.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                              bg="vacuum", use_stl=False, use_sibc=False)
        src = getattr(wakis.sources, c["kind"])(**c["kw"])
        s.emsolve(c["Nt"], source=src)
        for f in "EHJ":
            out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
        out[f"c{idx}_dt"] = np.array(s.dt)
    np.savez_compressed(os.path.join(HERE, "source_cases.npz"), **out)
    print("source_cases.npz:", len(cases.SOURCE_CASES), "cases")


def lossy_cases(wakis):
    out = {}
    for idx, c in enumerate(cases.LOSSY_CASES):
        x, y, z = cases.lossy_edges(c)
        g = wakis.GridFIT3D(x=x, y=y, z=z, verbose=0)
        refshim.inject_solids(g, {"cavity": cases.lossy_mask(c)}, {"cavity": "vacuum"})
        s = wakis.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                              dtype=np.dtype(c["dtype"]).type, bg=c["bg"], n_pml=c["n_pml"],
                              use_stl=True, use_sibc=False)
        E0, H0 = cases.case_fields(c, s.N)
        s.E.fromarray(E0.copy())
        s.H.fromarray(H0.copy())
        beam = wakis.sources.Beam(**c["beam"])
        for n in range(c["steps"]):
            beam.update(s, n * s.dt)
            s.one_step()
        for f in "EHJ":
            out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
        out[f"c{idx}_dt"] = np.array(s.dt)
    np.savez_compressed(os.path.join(HERE, "lossy_cases.npz"), **out)
    print("lossy_cases.npz:", len(cases.LOSSY_CASES), "cases")


def _sibc_grid(wakis, c):
    """Upstream grid of a SIBC case with the wall solid and its surface mask
    injected in place of VTK's gradient (GridFIT3D._mark_cells_in_surface)."""
    b, shape, wall, surf = cases.sibc_geometry(c)
    g = wakis.GridFIT3D(*b, *shape, verbose=0)
    refshim.inject_solids(g, {"wall": wall}, {"wall": [1.0, 1.0, c["sigma"]]})
    g._mark_cells_in_surface = lambda key: g.grid.__setitem__(
        key, np.asarray(surf, bool).ravel(order="C"))
    return g


def sibc_cases(wakis):
    out = {}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            for idx, c in enumerate(cases.SIBC_CASES):
                g = _sibc_grid(wakis, c)
                if c["kind"] == "step":
                    s = wakis.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"],
                                          verbose=0, dtype=np.dtype(c["dtype"]).type,
                                          bg="vacuum", use_stl=True, use_sibc=True)
                    E0, H0 = cases.initial_fields(c, s.N)
                    s.E.fromarray(E0.copy())
                    s.H.fromarray(H0.copy())
                    beam = wakis.sources.Beam(**c["beam"])
                    for n in range(c["steps"]):
                        beam.update(s, n * s.dt)
                        s.one_step()
                    for f in "EHJ":
                        out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
                else:
                    w = wakis.WakeSolver(save=False, verbose=0, **c["wake"])
                    s = wakis.SolverFIT3D(g, w, bc_low=c["bc_low"], bc_high=c["bc_high"],
                                          verbose=0, dtype=np.dtype(c["dtype"]).type,
                                          bg="vacuum", use_stl=True, use_sibc=True)
                    s.wakesolve(wakelength=c["wakelength"], compute_plane=c["compute_plane"])
                    for n in ["s", "WP", "Z", "f", "lambdaf", "WP_3d", "WPx", "WPy", "Zx", "Zy"]:
                        out[f"c{idx}_{n}"] = np.asarray(getattr(w, n))
                    out[f"c{idx}_Nt"] = np.array(s.Nt)
                    out[f"c{idx}_Ez"] = s.E.toarray()[2 * s.N:].copy()
                for f in ("ieps", "sigma"):
                    out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
                out[f"c{idx}_dt"] = np.array(s.dt)
        finally:
            os.chdir(cwd)
    np.savez_compressed(os.path.join(HERE, "sibc_cases.npz"), **out)
    print("sibc_cases.npz:", len(cases.SIBC_CASES), "cases")


def abc_cases(wakis):
    out = {}
    for idx, c in enumerate(cases.ABC_SOURCE_CASES):
        g = wakis.GridFIT3D(*cases.SOURCE_BOUNDS, *c["shape"], verbose=0)
        s = wakis.SolverFIT3D(g, bc_low=c["bc_low"], bc_high=c["bc_high"], verbose=0,
                              bg="vacuum", use_stl=False, use_sibc=False)
        assert s.activate_abc
        if c["abc_copies"]:
            # upstream's GPU path: every snapshot is a copy (cupy .get())
            live = s.get_abc
            s.get_abc = lambda: tuple({a: {k: np.array(v, copy=True) for k, v in d.items()}
                                       for a, d in snap.items()} for snap in live())
        src = getattr(wakis.sources, c["kind"])(**c["kw"])
        s.emsolve(c["Nt"], source=src)
        for f in "EHJ":
            out[f"c{idx}_{f}"] = getattr(s, f).toarray().copy()
        out[f"c{idx}_dt"] = np.array(s.dt)
    np.savez_compressed(os.path.join(HERE, "abc_cases.npz"), **out)
    print("abc_cases.npz:", len(cases.ABC_SOURCE_CASES), "cases")


def field_cases(wakis):
    F = wakis.field.Field
    Nx, Ny, Nz = cases.FIELD_CASE["shape"]
    a, b, m, flat = cases.field_inputs()
    f = F(Nx, Ny, Nz)
    f.fromarray(a.copy())
    g = F(Nx, Ny, Nz)
    g.fromarray(b.copy())
    out = {}
    for d in "xyz":
        out[f"mat_{d}"] = np.array(f.to_matrix(d))
    out["abs"] = np.array(f.get_abs())
    out["abs_flat"] = np.array(f.get_abs(as_matrix=False))
    for name, key in cases.FIELD_READS:
        out[name] = np.array(f[key])
    h = f.copy()
    for key, val in cases.FIELD_WRITES:
        if val == "arange5":
            val = np.arange(5.0)
        elif val == "plane_y4":
            val = m[:, :, 4]
        h[key] = val
    out["after_writes"] = np.array(h.toarray())
    out["mul_scalar"] = (f * 2.5).toarray()
    out["mul_matrix"] = (f * m).toarray()
    out["mul_flat"] = (f * flat).toarray()
    out["add_field"] = (f + g).toarray()
    out["add_matrix"] = (f + m).toarray()
    out["add_flat"] = (f + flat).toarray()
    out["ijk"] = np.array([f.compute_ijk(n) for n in cases.FIELD_IJK])
    np.savez_compressed(os.path.join(HERE, "field_cases.npz"), **out)
    print("field_cases.npz:", len(out), "arrays")


if __name__ == "__main__":
    wakis = refshim.install()
    only = sys.argv[1:]
    if not only or "test001" in only:
        upstream_test001()
    if not only or "step" in only:
        step_cases(wakis)
    if not only or "wake" in only:
        wake_cases(wakis)
    if not only or "source" in only:
        source_cases(wakis)
    if not only or "lossy" in only:
        lossy_cases(wakis)
    if not only or "sibc" in only:
        sibc_cases(wakis)
    if not only or "abc" in only:
        abc_cases(wakis)
    if not only or "field" in only:
        field_cases(wakis)
