"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs on a machine with a B200 and the reference harness built
(``make -C oracle ref`` -> oracle/_ref/libsophia_ref.so, compiled from
the unmodified reference sources).  For every case it writes the
synthetic bed in the reference's input formats, lets the reference's own
SOPHIA_single_ISPH (or, for the 2-D dam breaks, its 2-D WCSPH kernels in
the Lagrangian order of ref_run_wcsph) advance it, and stores inputs plus
the read-back state after each checkpoint in tests/golden/<case>.npz.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py --case contact

Each case runs in its own process because the reference keeps its state
in globals and changes the working directory.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fluidized_bed_master_b200.beds import dam_break_2d, spouted_bed, write_input_dir  # noqa: E402

SPH_FIELDS = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s",
              "pgfx", "pgfy", "pgfz", "rho_ref", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz",
              "p_type", "i_type", "buffer_type", "pid", "vis_t"]
DEM_FIELDS = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2",
              "Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp",
              "dem_idx"]

W_FIELDS = ["x", "y", "ux", "uy", "m", "rho", "pres", "flt_s", "pgfx", "pgfy", "rho_ref", "ftotalx", "ftotaly",
            "ftotal", "drho", "grad_rhox", "grad_rhoy", "p_type", "i_type", "buffer_type", "pid"]

# 2-D WCSPH dam breaks (reference constants), driven by ref_run_wcsph:
# name -> (generator kwargs, param overrides, checkpoints)
W_CASES = {
    # plain: pressure, viscous and artificial-viscosity forces, gravity
    "dam2d": (dict(dx=1.0e-2, seed=31, reference_compat=True), dict(), [1, 10, 1000]),
    # kernel gradient correction, Antuono delta-SPH, XSPH
    "dam2d_kgc": (dict(dx=1.0e-2, seed=32, reference_compat=True),
                  dict(kgc_solve=1, delSPH_solve=2, xsph_solve=1, c_xsph=0.5), [1, 10, 100]),
    # Molteni delta-SPH with XSPH, no correction
    "dam2d_molteni": (dict(dx=1.0e-2, seed=33, reference_compat=True),
                      dict(delSPH_solve=1, xsph_solve=1, c_xsph=0.5), [1, 10, 100]),
}

# name -> (generator kwargs, param overrides, checkpoints)
CASES = {
    # reference-compat bed, spheres starting in contact (Hertz-Mindlin,
    # tangential history insert/lookup/release), drag from moving spheres
    "contact": (dict(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=11, spacing=1.9, u_dem=0.05),
                dict(), [1, 8, 100]),
    # same bed with heat transfer on (SPH conduction, DEM shells,
    # radiation, contact conduction, convective exchange)
    "heat": (dict(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=12, spacing=1.9, u_dem=0.05),
             dict(con_solve=1), [1, 8, 100]),
    # the interface-sharpness and repulsive boundary forces of the advection
    # pass switched on (functions_PPE2.cuh:1450-1472)
    "forces": (dict(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=13, spacing=1.9, u_dem=0.05),
               dict(interface_solve=1, fb_solve=1), [1, 8, 100]),
    # the SPS eddy viscosity (functions_PREP2.cuh:2113-2171) and the
    # inter-particle surface tension (functions_PPE2.cuh:1490-1542), with the
    # concentration and particle-shifting switches on as well (no effect in
    # this step)
    "sps_ipf": (dict(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=14, spacing=1.9, u_dem=0.05),
                dict(fv_solve=1, turbulence_model=3, fs_solve=1, surf_model=1, concn_solve=1, pst_solve=1),
                [1, 8, 100]),
    # the curvature surface tension and the k-lm model: no force, no eddy
    # viscosity in this step
    "curvature": (dict(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=15, spacing=1.9, u_dem=0.05),
                  dict(fv_solve=1, turbulence_model=1, fs_solve=1, surf_model=2), [1, 8, 100]),
}


def case_inputs(name):
    gen, over, cps = CASES[name]
    p, sph, dem = spouted_bed(**gen)
    for k, v in over.items():
        setattr(p, k, v)
    p.freq_output = 1000000   # VTK only at step 0
    return p, sph, dem, cps


def w_worker(name, out):
    """A 2-D WCSPH case: SPH only, the state read back through the SPH slots."""
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libsophia_ref.so")
    L = C.CDLL(lib_path)
    L.ref_load_wcsph.argtypes = [C.c_char_p]
    L.ref_run_wcsph.argtypes = [C.c_int]
    L.ref_get.argtypes = [C.c_int, C.c_char_p, C.POINTER(C.c_double)]
    L.ref_counts.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    gen, over, cps = W_CASES[name]
    p, sph, dem = dam_break_2d(**gen)
    for k, v in over.items():
        setattr(p, k, v)
    p.freq_output = 1000000
    work = tempfile.mkdtemp(prefix="golden_")
    write_input_dir(os.path.join(work, "input"), p, sph, dem)
    os.makedirs(os.path.join(work, "plotdata"), exist_ok=True)
    rc = L.ref_load_wcsph(work.encode())
    if rc != 0:
        raise SystemExit(f"ref_load_wcsph failed: {rc}")
    ns, nd = C.c_int(), C.c_int()
    nijk = (C.c_int * 3)()
    L.ref_counts(C.byref(ns), C.byref(nd), nijk)
    blob = {"params_json": np.frombuffer(json.dumps(p.as_dict()).encode(), dtype=np.uint8),
            "nijk": np.array(list(nijk))}
    for k, v in sph.items():
        blob["in_sph_" + k] = np.asarray(v)
    done = 0
    for cp in cps:
        rc = L.ref_run_wcsph(cp - done)
        if rc != 0:
            raise SystemExit(f"ref_run_wcsph failed: {rc}")
        done = cp
        for f in W_FIELDS:
            a = np.zeros(ns.value)
            if L.ref_get(0, f.encode(), a.ctypes.data_as(C.POINTER(C.c_double))) != 0:
                raise SystemExit(f"ref_get {f}")
            blob[f"s{cp}_sph_{f}"] = a
    blob["checkpoints"] = np.array(cps)
    blob["meta"] = np.frombuffer(json.dumps({"case": name, "ns": ns.value, "nd": 0, "solver": "wcsph"}).encode(),
                                 dtype=np.uint8)
    np.savez_compressed(out, **blob)
    print(f"{name}: ns={ns.value} grid={list(nijk)} -> {out}")


def worker(name, out):
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libsophia_ref.so")
    L = C.CDLL(lib_path)
    L.ref_load.argtypes = [C.c_char_p]
    L.ref_run.argtypes = [C.c_int]
    L.ref_get.argtypes = [C.c_int, C.c_char_p, C.POINTER(C.c_double)]
    L.ref_counts.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_last_ms.restype = C.c_double
    p, sph, dem, cps = case_inputs(name)
    work = tempfile.mkdtemp(prefix="golden_")
    write_input_dir(os.path.join(work, "input"), p, sph, dem)
    os.makedirs(os.path.join(work, "plotdata"), exist_ok=True)
    rc = L.ref_load(work.encode())
    if rc != 0:
        raise SystemExit(f"ref_load failed: {rc}")
    ns, nd = C.c_int(), C.c_int()
    nijk = (C.c_int * 3)()
    L.ref_counts(C.byref(ns), C.byref(nd), nijk)
    blob = {"params_json": np.frombuffer(json.dumps(p.as_dict()).encode(), dtype=np.uint8),
            "nijk": np.array(list(nijk))}
    for k, v in sph.items():
        blob["in_sph_" + k] = np.asarray(v)
    for k, v in dem.items():
        blob["in_dem_" + k] = np.asarray(v)
    done = 0
    for cp in cps:
        rc = L.ref_run(cp - done)
        if rc != 0:
            raise SystemExit(f"ref_run failed: {rc}")
        done = cp
        for which, fields, n in ((0, SPH_FIELDS, ns.value), (1, DEM_FIELDS, nd.value)):
            for f in fields:
                a = np.zeros(n)
                if L.ref_get(which, f.encode(), a.ctypes.data_as(C.POINTER(C.c_double))) != 0:
                    raise SystemExit(f"ref_get {f}")
                blob[f"s{cp}_{'sph' if which == 0 else 'dem'}_{f}"] = a
            if which == 1:
                for s in range(16):
                    a = np.zeros(n)
                    L.ref_get(1, f"ct_idx{s}".encode(), a.ctypes.data_as(C.POINTER(C.c_double)))
                    blob[f"s{cp}_dem_ct_idx{s}"] = a
                    for c in range(3):
                        b = np.zeros(n)
                        L.ref_get(1, f"del_s{s}_{c}".encode(), b.ctypes.data_as(C.POINTER(C.c_double)))
                        blob[f"s{cp}_dem_del_s{s}_{c}"] = b
    vtk = os.path.join(work, "plotdata")
    vtks = sorted(os.listdir(vtk))
    if vtks:
        with open(os.path.join(vtk, vtks[0]), "rb") as fh:
            blob["vtk_step0"] = np.frombuffer(fh.read(), dtype=np.uint8)
    blob["checkpoints"] = np.array(cps)
    blob["meta"] = np.frombuffer(json.dumps({"case": name, "ns": ns.value, "nd": nd.value}).encode(), dtype=np.uint8)
    np.savez_compressed(out, **blob)
    print(f"{name}: ns={ns.value} nd={nd.value} grid={list(nijk)} -> {out}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default=None)
    ap.add_argument("--worker", nargs=2, metavar=("CASE", "OUT"))
    ap.add_argument("--outdir", default=HERE)
    a = ap.parse_args()
    if a.worker:
        (w_worker if a.worker[0] in W_CASES else worker)(*a.worker)
        return
    names = [a.case] if a.case else list(CASES) + list(W_CASES)
    for n in names:
        out = os.path.abspath(os.path.join(a.outdir, f"{n}.npz"))
        subprocess.run([sys.executable, os.path.abspath(__file__), "--worker", n, out], check=True)


if __name__ == "__main__":
    main()
