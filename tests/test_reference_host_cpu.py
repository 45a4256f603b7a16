"""The host build of the reference's own kernels, pinned to its CUDA build.

oracle/Makefile's `refhost` recipe compiles the reference sources (after a
mechanical rewrite of kernel launches and CUDA qualifiers, oracle/
host_rewrite.sed and host_shim.h) with g++ -fopenmp into
oracle/_ref/libsophia_ref_host.so: the reference's per-particle kernel
bodies looped over the CPU cores, which bench.py times as the CPU baseline.
Here it replays the golden fixtures that the reference's CUDA build wrote
(tests/golden/make_golden.py: the ISPH-DEM spouted beds and the 2-D WCSPH
dam breaks) and must agree with them: cell-sorted order exactly, every
real field to rel. L2 1e-9 at every checkpoint, contact partners exactly.  Both sides run the same FP64
expressions; only FMA contraction in the CUDA build differs.

Each fixture runs in a child process: the reference keeps its state in
globals and changes the working directory.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tests.helpers import golden_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libsophia_ref_host.so")
ISPH_GOLD = [p for p in golden_files() if json.loads(np.load(p)["meta"].tobytes()).get("solver", "isph") == "isph"]
WCSPH_GOLD = [p for p in golden_files() if json.loads(np.load(p)["meta"].tobytes()).get("solver") == "wcsph"]

CHILD = r'''
import ctypes as C, json, os, sys, tempfile
import numpy as np
sys.path.insert(0, sys.argv[1])
from tests.helpers import by_id, history_map, load_golden, rel_l2
from fluidized_bed_master_b200.beds import write_input_dir
g, p, sph, dem = load_golden(sys.argv[2])
L = C.CDLL(sys.argv[3])
L.ref_load.argtypes = [C.c_char_p]
L.ref_run.argtypes = [C.c_int]
L.ref_get.argtypes = [C.c_int, C.c_char_p, C.POINTER(C.c_double)]
L.ref_counts.argtypes = [C.POINTER(C.c_int)] * 3
work = tempfile.mkdtemp(prefix="refhost_")
write_input_dir(os.path.join(work, "input"), p, sph, dem)
os.makedirs(os.path.join(work, "plotdata"))
assert L.ref_load(work.encode()) == 0
ns, nd = C.c_int(), C.c_int()
nijk = (C.c_int * 3)()
L.ref_counts(C.byref(ns), C.byref(nd), nijk)
assert list(nijk) == list(g["nijk"])
def get(w, f, n):
    a = np.zeros(n)
    assert L.ref_get(w, f.encode(), a.ctypes.data_as(C.POINTER(C.c_double))) == 0, f
    return a
SPH = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s", "pgfx", "pgfy",
       "pgfz", "rho_ref", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz"]
DEM = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2", "Fdx_df",
       "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp"]
out = {"err": {}, "order": True, "partners": True}
done = 0
for cp in [int(c) for c in g["checkpoints"]]:
    assert L.ref_run(cp - done) == 0
    done = cp
    pre = f"s{cp}_"
    pid = get(0, "pid", ns.value)
    did = get(1, "dem_idx", nd.value)
    out["order"] &= bool(np.array_equal(pid, g[pre + "sph_pid"]) and np.array_equal(did, g[pre + "dem_dem_idx"]))
    for f in SPH + (["vis_t"] if pre + "sph_vis_t" in g.files else []):
        out["err"][f"{cp}.sph.{f}"] = rel_l2(get(0, f, ns.value), g[pre + "sph_" + f])
    for f in DEM:
        out["err"][f"{cp}.dem.{f}"] = rel_l2(get(1, f, nd.value), g[pre + "dem_" + f])
    ct_h = np.stack([get(1, f"ct_idx{s}", nd.value) for s in range(16)], 1)
    ct_g = np.stack([g[f"{pre}dem_ct_idx{s}"] for s in range(16)], 1)
    for a, b in zip(history_map(ct_h, np.zeros((nd.value, 16, 3))), history_map(ct_g, np.zeros((nd.value, 16, 3)))):
        out["partners"] &= set(a) == set(b)
print("RESULT " + json.dumps({k: (float(v) if not isinstance(v, (bool, dict)) else v) for k, v in out.items()}))
'''


CHILD_W = r'''
import ctypes as C, json, os, sys, tempfile
import numpy as np
sys.path.insert(0, sys.argv[1])
from tests.helpers import load_golden, rel_l2
from fluidized_bed_master_b200.beds import write_input_dir
g, p, sph, dem = load_golden(sys.argv[2])
L = C.CDLL(sys.argv[3])
L.ref_load_wcsph.argtypes = [C.c_char_p]
L.ref_run_wcsph.argtypes = [C.c_int]
L.ref_get.argtypes = [C.c_int, C.c_char_p, C.POINTER(C.c_double)]
L.ref_counts.argtypes = [C.POINTER(C.c_int)] * 3
work = tempfile.mkdtemp(prefix="refhost_")
write_input_dir(os.path.join(work, "input"), p, sph, dem)
os.makedirs(os.path.join(work, "plotdata"))
assert L.ref_load_wcsph(work.encode()) == 0
ns, nd = C.c_int(), C.c_int()
nijk = (C.c_int * 3)()
L.ref_counts(C.byref(ns), C.byref(nd), nijk)
def get(f):
    a = np.zeros(ns.value)
    assert L.ref_get(0, f.encode(), a.ctypes.data_as(C.POINTER(C.c_double))) == 0, f
    return a
F = ["x", "y", "ux", "uy", "m", "rho", "pres", "flt_s", "pgfx", "pgfy", "rho_ref", "ftotalx", "ftotaly", "ftotal",
     "drho", "grad_rhox", "grad_rhoy"]
out = {"err": {}, "order": True}
done = 0
for cp in [int(c) for c in g["checkpoints"]]:
    assert L.ref_run_wcsph(cp - done) == 0
    done = cp
    pre = f"s{cp}_sph_"
    out["order"] &= bool(np.array_equal(get("pid"), g[pre + "pid"]))
    for f in F:
        out["err"][f"{cp}.{f}"] = float(rel_l2(get(f), g[pre + f]))
print("RESULT " + json.dumps(out))
'''


def _run_child(child, path):
    r = subprocess.run([sys.executable, "-c", child, ROOT, os.path.abspath(path), LIB], capture_output=True,
                       text=True, timeout=900, env=dict(os.environ, OMP_NUM_THREADS="8"))
    assert r.returncode == 0, r.stderr[-3000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):])


@pytest.mark.skipif(not os.path.exists(LIB), reason="host build of the reference not built (needs its sources)")
@pytest.mark.parametrize("path", WCSPH_GOLD, ids=[p.split("/")[-1] for p in WCSPH_GOLD])
def test_host_reference_matches_cuda_reference_wcsph2d(path):
    """The reference's 2-D WCSPH kernels, host-compiled, against their CUDA
    run: cell-sorted order exact, every field to rel. L2 1e-9 at every
    checkpoint (up to 1,000 steps)."""
    res = _run_child(CHILD_W, path)
    assert res["order"], "cell-sorted order differs from the CUDA reference"
    bad = {k: v for k, v in res["err"].items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])[:10]


@pytest.mark.skipif(not os.path.exists(LIB), reason="host build of the reference not built (needs its sources)")
@pytest.mark.parametrize("path", ISPH_GOLD, ids=[p.split("/")[-1] for p in ISPH_GOLD])
def test_host_reference_matches_cuda_reference(path):
    res = _run_child(CHILD, path)
    assert res["order"], "cell-sorted order differs from the CUDA reference"
    assert res["partners"], "contact partners differ from the CUDA reference"
    bad = {k: v for k, v in res["err"].items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])[:10]
