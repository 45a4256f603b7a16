#!/usr/bin/env python
"""SPH-DEM particle-updates/s of one ISPH-DEM step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Workload: the 3-D SPH-DEM fluidized bed (0.1 x 0.02 x 0.4 m box,
200,000 fluid SPH particles on a dx = 1.25 mm lattice plus inlet and wall
particles, 20,000 DEM spheres of 2 mm, Wendland C2, h = 1.3 dx, heat
transfer on), generated from a seed: synthetic data of the benchmark's
shape.  A step is one call of the engine's step (the reference's
SOPHIA_single_ISPH + time/count update).  value = (N_sph + N_dem) x K x
ranks / max-over-ranks device time of the K timed steps; L2 is flushed
(a 256 MB write) before every timed step and each step is timed with CUDA
events on the engine's stream.

--gpus N (torchrun, one process per GPU): every rank steps its own,
independently seeded bed -- the reference's ISPH-DEM path runs on one GPU
(ISPH_Calc_seperate.cuh:907), so ranks are replicas and scaling is weak.

--impl reference: the reference arm, timed on the host CPU: the oracle
port of the reference step (all host threads) on a bounded sample of the
same bed (a quarter-height slice with the same lattice and sphere density).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = dict(n_fluid=200_000, n_dem=20_000, dx=1.25e-3)
SAMPLE = dict(n_fluid=50_000, n_dem=5_000, dx=1.25e-3, dem_height=0.025)
SPH_STATE = ["ux", "uy", "uz", "m", "rho", "pres", "temp", "dDEMpor", "flt_s"]
DEM_STATE = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "Fdx_df", "Fdy_df", "Fdz_df", "Q_sd"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="bed",
                    choices=["bed", "dam2d", "dam2d-batch", "bed2d-batch", "batch", "ppe-profile", "column", "mlp", "slabs"],
                    help="bed: the 3-D SPH-DEM fluidized bed (default); dam2d: the 2-D WCSPH dam break "
                         "(its protocol is --steps 1000); dam2d-batch: 64 uneven dam breaks in one handle "
                         "against the same beds run one after another; bed2d-batch: 64 uneven 2-D ISPH-DEM beds "
                         "(per-bed inlet velocities) in one handle, against the same beds one after another (batch is "
                         "the same workload); "
                         "ppe-profile: --steps steps of the bed with the "
                         "projected-start PCG and step graphs off, so that a kernel profiler sees the PPE "
                         "kernels (no timing); slabs: the bench bed cut into z slabs, one per rank (on one "
                         "GPU: --slabs slabs in one process), exchanging ghost bands every step")
    ap.add_argument("--slabs", type=int, default=2, help="slabs on one GPU for --workload slabs")
    ap.add_argument("--slab-bed", default="bench", choices=["bench", "scaled"],
                    help="--workload slabs: the bench bed cut along z, or the 10x wider scaled bed cut along x")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true", help="reference arm: skip the reference CUDA build")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP64-build and FP32-vs-FP64 keys")
    ap.add_argument("--no-ppe", action="store_true", help="skip the PPE solver comparison")
    ap.add_argument("--ppe-train", type=int, default=80,
                    help="steps before the PPE measurement (the learned warm start trains there)")
    ap.add_argument("--ppe-precond", default="jacobi", choices=["jacobi", "two-level"],
                    help="--workload ppe-profile: the PCG preconditioner")
    ap.add_argument("--profile-bed", default="bench", choices=["bench", "scaled"],
                    help="--workload ppe-profile: the bench bed or the scaled bed")
    ap.add_argument("--ppe-bed", default="scaled", choices=["scaled", "bench"],
                    help="bed of the PPE comparison: the 2.2 M-particle scaled bed or the bench bed")
    args = ap.parse_args()
    if args.workload == "batch":
        args.workload = "bed2d-batch"
    return args


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl"
        import torch

        if not torch.cuda.is_available():
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_over_ranks(pg, value, op, device="cpu"):
    """value reduced over all ranks (op: "max" or "sum"); value itself when
    there is no process group.  Every rank must call it at the same point."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX if op == "max" else pg.ReduceOp.SUM)
    return float(t.item())


WORKLOAD_TEXT = ("3-D SPH-DEM fluidized bed 0.1x0.02x0.4 m: 200,000 fluid SPH on dx=1.25 mm (+inlet/wall "
                 "particles) and 20,000 DEM spheres d=2 mm, Wendland C2, h=1.3dx, heat transfer, ISPH-DEM step "
                 "(reference PPE sweep)")


def bench_config(n_sph, n_dem, world, fields):
    return {"workload": WORKLOAD_TEXT, "n_sph": n_sph, "n_dem": n_dem,
            "l2": "256 MB buffer written before every timed step",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "positions": "f64", "fields": fields}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch (field manifest of each kernel, SoA precision)
# ---------------------------------------------------------------------------
def manifest_bytes(kernel, ns, nd, nwall, nbuf, avg_nb, r):
    """Bytes each pass must move: every particle's own fields once (read +
    write), neighbour fields counted once per particle (perfect reuse), and
    the neighbour list it streams (4 B per entry)."""
    L = 4 * avg_nb + 4
    pos = 32  # x, y, z, h (double)
    per = {
        "build_list": ns * (pos + L),
        "passA": ns * (pos + 8 + L + 3 * r + 15 * r),
        "passB": ns * (pos + 12 + L + 17 * r + 8 * r),
        "ppe": ns * (pos + 12 + L + 18 * r + r),
        "passC": ns * (pos + 12 + L + 19 * r + 6 * r),
        "xsph": ns * (pos + 8 + L + 7 * r + 4 * r),
        "neumann": nwall * (pos + 4 * r),
        "open_bc": nbuf * (pos + 8 * r),
        "sph_coupling": ns * (pos + 12 * r),
        # the DEM set is FP64 in both builds
        "dem_contact": nd * (5 * 8 + 12 * 8 + 16 * 28),
        "dem_coupling": nd * (5 * 8 + 20 * 8),
        "dem_prep": nd * (5 * 8 + 6 * 8),
        "dem_update": nd * (3 * 8 + 20 * 8),
        "cells_gather_sph": ns * 2 * (pos + 9 * r + 16) + ns * 8,
        "cells_gather_dem": nd * 2 * (5 * 8 + 17 * 8 + 20 + 16 * 28) + nd * 8,
        "hash_sph": ns * (24 + 4 + 8),
        "hash_dem": nd * (24 + 4 + 8),
    }
    return per.get(kernel)


def profiled_traffic(kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of `kernel` on this workload, from the ncu summaries in profiles/
    (a line 'traffic_bytes_per_launch: <kernel> <bytes>'), or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith(".md"):
            continue
        with open(os.path.join(d, fn)) as fh:
            for ln in fh:
                parts = ln.split()
                if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch:" and parts[1] == kernel:
                    return float(parts[2])
    return None


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU reference (oracle port of the reference step)
# ---------------------------------------------------------------------------
class RefHarness:
    """A build of oracle/ref_harness.cu (the reference's own sources): the
    CUDA build (oracle/_ref/libsophia_ref.so) or the host build of the same
    kernels, looped with OpenMP over the CPU cores (libsophia_ref_host.so).
    It is loaded with one bed written in the reference's input formats and
    stepped with SOPHIA_single_ISPH's launch sequence without the three
    hard-wired DEM wall kernels (ref_run_without_dem_walls).  The bed runs
    with its open boundary off: the reference hard-wires its inlet/outlet
    slabs to its own spouted geometry.  The reference keeps its state in
    globals, so a process loads one bed per build."""

    def __init__(self, kind, p, sph, dem, solver="isph"):
        import ctypes as C
        import tempfile

        from fluidized_bed_master_b200.beds import write_input_dir

        name = "libsophia_ref.so" if kind == "cuda" else "libsophia_ref_host.so"
        path = os.path.join(ROOT, "oracle", "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle/_ref/{name} was not built (needs the reference sources)")
        q = p.copy()
        q.open_boundary = 0
        q.freq_output = 1 << 30
        work = tempfile.mkdtemp(prefix="ref_")
        write_input_dir(os.path.join(work, "input"), q, sph, dem)
        os.makedirs(os.path.join(work, "plotdata"), exist_ok=True)
        L = C.CDLL(path)
        L.ref_load.argtypes = [C.c_char_p]
        L.ref_load_wcsph.argtypes = [C.c_char_p]
        L.ref_run_without_dem_walls.argtypes = [C.c_int]
        L.ref_run_wcsph.argtypes = [C.c_int]
        L.ref_last_ms.restype = C.c_double
        L.ref_counts.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        cwd = os.getcwd()
        try:
            rc = (L.ref_load_wcsph if solver == "wcsph" else L.ref_load)(work.encode())
        finally:
            os.chdir(cwd)
        if rc != 0:
            raise RuntimeError(f"ref_load returned {rc}")
        self.run_fn = L.ref_run_wcsph if solver == "wcsph" else L.ref_run_without_dem_walls
        ns, nd = C.c_int(), C.c_int()
        nijk = (C.c_int * 3)()
        L.ref_counts(C.byref(ns), C.byref(nd), nijk)
        self.L, self.work, self.ns, self.nd = L, work, ns.value, nd.value

    def run(self, nsteps):
        """nsteps steps; returns their wall-clock ms (device sync at both ends)."""
        cwd = os.getcwd()
        try:
            os.chdir(self.work)
            rc = self.run_fn(nsteps)
        finally:
            os.chdir(cwd)
        if rc != 0:
            raise RuntimeError(f"reference step returned {rc}")
        return self.L.ref_last_ms()


def omp_threads():
    """Threads an OpenMP CPU leg uses: OMP_NUM_THREADS when set, else every core."""
    try:
        return int(os.environ["OMP_NUM_THREADS"])
    except (KeyError, ValueError):
        return os.cpu_count() or 1


HOST_REF_TEXT = ("the reference's own kernel bodies (its sources host-compiled with g++ -O2 -fopenmp, oracle/Makefile "
                 "refhost), FP64 AoS, blocks spread over the OpenMP threads, SOPHIA_single_ISPH's launch sequence "
                 "without the 3 hard-wired DEM wall kernels, open boundary off")


def cpu_reference(seconds=None, warmup=1, steps=None):
    """The CPU baseline on a bounded sample of the bench bed (a quarter-height
    slice with the same lattice and sphere density): the host build of the
    reference's kernels when it was built, else the oracle port."""
    from fluidized_bed_master_b200.beds import box_bed

    p, sph, dem = box_bed(**SAMPLE)
    threads = omp_threads()
    try:
        ref = RefHarness("host", p, sph, dem)
    except FileNotFoundError:
        return cpu_port(seconds, warmup, steps)
    n = ref.ns + ref.nd
    ref.run(warmup)
    ms, k = 0.0, 0
    while True:
        ms += ref.run(1)
        k += 1
        if steps is not None and k >= steps:
            break
        if steps is None and (ms / 1e3 >= seconds or k >= 200):
            break
    sample = (f"box bed slice: {ref.ns} SPH + {ref.nd} DEM (n_fluid=50000, n_dem=5000, same dx and sphere "
              f"density), {k} steps after {warmup} warm-up; {HOST_REF_TEXT}")
    return n * k / (ms / 1e3), threads, sample, ms / 1e3 / k, "reference"


def cpu_port(seconds=None, warmup=1, steps=None):
    """The oracle port of the reference step on the same slice (all host threads)."""
    from fluidized_bed_master_b200.beds import box_bed
    from oracle import Oracle

    p, sph, dem = box_bed(**SAMPLE)
    threads = os.cpu_count() or 1
    orc = Oracle(p, sph, dem, threads=threads)
    n = orc.ns + orc.nd
    orc.step(warmup)
    t0 = time.perf_counter()
    k = 0
    while True:
        orc.step(1)
        k += 1
        el = time.perf_counter() - t0
        if steps is not None and k >= steps:
            break
        if steps is None and (el >= seconds or k >= 200):
            break
    el = time.perf_counter() - t0
    sample = (f"box bed slice: {orc.ns} SPH + {orc.nd} DEM (n_fluid=50000, n_dem=5000, same dx and sphere "
              f"density), {k} steps after {warmup} warm-up; the oracle's FP64 port of the reference step")
    return n * k / el, threads, sample, el / k, "port"


def cpu_reference_full(warmup, steps):
    """The host build of the reference's kernels on the whole bench bed (all
    host threads): particle-updates/s, threads, sample text, s/step, kind."""
    from fluidized_bed_master_b200.beds import box_bed

    p, sph, dem = box_bed(seed=0, **WORKLOAD)
    threads = omp_threads()
    ref = RefHarness("host", p, sph, dem)
    n = ref.ns + ref.nd
    ref.run(warmup)
    ms = ref.run(steps)
    sample = (f"the whole bench bed ({ref.ns} SPH + {ref.nd} DEM), {steps} steps after {warmup} warm-up, "
              f"{threads} threads; {HOST_REF_TEXT}")
    return n * steps / (ms / 1e3), threads, sample, ms / 1e3 / steps, "reference"


def cpu_reference_full_port(warmup, steps):
    """The oracle port on the whole bench bed (when the reference was not built)."""
    from fluidized_bed_master_b200.beds import box_bed
    from oracle import Oracle

    p, sph, dem = box_bed(seed=0, **WORKLOAD)
    threads = os.cpu_count() or 1
    orc = Oracle(p, sph, dem, threads=threads)
    n = orc.ns + orc.nd
    orc.step(warmup)
    t0 = time.perf_counter()
    orc.step(steps)
    el = time.perf_counter() - t0
    sample = (f"the whole bench bed ({orc.ns} SPH + {orc.nd} DEM), {steps} steps after {warmup} warm-up, "
              f"{threads} threads; the oracle's FP64 port of the reference step")
    return n * steps / el, threads, sample, el / steps


def reference_cuda(warmup, steps):
    """The reference's own CUDA kernels (oracle/_ref/libsophia_ref.so, built
    from the unmodified reference sources with its nvcc flags for sm_100a) on
    this GPU, on the bench bed's particle set (RefHarness), with the
    reference's hard-wired material constants.  Wall clock around the step
    loop with a device sync at both ends, as the reference's time loop runs."""
    from fluidized_bed_master_b200.beds import box_bed

    p, sph, dem = box_bed(seed=0, **WORKLOAD)
    try:
        ref = RefHarness("cuda", p, sph, dem)
        ref.run(warmup)
        ms = ref.run(steps) / steps
    except (FileNotFoundError, RuntimeError) as e:
        return {"unavailable": str(e)}
    n = ref.ns + ref.nd
    return {"value": n / (ms / 1e3), "unit": "particle-updates/s", "ms_per_step": ms, "n_sph": ref.ns,
            "n_dem": ref.nd, "steps": steps, "warmup": warmup, "dtype": "f64",
            "how": "reference CUDA build (sm_100a, the reference's nvcc flags), SOPHIA_single_ISPH launch "
                   "sequence without the 3 hard-wired DEM wall kernels, open boundary off, the reference's "
                   "hard-wired materials; wall clock around the step loop, device sync at both ends"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from fluidized_bed_master_b200.beds import box_bed

    _, sph_full, dem_full = box_bed(seed=0, **WORKLOAD)
    config = bench_config(len(sph_full["x"]), len(dem_full["x"]), world, "f64")
    try:
        val, cores, sample, s_per_step, kind = cpu_reference_full(args.warmup, args.steps)
    except FileNotFoundError:
        val, cores, sample, s_per_step = cpu_reference_full_port(args.warmup, args.steps)
        kind = "port"
    unit = "particle-updates/s"
    line = {
        "metric": "SPH-DEM particle-updates/s on 1 B200 (3-D fluidized bed, ISPH-DEM step)",
        "impl": "reference", "value": val, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": s_per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded box bed, the whole bed every step)",
        "config": config,
        "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_cuda:
        line["reference_cuda"] = reference_cuda(args.warmup, args.steps)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# 2-D WCSPH dam break (--workload dam2d)
# ---------------------------------------------------------------------------
DAM_TEXT = ("2-D WCSPH dam break: 1.6x1.0 m tank, 0.4x0.8 m water column at dx=5 mm (12,800 fluid + 2,178 wall "
            "particles, seeded jitter 0.01 dx), Wendland C2, h=1.3dx, Tait EOS gamma=7, c0=10 sqrt(2 g 0.8), "
            "artificial viscosity alpha=0.02, gravity 9.81, dt=0.2 h/c0, predictor-corrector, continuity")
W_STATE = ["x", "y", "ux", "uy", "rho", "pres", "flt_s", "ftotalx", "ftotaly", "drho"]


def w_manifest_bytes(kernel, n, avg_nb, r):
    """Bytes each 2-D WCSPH pass must move (own fields once, neighbour
    fields once per particle, 4 B per list entry): positions x, y, h and
    mass, density are FP64 (8 B), the other fields r bytes."""
    L = 4 * avg_nb + 4
    pos = 24
    per = {
        "w.list": n * (pos + 4 + L),
        "w.prep": n * (pos + 16 + L + 8 + 3 * r),
        "w.continuity": n * (pos + 4 + 16 + L + 8 + 6 * r),   # with the EOS (pressure write)
        "w.interaction": n * (pos + 16 + L + 3 * r + 5 * r),
        "w.kgc": n * (pos + 16 + L + 4 * r),
        "w.xsph": n * (pos + 16 + L + 3 * r + 16),
        "w.predictor": n * (16 + 16 + 4 * r + 8 + 16 + 2 * r + 8),
        "w.corrector": n * (16 + 16 + 4 * r + 24 + 2 * r),
        "w.finish": n * 48,
    }
    return per.get(kernel)


def dam2d_cpu(seconds):
    from fluidized_bed_master_b200.beds import dam_break_2d
    from oracle import Oracle

    p, sph, _ = dam_break_2d(seed=0)
    threads = os.cpu_count() or 1
    orc = Oracle(p, sph, {}, threads=threads)
    orc.step(1)
    t0 = time.perf_counter()
    k = 0
    while True:
        orc.step(10)
        k += 10
        if time.perf_counter() - t0 >= seconds or k >= 5000:
            break
    el = time.perf_counter() - t0
    return orc.ns * k / el, threads, f"the whole dam break ({orc.ns} particles), {k} steps after 1 warm-up", el / k


def run_ppe_profile(args):
    """A few steps of the bench bed (or, with --profile-bed scaled, the
    scaled bed) with the PCG PPE (projected start over 8 solution changes;
    --ppe-precond two-level for the two-level preconditioner) and graphs
    off: the launch sequence a kernel profiler can see (kernels inside
    conditional graph nodes are hidden from it)."""
    from fluidized_bed_master_b200.beds import box_bed, scaled_box_bed
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import PPE_PCG, PRECOND_TWO_LEVEL, WARM_PROJECT

    if args.profile_bed == "scaled":
        p, sph, dem = scaled_box_bed(seed=0)
    else:
        p, sph, dem = box_bed(seed=0, **WORKLOAD)
    p.ppe_precond = PRECOND_TWO_LEVEL if args.ppe_precond == "two-level" else 0
    p.precision = 0
    p.ppe_mode = PPE_PCG
    p.kgc_solve = 0
    p.ppe_tol = 1e-6
    p.ppe_max_iter = 2000
    p.warm_start = WARM_PROJECT
    p.warm_hist = 8
    eng = Engine(p, sph, dem)
    eng.set_graphs(False)
    eng.step(args.steps)
    s = eng.stats()
    print(json.dumps({"workload": "ppe-profile", "steps": args.steps, "ppe_iters": s["ppe_iters"],
                      "ppe_status": s["ppe_status"], "n_sph": eng.ns, "n_dem": eng.nd}), flush=True)
    eng.close()


def _timed_steps(eng, stream, flush, k):
    """Device time (ms) of k steps, each timed with events on the engine's
    stream after a 256 MB L2 flush."""
    import torch

    tot = 0.0
    for _ in range(k):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        eng.step(1)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    return tot


COLUMN_TEXT = ("3-D ISPH column without DEM: 0.2x0.2x0.4 m water-like column at dx=4 mm (50x50x100 = 250,000 "
               "fluid, seeded jitter +/-0.01 dx) in a closed box of three wall layers, Wendland C2, h=1.3dx, "
               "hydrostatic pressure plus one sloshing roll (max 0.05 m/s), projection with the PPE solved by "
               "Jacobi-PCG to relative residual 1e-6, dt=1e-4 s")
COLUMN_CHECK_STEPS = 200


def run_column(args, world, rank, local, pg):
    """The 3-D ISPH column: particle-updates/s of the FP32 build, PCG
    iterations per step, and every field of the FP32 build against the FP64
    build of the same kernels after 200 steps."""
    import torch

    from fluidized_bed_master_b200.beds import isph_column
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import SPH

    metric = "ISPH particle-updates/s on 1 B200 (3-D column, PPE by PCG to 1e-6)"
    unit = "particle-updates/s"
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import Oracle
        threads = os.cpu_count() or 1
        p, sph, _ = isph_column(dx=1.0e-2, seed=0)
        o = Oracle(p, sph, {}, threads=threads)
        o.step(1)
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < max(5.0, args.cpu_seconds) and k < 2000:
            o.step(2)
            k += 2
        el = time.perf_counter() - t0
        val = o.ns * k / el
        line = {"metric": metric, "impl": "reference", "value": val, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded column)",
                "config": {"workload": COLUMN_TEXT},
                "cpu_baseline": {"value": val, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": f"the same column at dx=10 mm ({o.ns} particles), {k} steps"},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local)
    p, sph, _ = isph_column(seed=rank)
    q = p.copy()
    q.precision = 1 if args.precision == "fp64" else 0
    eng = Engine(q, sph, {})
    n = eng.ns
    stream = torch.cuda.ExternalStream(eng.stream_ptr())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng.step(args.warmup)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0]
    sampler = ClockSampler(int(vis) if vis.isdigit() else local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    t_tot, launches, iters = 0.0, 0, []
    for _ in range(args.steps):
        t_tot += _timed_steps(eng, stream, flush, 1)
        launches += eng.launches()
        st = eng.stats()
        iters.append(st["ppe_iters"])
        if st["ppe_status"] != 0 or not st["ppe_rel_residual"] <= p.ppe_tol:
            raise RuntimeError(f"PCG did not reach {p.ppe_tol}: {st}")
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    t_max = reduce_over_ranks(pg, t_tot, "max", "cuda")
    n_all = reduce_over_ranks(pg, n, "sum", "cuda")
    value = n_all * args.steps / (t_max / 1e3)
    e2e = None
    if not args.no_e2e:
        def pinned(k, dt):
            return torch.empty(k, dtype=dt, pin_memory=True).numpy()
        fields = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp"]
        hs = {f: pinned(n, torch.float64) for f in fields}
        for f in fields:
            hs[f][:] = eng.get(SPH, f)
        hb = sum(a.nbytes for a in hs.values())
        ke = max(3, min(args.steps, 20))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            eng.set_fields(SPH, hs)
            eng.step(1)
            eng.get_fields(SPH, hs)
        torch.cuda.synchronize()
        te = reduce_over_ranks(pg, time.perf_counter() - t0, "max", "cuda")
        e2e = {"value": n_all * ke / te, "unit": unit, "h2d_bytes_per_step": hb, "d2h_bytes_per_step": hb,
               "ms_per_step": te / ke * 1e3,
               "how": "per step: sphdem_set_fields of the particle state from pinned host arrays, sphdem_step, "
                      "sphdem_get_fields back"}
    eng.close()
    # the same steps with the two-level preconditioner (ppe_precond TWO_LEVEL)
    two = None
    if rank == 0:
        from fluidized_bed_master_b200.params import PRECOND_TWO_LEVEL

        q2 = q.copy()
        q2.ppe_precond = PRECOND_TWO_LEVEL
        e2 = Engine(q2, sph, {})
        s2 = torch.cuda.ExternalStream(e2.stream_ptr())
        e2.step(args.warmup)
        it2, t2 = [], 0.0
        for _ in range(args.steps):
            t2 += _timed_steps(e2, s2, flush, 1)
            it2.append(e2.stats()["ppe_iters"])
        e2.close()
        two = {"ms_per_step": t2 / args.steps, "value": n * args.steps / (t2 / 1e3), "unit": unit,
               "ppe_iters_per_step": float(np.mean(it2))}
    check = None
    if rank == 0 and not args.no_cpu:
        # every field of the FP32 build against the FP64 build after 200 steps
        runs = {}
        for prec in (0, 1):
            r = p.copy()
            r.precision = prec
            e = Engine(r, sph, {})
            e.step(COLUMN_CHECK_STEPS)
            ids = e.get(SPH, "pid")
            runs[prec] = {f: np.empty(n) for f in ("x", "y", "z", "ux", "uy", "uz", "rho", "pres")}
            for f in runs[prec]:
                runs[prec][f][ids] = e.get(SPH, f)
            e.close()
        rel = {f: float(np.linalg.norm(runs[0][f] - runs[1][f]) / max(np.linalg.norm(runs[1][f]), 1e-300))
               for f in runs[0]}
        check = {"steps": COLUMN_CHECK_STEPS, "rel_l2": rel, "max": max(rel.values())}
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if q.precision == 0 else "f64", "data": "synthetic (seeded column)",
        "config": {"workload": COLUMN_TEXT, "n": n, "n_fluid": int((sph["p_type"] == 1).sum()),
                   "l2": "256 MB buffer written before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "ppe_iters_per_step": float(np.mean(iters)) if iters else None,
        "two_level": two,
        "fp32_vs_fp64": check, "roofline": None, "cpu_baseline": None, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_dam2d_batch(args, world, rank, local, pg):
    """64 dam breaks of uneven size (fluid counts log-uniform in [2k, 50k],
    seeded) in one handle, one step graph for all; against the same beds
    stepped one after another, each in its own handle."""
    import torch

    from fluidized_bed_master_b200.beds import dam_break_batch
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import SPH

    metric = "2-D WCSPH particle-updates/s on 1 B200 (64 uneven dam breaks in one handle)"
    unit = "particle-updates/s"
    text = ("64 independent 2-D WCSPH dam breaks in one handle (sphdem_create_batch), fluid counts log-uniform in "
            "[2,000, 50,000] (seeded), columns twice as high as wide in tanks 4 columns wide, three wall layers, "
            "dx=5 mm, shared parameters (sound speed and CFL dt of the tallest column)")
    p, beds = dam_break_batch(seed=rank)
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import Oracle
        threads = os.cpu_count() or 1
        sel = [b for b in beds if len(b["x"]) < 8000][:2]
        t0, k, npart = time.perf_counter(), 0, sum(len(b["x"]) for b in sel)
        orcs = [Oracle(p, b, {}, threads=threads) for b in sel]
        while time.perf_counter() - t0 < max(5.0, args.cpu_seconds) and k < 2000:
            for o in orcs:
                o.step(5)
            k += 5
        el = time.perf_counter() - t0
        val = npart * k / el
        line = {"metric": metric, "impl": "reference", "value": val, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded dam breaks)",
                "config": {"workload": text},
                "cpu_baseline": {"value": val, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": f"2 of the beds ({npart} particles), {k} steps each"},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local)
    q = p.copy()
    q.precision = 1 if args.precision == "fp64" else 0
    eng = Engine.batch(q, beds)
    n = eng.ns
    stream = torch.cuda.ExternalStream(eng.stream_ptr())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng.step(args.warmup)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0]
    sampler = ClockSampler(int(vis) if vis.isdigit() else local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches = 0
    t_batch = 0.0
    for _ in range(args.steps):
        t_batch += _timed_steps(eng, stream, flush, 1)
        launches += eng.launches()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    t_max = reduce_over_ranks(pg, t_batch, "max", "cuda")
    n_all = reduce_over_ranks(pg, n, "sum", "cuda")
    value = n_all * args.steps / (t_max / 1e3)
    lanes = eng.stats()["w_lanes"]
    e2e = None
    if not args.no_e2e:
        def pinned(k, dt):
            return torch.empty(k, dtype=dt, pin_memory=True).numpy()
        hs = {f: pinned(n, torch.float64) for f in W_STATE}
        for f in W_STATE:
            hs[f][:] = eng.get(SPH, f)
        hb = sum(a.nbytes for a in hs.values())
        ke = max(3, min(args.steps, 50))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            eng.set_fields(SPH, hs)
            eng.step(1)
            eng.get_fields(SPH, hs)
        torch.cuda.synchronize()
        te = reduce_over_ranks(pg, time.perf_counter() - t0, "max", "cuda")
        e2e = {"value": n_all * ke / te, "unit": unit, "h2d_bytes_per_step": hb, "d2h_bytes_per_step": hb,
               "ms_per_step": te / ke * 1e3,
               "how": "per step: sphdem_set_fields of all beds' state (x, y in each bed's own coordinates) from "
                      "pinned host arrays, sphdem_step, sphdem_get_fields back"}
    eng.close()
    # the same beds one after another, each in its own handle (same lanes)
    seq_ms, ks = 0.0, 10
    if rank == 0:
        q1 = q.copy()
        q1.w_lanes = lanes
        for bd in beds:
            e = Engine(q1, bd, {})
            st = torch.cuda.ExternalStream(e.stream_ptr())
            e.step(3)
            seq_ms += _timed_steps(e, st, flush, ks) / ks
            e.close()
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if q.precision == 0 else "f64", "data": "synthetic (seeded dam breaks)",
        "config": {"workload": text, "n": n, "beds": len(beds), "bed_sizes": [len(b["x"]) for b in beds],
                   "l2": "256 MB buffer written before every timed step", "w_lanes": lanes,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "sequential": {"ms_per_step": seq_ms, "how": f"each bed alone in its own handle, {ks} timed steps each "
                       "after 3 warm-up steps, per-step device times summed over the beds",
                       "value": n * 1e3 / seq_ms if seq_ms else None, "unit": unit},
        "batch_speedup_vs_sequential": (seq_ms / (t_max / args.steps)) if seq_ms else None,
        "roofline": None, "cpu_baseline": None, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_bed2d_batch(args, world, rank, local, pg):
    """64 two-dimensional ISPH-DEM beds of uneven size (fluid counts
    log-uniform in [2k, 50k], seeded; spheres 10 %; inlet velocities
    U(0.1, 0.3)) in one handle, each in its own plane with its own
    open-boundary row, one step graph for all; against the same beds
    stepped one after another, each in its own handle."""
    import torch

    from fluidized_bed_master_b200.beds import bed2d_batch
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import DEM, SPH

    metric = "2-D ISPH-DEM particle-updates/s on 1 B200 (64 uneven beds in one handle)"
    unit = "particle-updates/s"
    text = ("64 independent 2-D ISPH-DEM beds (box_bed_2d: 0.1 m wide, dx=1.25 mm, Wendland C2, h=1.3 dx, "
            "water-like fluid, spheres d=2 mm +-5 % at 2500 kg/m3, Hertz-Mindlin E=1e7, heat transfer, XSPH, "
            "inlet/outlet slabs) in one handle, fluid counts log-uniform in [2,000, 50,000] (seeded), spheres "
            "10 % of the fluid count, inlet velocity U(0.1, 0.3) m/s per bed (sphdem_set_beds)")
    p, sph, dem, rows, parts = bed2d_batch(seed=rank)
    n_sph, n_dem = len(sph["x"]), len(dem["x"])
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import Oracle
        threads = os.cpu_count() or 1
        sel = sorted(parts, key=lambda pt: len(pt[0]["x"]))[:2]
        npart = sum(len(s["x"]) + len(d["x"]) for s, d, _ in sel)
        orcs = [Oracle(p, s, d, threads=threads, beds=r) for s, d, r in sel]
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < max(5.0, args.cpu_seconds) and k < 2000:
            for o in orcs:
                o.step(2)
            k += 2
        el = time.perf_counter() - t0
        val = npart * k / el
        line = {"metric": metric, "impl": "reference", "value": val, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 2-D beds)",
                "config": {"workload": text},
                "cpu_baseline": {"value": val, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": f"the 2 smallest beds ({npart} particles), {k} steps each"},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local)
    q = p.copy()
    q.precision = 1 if args.precision == "fp64" else 0
    eng = Engine(q, sph, dem, beds=rows)
    list_mode = eng.list_build()
    n = eng.ns + eng.nd
    stream = torch.cuda.ExternalStream(eng.stream_ptr())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng.step(args.warmup)
    torch.cuda.synchronize()
    # per-kernel breakdown (in-graph events, every kernel) before the timed
    # region, which runs without events
    eng.set_timing(True)
    eng.step(2)
    eng.collect_timing()
    b0 = eng.timing()
    for _ in range(PROFILE_STEPS // 2):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.step(1)
        eng.collect_timing()
    kms = {k: (v[0] - b0.get(k, (0, 0))[0]) / (PROFILE_STEPS // 2) for k, v in eng.timing().items()}
    kms = {k: round(v, 4) for k, v in sorted(kms.items(), key=lambda kv: -kv[1]) if v > 0}
    # the same with the DEM branch on the step stream: each kernel alone
    eng.set_concurrency(False)
    eng.step(2)
    eng.collect_timing()
    b1 = eng.timing()
    for _ in range(PROFILE_STEPS // 2):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.step(1)
        eng.collect_timing()
    kser = {k: (v[0] - b1.get(k, (0, 0))[0]) / (PROFILE_STEPS // 2) for k, v in eng.timing().items()}
    kser = {k: round(v, 4) for k, v in sorted(kser.items(), key=lambda kv: -kv[1]) if v > 0}
    eng.set_concurrency(True)
    eng.set_timing(False)
    eng.step(2)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0]
    sampler = ClockSampler(int(vis) if vis.isdigit() else local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches = 0
    t_batch = 0.0
    for _ in range(args.steps):
        t_batch += _timed_steps(eng, stream, flush, 1)
        launches += eng.launches()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    t_max = reduce_over_ranks(pg, t_batch, "max", "cuda")
    n_all = reduce_over_ranks(pg, n, "sum", "cuda")
    value = n_all * args.steps / (t_max / 1e3)
    finite = bool(np.all(np.isfinite(eng.get(SPH, "pres"))) and np.all(np.isfinite(eng.get(DEM, "uz"))))
    e2e = None
    if not args.no_e2e:
        def pinned(k, dt):
            return torch.empty(k, dtype=dt, pin_memory=True).numpy()
        hs = {f: pinned(eng.ns, torch.float64) for f in ["x", "y", "z"] + SPH_STATE}
        hd = {f: pinned(eng.nd, torch.float64) for f in DEM_STATE}
        for f in hs:
            hs[f][:] = eng.get(SPH, f)
        for f in hd:
            hd[f][:] = eng.get(DEM, f)
        hb = sum(a.nbytes for a in hs.values()) + sum(a.nbytes for a in hd.values())
        ke = max(3, min(args.steps, 30))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            eng.set_fields(SPH, hs)
            eng.set_fields(DEM, hd)
            eng.step(1)
            eng.get_fields(SPH, hs)
            eng.get_fields(DEM, hd)
        torch.cuda.synchronize()
        te = reduce_over_ranks(pg, time.perf_counter() - t0, "max", "cuda")
        e2e = {"value": n_all * ke / te, "unit": unit, "h2d_bytes_per_step": hb, "d2h_bytes_per_step": hb,
               "ms_per_step": te / ke * 1e3,
               "how": "per step: sphdem_set_fields of every bed's SPH and DEM state from pinned host arrays, "
                      "sphdem_step, sphdem_get_fields back"}
    eng.close()
    # the same beds one after another, each in its own handle
    seq_ms, ks = 0.0, 5
    if rank == 0:
        for sb, db, rb in parts:
            e = Engine(q, sb, db, beds=rb)
            st = torch.cuda.ExternalStream(e.stream_ptr())
            e.step(3)
            seq_ms += _timed_steps(e, st, flush, ks) / ks
            e.close()
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if q.precision == 0 else "f64", "data": "synthetic (seeded 2-D beds)",
        "config": {"workload": text, "n_sph": n_sph, "n_dem": n_dem, "beds": len(parts),
                   "fluid_counts": [int(np.sum((s["p_type"] == 1) & (s["z"] >= 0))) for s, _, _ in parts],
                   "inlet_uz": [round(r["inlet_uz"], 4) for r in rows],
                   "list_build": list_mode, "list_build_how": LIST_BUILD_HOW,
                   "l2": "256 MB buffer written before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "state_finite": finite,
        "kernels_ms_per_step": kms,
        "kernels_ms_per_step_from": f"{PROFILE_STEPS // 2} steps with every kernel timed, before the timed region",
        "kernels_ms_per_step_serialised": kser,
        "sequential": {"ms_per_step": seq_ms, "how": f"each bed alone in its own handle, {ks} timed steps each "
                       "after 3 warm-up steps, per-step device times summed over the beds",
                       "value": n * 1e3 / seq_ms if seq_ms else None, "unit": unit},
        "batch_speedup_vs_sequential": (seq_ms / (t_max / args.steps)) if seq_ms else None,
        "roofline": None, "cpu_baseline": None, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_dam2d(args, world, rank, local, pg):
    import torch

    from fluidized_bed_master_b200.beds import dam_break_2d
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import SPH

    metric = "2-D WCSPH particle-updates/s on 1 B200 (dam break)"
    unit = "particle-updates/s"
    if args.impl == "reference":
        if rank != 0:
            return
        p0, sph0, _ = dam_break_2d(seed=0)
        kind = "reference"
        try:
            ref = RefHarness("host", p0, sph0, {}, solver="wcsph")
            ref.run(args.warmup)
            ms = ref.run(args.steps) / args.steps
            val, cores, s_per_step = ref.ns / (ms / 1e3), omp_threads(), ms / 1e3
            sample = (f"the whole dam break ({ref.ns} particles), {args.steps} steps after {args.warmup} warm-up; "
                      "the reference's own 2-D WCSPH kernel bodies host-compiled (oracle/Makefile refhost), FP64, "
                      "in the Lagrangian order of oracle/ref_harness.cu")
        except FileNotFoundError:
            val, cores, sample, s_per_step = dam2d_cpu(max(5.0, args.cpu_seconds))
            kind = "port"
        line = {"metric": metric, "impl": "reference", "value": val, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": s_per_step * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded dam break)", "config": {"workload": DAM_TEXT},
                "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if not args.no_ref_cuda:
            try:
                rc_ = RefHarness("cuda", p0, sph0, {}, solver="wcsph")
                rc_.run(args.warmup)
                ms = rc_.run(args.steps) / args.steps
                line["reference_cuda"] = {
                    "value": rc_.ns / (ms / 1e3), "unit": unit, "ms_per_step": ms, "n": rc_.ns, "steps": args.steps,
                    "warmup": args.warmup, "dtype": "f64",
                    "how": "reference CUDA build (sm_100a), its 2-D WCSPH kernels in the Lagrangian order of "
                           "oracle/ref_harness.cu (ref_run_wcsph); wall clock around the step loop"}
            except (FileNotFoundError, RuntimeError) as e:
                line["reference_cuda"] = {"unavailable": str(e)}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local)
    p, sph, _ = dam_break_2d(seed=rank)
    p.precision = 1 if args.precision == "fp64" else 0
    eng = Engine(p, sph, {})
    n = eng.ns
    stream = torch.cuda.ExternalStream(eng.stream_ptr())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng.step(args.warmup)
    torch.cuda.synchronize()
    eng.set_timing(True)
    eng.step(2)
    eng.collect_timing()
    counts, _ = eng.neighbors(cap=1)
    avg_nb = float(counts.mean())
    base = eng.timing()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0]
    sampler = ClockSampler(int(vis) if vis.isdigit() else local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms, launches = 0.0, 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        eng.step(1)
        launches += eng.launches()
        with torch.cuda.stream(stream):
            e1.record(stream)
        eng.collect_timing()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    t_max = reduce_over_ranks(pg, total_ms, "max", "cuda")
    n_all = reduce_over_ranks(pg, n, "sum", "cuda")
    value = n_all * args.steps / (t_max / 1e3)
    tim = eng.timing()
    per_kernel = {k: (v[0] - base.get(k, (0, 0))[0], v[1] - base.get(k, (0, 0))[1]) for k, v in tim.items()}
    # dominant single kernel (the NNPS timer spans hash, CUB's sort, gather and rows)
    single = {k: v for k, v in per_kernel.items() if k != "w.nnps"}
    dom_name, (dom_ms, dom_n) = max(single.items(), key=lambda kv: kv[1][0])
    r = 8 if args.precision == "fp64" else 4
    bytes_dom = w_manifest_bytes(dom_name, n, avg_nb, r)
    peak, peak_kind = load_peaks()
    achieved = bytes_dom / (dom_ms / max(dom_n, 1) / 1e3) / 1e9 if (bytes_dom and dom_n) else None
    traffic = profiled_traffic(dom_name) if args.precision == "fp32" else None
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "bytes_per_launch": bytes_dom, "launch_ms": dom_ms / max(dom_n, 1), "peak_source": peak_kind,
                "share_of_step": dom_ms / max(sum(v[0] for v in per_kernel.values()), 1e-12)}
    e2e = None
    if not args.no_e2e:
        def pinned(k, dt):
            return torch.empty(k, dtype=dt, pin_memory=True).numpy()
        hs = {f: pinned(n, torch.float64) for f in W_STATE}
        for f in W_STATE:
            hs[f][:] = eng.get(SPH, f)
        hb = sum(a.nbytes for a in hs.values())
        eng.set_timing(False)
        ke = max(3, min(args.steps, 200))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            eng.set_fields(SPH, hs)
            eng.step(1)
            eng.get_fields(SPH, hs)
        torch.cuda.synchronize()
        te = reduce_over_ranks(pg, time.perf_counter() - t0, "max", "cuda")
        e2e = {"value": n_all * ke / te, "unit": unit, "h2d_bytes_per_step": hb, "d2h_bytes_per_step": hb,
               "ms_per_step": te / ke * 1e3,
               "how": "per step: sphdem_set_fields of the WCSPH state (incl. the rates the predictor reads) from "
                      "pinned host arrays, sphdem_step, sphdem_get_fields back"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample, _ = dam2d_cpu(min(args.cpu_seconds, 10.0))
        cpu = {"value": v, "unit": unit, "cores": cores, "kind": "port", "sample": sample}
    stats = eng.stats()
    eng.close()
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if r == 4 else "f64", "data": "synthetic (seeded dam break)",
        "config": {"workload": DAM_TEXT, "n": n, "l2": "256 MB buffer written before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "positions": "f64",
                   "density_mass": "f64", "fields": "f32" if r == 4 else "f64"},
        "avg_neighbours": avg_nb, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clocks,
        "stats": {k: stats[k] for k in ("rho_max_sph", "u_max_sph", "overflow_flags", "nan_flag", "w_lanes")},
        "kernels_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in per_kernel.items() if v[1]},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------
def run_engine(args, world, rank, local, pg):
    import torch

    from fluidized_bed_master_b200.beds import box_bed
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import DEM, SPH

    torch.cuda.set_device(local)
    p, sph, dem = box_bed(seed=rank, **WORKLOAD)
    p.precision = 1 if args.precision == "fp64" else 0
    eng = Engine(p, sph, dem)
    list_mode = eng.list_build()
    n_part = eng.ns + eng.nd
    stream = torch.cuda.ExternalStream(eng.stream_ptr())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    eng.step(args.warmup)
    torch.cuda.synchronize()
    # Per-kernel breakdown: every kernel timed by in-graph events over
    # PROFILE_STEPS steps before the timed region (each timed kernel adds two
    # event records to the step graph, ~0.1 ms per step for all of them).
    # The timed region then times only the dominant kernel, live, for the
    # roofline.
    eng.set_timing(True)
    eng.step(2)          # capture both graph parities with timing events
    eng.collect_timing()
    b0 = eng.timing()
    for _ in range(PROFILE_STEPS):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.step(1)
        eng.collect_timing()
    t_prof = eng.timing()
    per_kernel = {k: (v[0] - b0.get(k, (0, 0))[0], v[1] - b0.get(k, (0, 0))[1]) for k, v in t_prof.items()}
    dom_name = max(per_kernel.items(), key=lambda kv: kv[1][0])[0]
    eng.set_timing_only(dom_name)
    eng.step(2)          # recapture with the dominant kernel's events only
    eng.collect_timing()
    counts, _ = eng.neighbors(cap=1)
    avg_nb = float(counts.mean()) if eng.ns else 0.0
    base = eng.timing()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0]
    sampler = ClockSampler(int(vis) if vis.isdigit() else local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms = 0.0
    launches0 = 0
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        eng.step(1)
        launches0 += eng.launches()
        with torch.cuda.stream(stream):
            e1.record(stream)
        eng.collect_timing()  # synchronises the engine stream
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    t_max = reduce_over_ranks(pg, total_ms, "max", "cuda")
    n_all = reduce_over_ranks(pg, n_part, "sum", "cuda")
    value = n_all * args.steps / (t_max / 1e3)
    ms_per_step = t_max / args.steps

    # dominant kernel and its roofline: its events in the timed steps
    tim = eng.timing()
    timed = {k: (v[0] - base.get(k, (0, 0))[0], v[1] - base.get(k, (0, 0))[1]) for k, v in tim.items()}
    r = 8 if args.precision == "fp64" else 4
    nwall = int((sph["p_type"] <= 0).sum())
    nbuf = int(((sph["p_type"] == 1) & ((sph["z"] < p.obc_L2 - 1e-6) | (sph["z"] >= p.obc_L3 - 1e-6))).sum())
    peak, peak_kind = load_peaks()

    def roofline_of(per, live=None):
        dom_name, (dom_ms, dom_n) = max(per.items(), key=lambda kv: kv[1][0])
        share = dom_ms / max(sum(v[0] for v in per.values()), 1e-12)
        if live is not None:
            dom_ms, dom_n = live[dom_name]
        bytes_dom = manifest_bytes(dom_name, eng.ns, eng.nd, nwall, nbuf, avg_nb, r)
        achieved = bytes_dom / (dom_ms / max(dom_n, 1) / 1e3) / 1e9 if (bytes_dom and dom_n) else None
        traffic = profiled_traffic(dom_name) if args.precision == "fp32" else None
        return {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "bytes_per_launch": bytes_dom, "launch_ms": dom_ms / max(dom_n, 1), "peak_source": peak_kind,
                "share_of_step": share}

    roofline = roofline_of(per_kernel, live=timed)
    roofline["timed_in"] = ("the timed steps (its own CUDA events on its stream; its share of the step from "
                            f"{PROFILE_STEPS} steps with every kernel timed before the timed region)")
    eng.set_timing_only(None)
    # The DEM branch runs concurrently with the SPH passes, so the event
    # times above include the SMs each kernel shares with the other branch.
    # The same steps with the branch serialised on the step stream give
    # each kernel's own duration (not timed as the headline).
    serial = None
    if eng.ns and eng.nd:
        eng.set_concurrency(False)
        eng.step(2)
        eng.collect_timing()
        b2 = eng.timing()
        ks = max(3, min(args.steps, 10))
        t_ser = 0.0
        for _ in range(ks):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            eng.step(1)
            with torch.cuda.stream(stream):
                e1.record(stream)
            eng.collect_timing()
            t_ser += e0.elapsed_time(e1)
        t2 = eng.timing()
        per_ser = {k: (v[0] - b2.get(k, (0, 0))[0], v[1] - b2.get(k, (0, 0))[1]) for k, v in t2.items()}
        serial = {"ms_per_step": t_ser / ks, "steps": ks, "roofline": roofline_of(per_ser),
                  "kernels_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in per_ser.items() if v[1]}}
        eng.set_concurrency(True)

    # end to end through the C ABI with host buffers: each step uploads the
    # mutable particle state from pinned host arrays, steps, reads it back
    e2e = None
    if not args.no_e2e:
        def pinned(n, dt):
            return torch.empty(n, dtype=dt, pin_memory=True).numpy()
        hs = {f: pinned(eng.ns, torch.float64) for f in SPH_STATE}
        hd = {f: pinned(eng.nd, torch.float64) for f in DEM_STATE}
        for f in SPH_STATE:
            hs[f][:] = eng.get(SPH, f)
        for f in DEM_STATE:
            hd[f][:] = eng.get(DEM, f)
        hid = pinned(eng.nd * 16, torch.int32).reshape(eng.nd, 16)
        hsp = pinned(eng.nd * 48, torch.float64).reshape(eng.nd, 16, 3)
        eng.history(out=(hid, hsp))
        hb = sum(a.nbytes for a in hs.values()) + sum(a.nbytes for a in hd.values()) + hid.nbytes + hsp.nbytes
        eng.set_timing(False)
        ke = max(3, min(args.steps, 10))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            eng.set_fields(SPH, hs)
            eng.set_fields(DEM, hd)
            eng.set_history(hid, hsp)
            eng.step(1)
            eng.get_fields(SPH, hs)
            eng.get_fields(DEM, hd)
            eng.history(out=(hid, hsp))
        torch.cuda.synchronize()
        te = reduce_over_ranks(pg, time.perf_counter() - t0, "max", "cuda")
        e2e = {"value": n_all * ke / te, "unit": "particle-updates/s", "h2d_bytes_per_step": hb,
               "d2h_bytes_per_step": hb, "ms_per_step": te / ke * 1e3,
               "how": "per step: sphdem_set_fields/set_history of the mutable state from pinned host arrays, "
                      "sphdem_step, sphdem_get_fields/get_history back into them"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample, _, kind = cpu_reference(seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": "particle-updates/s", "cores": cores, "kind": kind, "sample": sample}

    stats = eng.stats()
    eng.close()
    fp64, fp32_vs_fp64 = None, None
    if rank == 0 and world == 1 and not args.no_precision and r == 4:
        fp64, fp32_vs_fp64 = precision_keys(args, rank)
    ppe = None
    if rank == 0 and world == 1 and not args.no_ppe:
        ppe = ppe_comparison(args)
    line = {
        "metric": "SPH-DEM particle-updates/s on 1 B200 (3-D fluidized bed, ISPH-DEM step)",
        "value": value, "unit": "particle-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if r == 4 else "f64",
        "data": "synthetic (seeded box bed; reference input.txt not shipped)",
        "config": dict(bench_config(eng.ns, eng.nd, world, "f32" if r == 4 else "f64"),
                       list_build=list_mode, list_build_how=LIST_BUILD_HOW),
        "avg_neighbours": avg_nb,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(launches0),
        "clocks": clocks,
        "stats": {k: stats[k] for k in ("rho_max_sph", "u_max_sph", "u_max_dem", "overflow_flags", "nan_flag")},
        "kernels_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in per_kernel.items() if v[1]},
        "kernels_ms_per_step_from": f"{PROFILE_STEPS} steps with every kernel timed, before the timed region",
        "dem_branch_serialised": serial,
        "fp64_build": fp64,
        "fp32_vs_fp64": fp32_vs_fp64,
        "ppe": ppe,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


PREC_SPH = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s", "ftotalx",
            "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "pgfx", "pgfy", "pgfz", "rho_ref", "dtemp"]
PREC_DEM = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_sd", "flt_sd2", "Fdx_df",
            "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp", "Q_sd"]
PREC_STEPS = 100
PROFILE_STEPS = 10
LIST_BUILD_HOW = ("SPH list build picked at commit by timing (sphdem_get_list_build): 1 = a thread per particle, "
                  "2/4/8 = a warp per cell with that many cells per block")


def precision_keys(args, seed):
    """The FP64 build of the same kernels on the bench bed: its throughput
    (same protocol as the headline: warm-up, L2 flush and CUDA events per
    step) and, after PREC_STEPS steps from the same input, every field of
    the FP32 build against it (rel. L2 per field, matched by particle id)."""
    import torch

    from fluidized_bed_master_b200.beds import box_bed
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import DEM, SPH

    p, sph, dem = box_bed(seed=seed, **WORKLOAD)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    q = p.copy()
    q.precision = 1
    e64 = Engine(q, sph, dem)
    stream = torch.cuda.ExternalStream(e64.stream_ptr())
    e64.step(args.warmup)
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        e64.step(1)
        with torch.cuda.stream(stream):
            b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    n = e64.ns + e64.nd
    fp64 = {"value": n * args.steps / (total / 1e3), "unit": "particle-updates/s", "ms_per_step": total / args.steps,
            "dtype": "f64", "how": "FP64 build of the same kernels (positions and every field FP64), same bed, "
                                   "warm-up, L2 flush and CUDA events as the headline"}
    e64.close()
    q32 = p.copy()
    q32.precision = 0
    e32 = Engine(q32, sph, dem)
    e64 = Engine(q, sph, dem)
    e32.step(PREC_STEPS)
    e64.step(PREC_STEPS)

    def rel(a, b):
        den = np.linalg.norm(b)
        return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))

    err = {}
    for which, fields, idn in ((SPH, PREC_SPH, "pid"), (DEM, PREC_DEM, "dem_idx")):
        o32 = np.argsort(e32.get(which, idn))
        o64 = np.argsort(e64.get(which, idn))
        for f in fields:
            err[("dem." if which else "sph.") + f] = rel(e32.get(which, f)[o32], e64.get(which, f)[o64])
    e32.close()
    e64.close()
    worst = max(err, key=err.get)
    cmp = {"steps": PREC_STEPS, "rel_l2": err, "worst_field": worst, "worst": err[worst],
           "how": "FP32 build (FP32 fields, FP64 positions) vs the FP64 build of the same kernels, same input, "
                  f"after {PREC_STEPS} steps, rel. L2 per field matched by particle id"}
    return fp64, cmp


MLP_FWD_FLOP = 2 * (16 * 64 + 64 * 64 + 64)            # per row: 16->64->64->1
MLP_GRAD_FLOP = MLP_FWD_FLOP + 2 * (64 * 64 + 64 * 64 + 16 * 64 + 64)   # + dH1, dW2, dW1, output layer


def run_mlp(args):
    """--workload mlp: the learned warm start's tcgen05 kernels on the scaled
    bed's row count (2,827,520 rows of 16 BF16 features), through the C ABI
    (sphdem_mlp_forward / sphdem_mlp_grad on device arrays); each call's
    kernel time comes from CUDA events around its launch (sphdem_mlp_last_ms).
    Dense BF16 tensor-core work: 10,368 FLOP per row forward, 29,120 per row
    for the gradient pass, against the measured cuBLAS BF16 peak."""
    import ctypes as C

    import torch

    from fluidized_bed_master_b200.engine import lib

    L = lib()
    L.sphdem_mlp_param_count.restype = C.c_int32
    L.sphdem_mlp_forward.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sphdem_mlp_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_double,
                                  C.c_void_p, C.c_void_p]
    L.sphdem_mlp_last_ms.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    n = 2_827_520
    g = torch.Generator(device="cpu").manual_seed(3)
    feat = torch.randn(n, 16, generator=g).to(torch.bfloat16).cuda()
    npar = L.sphdem_mlp_param_count()
    params = (0.2 * torch.randn(npar, generator=g)).float().cuda()
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    target = torch.randn(n, generator=g).float().cuda()
    weight = torch.ones(n, dtype=torch.float32, device="cuda")
    grad = torch.empty(npar + 2, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    fwd, grd = C.c_double(), C.c_double()
    tf, tg = [], []
    for k in range(args.warmup + args.steps):
        r = L.sphdem_mlp_forward(feat.data_ptr(), n, params.data_ptr(), out.data_ptr(), st)
        r |= L.sphdem_mlp_grad(feat.data_ptr(), target.data_ptr(), weight.data_ptr(), n, params.data_ptr(),
                               float(n), grad.data_ptr(), st)
        if r:
            raise RuntimeError(f"mlp entry returned {r}")
        L.sphdem_mlp_last_ms(C.byref(fwd), C.byref(grd))
        if k >= args.warmup:
            tf.append(fwd.value)
            tg.append(grd.value)
    peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("bf16_tflops") if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1590.0
    mf, mg = float(np.median(tf)), float(np.median(tg))
    tff = MLP_FWD_FLOP * n / (mf / 1e3) / 1e12
    tfg = MLP_GRAD_FLOP * n / (mg / 1e3) / 1e12
    line = {"metric": "learned warm start network: rows/s through the tcgen05 kernels", "value": n / (mf / 1e3),
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic (seeded normal features)",
            "config": {"workload": "MLP 16->64->64->1 on 2,827,520 rows (the scaled bed's SPH count)"},
            "forward": {"ms": mf, "tflops": tff, "frac_of_bf16_peak": tff / peak},
            "grad": {"ms": mg, "tflops": tfg, "frac_of_bf16_peak": tfg / peak},
            "roofline": {"bound": "tensor", "achieved": tff, "peak": peak, "unit": "TFLOP/s", "frac": tff / peak,
                         "traffic": None, "kernel": "k_mlp_infer"},
            "how": "median over the timed calls of the CUDA-event time around each kernel launch"}
    print(json.dumps(line), flush=True)


def ppe_comparison(args):
    """PPE ms/step and iterations at a relative residual of 1e-6 on the same
    bed, for four initial iterates of the same Jacobi-PCG (and three of them
    again with the two-level preconditioner, arms *_two_level; *_hist2 with
    2 solution changes instead of 8):
      plain        the previous pressure;
      extrapolated the previous pressure plus its last change;
      projected    the Galerkin projection onto {previous pressure, its
                   one-sweep increment, the last 8 solution changes};
      learned      the same projection with the MLP's predicted change as
                   one more direction, after args.ppe_train training steps.
    Every arm runs the same args.ppe_train steps first (the learned arm
    trains there), then 40 measured steps.  With the converged pressure
    the box beds stay bounded for about 150 steps; after ~200 the
    porosity-rate source of the PPE (2 d_eps - d_eps_prev)/dt and the
    pressure-gradient force on the spheres feed each other until the state
    overflows (with the reference's single sweep they stay bounded), so
    the measurement sits inside the first 150 steps.  Times are the in-graph event
    times of the whole PPE (assembly, features, network, projection and
    iterations).  The bed is the scaled bed (2,000,000 fluid SPH + 200,000
    DEM) unless args.ppe_bed says "bench"."""
    from fluidized_bed_master_b200.beds import box_bed, scaled_box_bed
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import PPE_PCG, PRECOND_TWO_LEVEL, WARM_EXTRAPOLATE, WARM_MLP, WARM_PROJECT

    if args.ppe_bed == "bench":
        p, sph, dem = box_bed(seed=0, **WORKLOAD)
        bed = "box bed (bench workload)"
    else:
        p, sph, dem = scaled_box_bed(seed=0)
        bed = "scaled box bed 1.0x0.02x0.4 m: 2,000,000 fluid SPH + 200,000 DEM"
    meas = 40
    out = {"solver": "Jacobi-PCG, Chronopoulos-Gear form, mass-weighted inner products (FP64 vectors and dots, "
                     "FP32 operator)", "tol": 1e-6, "kgc": 0, "bed": bed, "n_sph": len(sph["x"]),
           "n_dem": len(dem["x"]), "steps_before": args.ppe_train, "measured_steps": meas, "warm_hist": 8}
    arms = (("plain", 0, 0, 8), ("extrapolated", WARM_EXTRAPOLATE, 0, 8), ("projected", WARM_PROJECT, 0, 8),
            ("learned", WARM_MLP, 0, 8), ("plain_two_level", 0, PRECOND_TWO_LEVEL, 8),
            ("projected_two_level", WARM_PROJECT, PRECOND_TWO_LEVEL, 8),
            ("learned_two_level", WARM_MLP, PRECOND_TWO_LEVEL, 8),
            ("projected_two_level_hist2", WARM_PROJECT, PRECOND_TWO_LEVEL, 2),
            ("learned_two_level_hist2", WARM_MLP, PRECOND_TWO_LEVEL, 2))
    for name, warm, precond, hist in arms:
        q = p.copy()
        q.precision = 0
        q.ppe_mode = PPE_PCG
        q.kgc_solve = 0
        q.ppe_tol = 1e-6
        q.ppe_max_iter = 2000
        q.warm_start = warm
        q.warm_hist = hist
        q.warm_fit = 0
        q.mlp_train_steps = args.ppe_train
        q.ppe_precond = precond
        eng = Engine(q, sph, dem)
        eng.step(args.ppe_train)
        eng.set_timing(True)
        its, st, gain = [], 0, []
        for _ in range(meas):
            eng.step(1)
            eng.collect_timing()
            s = eng.stats()
            its.append(s["ppe_iters"])
            st = max(st, s["ppe_status"])
            gain.append(s["ppe_warm_gain"])
        t = eng.timing()
        out[name] = {"ppe_ms_per_step": t["ppe"][0] / max(t["ppe"][1], 1), "iters_per_step": float(np.mean(its)),
                     "converged": st == 0}
        if "ppe.warm_start" in t and t["ppe.warm_start"][1]:
            out[name]["warm_start_ms"] = t["ppe.warm_start"][0] / t["ppe.warm_start"][1]
        if warm == WARM_MLP:
            out[name]["train_loss"] = s["mlp_loss"]
        eng.close()
    out["learned_speedup_vs_plain"] = out["plain"]["ppe_ms_per_step"] / out["learned"]["ppe_ms_per_step"]
    out["learned_speedup_vs_projected"] = out["projected"]["ppe_ms_per_step"] / out["learned"]["ppe_ms_per_step"]
    # the same starts with the two-level preconditioner (ppe_precond TWO_LEVEL) against the Jacobi arms
    out["two_level_speedup_plain"] = out["plain"]["ppe_ms_per_step"] / out["plain_two_level"]["ppe_ms_per_step"]
    out["learned_two_level_speedup_vs_plain"] = (out["plain"]["ppe_ms_per_step"] /
                                                 out["learned_two_level"]["ppe_ms_per_step"])
    out["learned_two_level_hist2_speedup_vs_plain"] = (out["plain"]["ppe_ms_per_step"] /
                                                       out["learned_two_level_hist2"]["ppe_ms_per_step"])
    return out


def run_slabs(args, world, rank, local, pg):
    """The bench bed cut into z slabs (fluidized_bed_master_b200/slabs.py):
    one slab per rank with the ghost bands exchanged over NCCL every step, or
    with one rank --slabs slabs stepped one after another on one GPU.  Each
    timed step is every slab's step plus the exchange; the time is taken by
    the host clock between device synchronisations (the exchange synchronises
    with the host), max over ranks.  value = particles of the whole bed x
    steps / time: the same work at every N, so "scaling" is strong."""
    import torch

    from fluidized_bed_master_b200.beds import box_bed
    from fluidized_bed_master_b200.params import DEM, SPH
    from fluidized_bed_master_b200.slabs import DistExchange, LocalExchange, SlabBed, step_dist, step_local

    from fluidized_bed_master_b200.beds import scaled_box_bed

    torch.cuda.set_device(local)
    if args.slab_bed == "scaled":
        p, sph, dem = scaled_box_bed(seed=0)
        axis, text = 0, "scaled box bed 1.0x0.02x0.4 m: 2,000,000 fluid SPH + 200,000 DEM, cut along x"
    else:
        p, sph, dem = box_bed(seed=0, **WORKLOAD)
        axis, text = 2, WORKLOAD_TEXT
    p.precision = 1 if args.precision == "fp64" else 0
    n_whole = len(sph["x"]) + len(dem["x"])
    if world > 1:
        beds = [SlabBed(p, sph, dem, rank, world, axis=axis)]
        tr = DistExchange()
        run = lambda n: step_dist(beds[0], tr, n)
    else:
        beds = [SlabBed(p, sph, dem, r, args.slabs, axis=axis) for r in range(args.slabs)]
        tr = LocalExchange(args.slabs)
        run = lambda n: step_local(beds, tr, n)
    run(args.warmup)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    run(args.steps)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    if pg:
        pg.barrier()
    t_max = reduce_over_ranks(pg, t, "max", "cuda")
    act = sum(b.eng.slab_active(SPH) + b.eng.slab_active(DEM) for b in beds)
    act_all = reduce_over_ranks(pg, act, "sum", "cuda")
    slabs = [(b.lo, b.hi) for b in beds] if world == 1 else None
    line = {
        "metric": "SPH-DEM particle-updates/s (3-D fluidized bed, ISPH-DEM step, slabs)",
        "value": n_whole * args.steps / t_max, "unit": "particle-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if p.precision == 1 else "f32", "data": "synthetic (seeded box bed)",
        "config": {"workload": text, "axis": "xyz"[axis], "n_sph": len(sph["x"]), "n_dem": len(dem["x"]),
                   "slabs": world if world > 1 else args.slabs, "ghost_layers": beds[0].ghost,
                   "layers": beds[0].n_layers, "slab_layers": slabs,
                   "parallelism": f"slabs x{world}" if world > 1 else f"{args.slabs} slabs on 1 GPU"},
        "active_over_whole": act_all / n_whole,
        "how": "each step: every slab steps, then sends its particles in the neighbours' ghost bands, parks what "
               "left its layers and imports what its neighbours sent (host clock between device syncs)",
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, pg = dist_setup()
    try:
        if args.workload == "dam2d":
            run_dam2d(args, world, rank, local, pg)
        elif args.workload == "dam2d-batch":
            run_dam2d_batch(args, world, rank, local, pg)
        elif args.workload == "bed2d-batch":
            run_bed2d_batch(args, world, rank, local, pg)
        elif args.workload == "column":
            run_column(args, world, rank, local, pg)
        elif args.workload == "mlp":
            if rank == 0:
                run_mlp(args)
        elif args.workload == "ppe-profile":
            if rank == 0:
                run_ppe_profile(args)
        elif args.workload == "slabs":
            run_slabs(args, world, rank, local, pg)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_engine(args, world, rank, local, pg)
    finally:
        if pg:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
