"""The slab exchange protocol of fluidized_bed_master_b200/slabs.py over
torch.distributed (gloo, world sizes 2 and 3, on CPU).

The engine is replaced by a model with the same slab calls (select, export,
keep, import, active) whose particles move with their own constant velocity,
so that many of them cross slab boundaries; the real bed domain and cell
layers are used.  After every step and exchange:
* every particle is active on exactly one rank inside that rank's own layers,
  at the position of the same motion run on the whole bed;
* each rank's ghost bands hold exactly the particles of the whole bed that
  lie in them;
* parked slots are reused, and nothing is lost when particles cross.
The GPU test (tests/test_slabs_gpu.py) runs the same driver on the engine.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DT = 4.0e-4
STEPS = 6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bed(seed=5):
    sys.path.insert(0, ROOT)
    from fluidized_bed_master_b200.engine import default_params

    rng = np.random.default_rng(seed)
    p = default_params()
    p.solver_type = 1
    p.dim = 3
    p.kappa = 2.0
    h = 2.0e-3
    n, nd = 3000, 300

    def cloud(m):
        return {"x": rng.uniform(0, 0.02, m), "y": rng.uniform(0, 0.02, m), "z": rng.uniform(0, 0.3, m),
                "ux": rng.uniform(-1, 1, m), "uy": rng.uniform(-1, 1, m), "uz": rng.uniform(-40, 40, m),
                "h": np.full(m, h), "temp": np.full(m, 300.0), "p_type": np.ones(m, dtype=np.int32)}

    sph = cloud(n)
    dem = cloud(nd)
    dem["p_type"] = np.full(nd, 1001, dtype=np.int32)
    dem["dem_idx"] = np.arange(1, nd + 1, dtype=np.int32)
    return p, sph, dem


class ModelEngine:
    """Particles moving with constant velocity, with the engine's slab calls
    on CPU tensors.  A record is (id, x, y, z, ux, uy, uz) as doubles."""

    def __init__(self, params, sph, dem, domain=None):
        from fluidized_bed_master_b200.slabs import grid_layers

        self.domain = domain
        self.n_layers = grid_layers(params, domain[0], domain[1], 2)
        self.sets = []
        for d in (sph, dem):
            s = {k: np.array(d[k], dtype=np.float64) for k in ("x", "y", "z", "ux", "uy", "uz")}
            s["pid"] = np.array(d["pid"], dtype=np.int64)
            s["i_type"] = np.where(np.asarray(d["i_type"]) == 3, 3, 1)
            self.sets.append(s)
        self.ns, self.nd = len(sph["x"]), len(dem["x"])

    @staticmethod
    def bed_domain(params, sph, dem):
        from fluidized_bed_master_b200.engine import bed_domain

        return bed_domain(params, sph, dem)

    def step(self, n=1):
        for s in self.sets:
            a = s["i_type"] != 3
            for _ in range(n):
                for c in "xyz":
                    s[c][a] = s[c][a] + s["u" + c][a] * DT

    def get(self, which, f):
        return self.sets[which][f].copy()

    def _layer(self, which, axis):
        from fluidized_bed_master_b200.slabs import cell_layer

        s = self.sets[which]
        bb = self.domain[0]
        lay = cell_layer(s["xyz"[axis]], bb[2 * axis], bb[2 * axis + 1], self.n_layers)
        return np.where(s["i_type"] == 3, -1, lay)

    def slab_select(self, which, axis, lo, hi):
        import torch

        lay = self._layer(which, axis)
        return torch.from_numpy(np.flatnonzero((lay >= lo) & (lay < hi)).astype(np.int32))

    def slab_export(self, which, slots):
        import torch

        s = self.sets[which]
        i = slots.numpy()
        rec = np.stack([s["pid"][i].astype(np.float64)] + [s[k][i] for k in ("x", "y", "z", "ux", "uy", "uz")], 1)
        return torch.from_numpy(np.ascontiguousarray(rec).view(np.uint8).reshape(-1))

    def slab_keep(self, which, axis, lo, hi):
        lay = self._layer(which, axis)
        s = self.sets[which]
        s["i_type"][(lay >= 0) & ((lay < lo) | (lay >= hi))] = 3

    def slab_import(self, which, records):
        rec = records.numpy().view(np.float64).reshape(-1, 7)
        s = self.sets[which]
        free = np.flatnonzero(s["i_type"] == 3)[: len(rec)]
        assert len(free) == len(rec), "out of parked slots"
        s["pid"][free] = rec[:, 0].astype(np.int64)
        for c, k in enumerate(("x", "y", "z", "ux", "uy", "uz")):
            s[k][free] = rec[:, 1 + c]
        s["i_type"][free] = 1

    def slab_active(self, which):
        return int((self.sets[which]["i_type"] != 3).sum())


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from fluidized_bed_master_b200.params import DEM, SPH
    from fluidized_bed_master_b200.slabs import DistExchange, SlabBed, cell_layer, step_dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        p, sph, dem = _bed()
        bed = SlabBed(p, sph, dem, rank, world, axis=2, ghost=4, spare=1.0, engine=ModelEngine)
        tr = DistExchange()
        out = []
        for k in range(STEPS):
            step_dist(bed, tr, 1)
            snap = {}
            for which in (SPH, DEM):
                e = bed.eng.sets[which]
                lay = bed.eng._layer(which, 2)
                act = e["i_type"] != 3
                snap[which] = {"pid": e["pid"][act], "z": e["z"][act], "lay": lay[act]}
            out.append(snap)
        q.put((rank, bed.lo, bed.hi, bed.n_layers, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_protocol_over_gloo(world):
    import torch.multiprocessing as mp

    sys.path.insert(0, ROOT)
    from fluidized_bed_master_b200.engine import bed_domain
    from fluidized_bed_master_b200.params import DEM, SPH
    from fluidized_bed_master_b200.slabs import cell_layer, grid_layers

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    for _ in range(world):
        r, lo, hi, nl, out = q.get(timeout=240)
        got[r] = (lo, hi, nl, out)
    for pr in procs:
        pr.join(60)
        assert pr.exitcode == 0
    # the same motion on the whole bed
    p, sph, dem = _bed()
    bbox, h0, _ = bed_domain(p, sph, dem)
    nl = grid_layers(p, bbox, h0, 2)
    ghost = 4
    ref = [{k: np.array(d[k], dtype=np.float64) for k in ("z", "uz")} for d in (sph, dem)]
    assert [got[r][0] for r in range(world)][0] == 0 and got[world - 1][1] == nl
    for r in range(world - 1):
        assert got[r][1] == got[r + 1][0], "slabs tile the layers"
    crossed = 0
    prev = {}
    for k in range(STEPS):
        for which in (SPH, DEM):
            ref[which]["z"] = ref[which]["z"] + ref[which]["uz"] * DT
            zr = ref[which]["z"]
            lay = cell_layer(zr, bbox[4], bbox[5], nl)
            owners = np.full(len(zr), -1)
            for r in range(world):
                lo, hi, _, out = got[r]
                s = out[k][which]
                own = (s["lay"] >= lo) & (s["lay"] < hi)
                assert np.all(owners[s["pid"][own]] == -1), "a particle owned twice"
                owners[s["pid"][own]] = r
                assert np.array_equal(s["z"], zr[s["pid"]]), "a slab's particle left the whole bed's motion"
                # ghost bands hold exactly the whole bed's particles there
                band = ((lay >= lo - ghost) & (lay < lo)) | ((lay >= hi) & (lay < hi + ghost))
                ghost_ids = np.sort(s["pid"][~own])
                assert np.array_equal(ghost_ids, np.flatnonzero(band)), (k, which, r)
            assert np.all(owners >= 0), "a particle owned by no slab"
            if k:
                crossed += int((owners != prev[which]).sum())
            prev[which] = owners
    assert crossed > 50, "too few particles crossed a slab boundary for the test to mean anything"
