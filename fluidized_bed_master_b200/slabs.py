"""A spatially sharded ISPH-DEM bed: one slab of cell layers per rank.

The reference shards only its WCSPH step: x slabs, each GPU holding its own
particles plus a halo received from its neighbours every step
(SOPHIA_multi, WCSPH_Calc.cuh:368-738; the send/receive marking of
functions_NNPS.cuh:202-303).  SlabBed carries that scheme to the ISPH-DEM
step on top of the engine's slab calls (include/sphdem.h, sphdem_slab_*):

* the whole bed's cell grid is cut along one axis into slabs of whole cell
  layers [lo, hi), one per rank, balanced by SPH particle count;
* a rank's handle holds its own layers, a ghost band of G layers on each
  side, and spare slots parked with i_type 3;
* between steps a rank sends the particles of its own layers that lie in a
  neighbour's ghost band (those are exact here), parks everything outside
  its own layers (the stale ghosts and the particles that left), and imports
  what its neighbours sent: their exact particles of its ghost bands, and the
  particles that crossed into its layers.

One step moves information by one cell layer per dependent neighbour pass:
the SPH and DEM lists, pass A, pass B, the DEM coupling, the SPH coupling,
the walls, the PPE sweep, the walls again, pass C, the open boundary and
XSPH, eleven in all, plus the first step's extra wall pass.  With
G >= 12 the particles of a rank's own layers are exact after every step:
they step as in the unsharded bed, up to the order of the sums inside a cell.
The price is the redundant stepping of 2G ghost layers per slab, against one
exchange per step instead of one per pass.

Transports: DistExchange moves the records with torch.distributed
point-to-point operations (NCCL between GPUs; gloo with CPU copies), and
LocalExchange hands them between SlabBeds of one process (several slabs on
one GPU, for tests).  The PPE must be the reference's sweep: a Krylov solve
needs global dot products, which this scheme does not provide.
"""
import numpy as np

from .engine import Engine, bed_domain
from .params import DEM, PPE_REFERENCE, SPH

GHOST_LAYERS = 12


def cell_layer(v, vmin, vmax, n):
    """Cell index along one axis, as the engine's hash computes it
    (functions_NNPS.cuh:776: min(floor((v - vmin) / (vmax - vmin) * n), n - 1),
    clamped at 0)."""
    v = np.asarray(v, dtype=np.float64)
    if vmax == vmin:
        return np.zeros(v.shape, dtype=np.int64)
    k = np.minimum(np.floor((v - vmin) / (vmax - vmin) * n), n - 1)
    return np.maximum(k, 0).astype(np.int64)


def grid_layers(params, bbox, h0, axis):
    """Number of cell layers along axis of the bed's grid (dcell = 1.1 kappa h0)."""
    dcell = 1.1 * params.kappa * h0
    return int((bbox[2 * axis + 1] - bbox[2 * axis]) / dcell) + 1


def split_layers(layers_of_sph, n_layers, world, ghost):
    """Slab bounds [lo_r, hi_r) over n_layers, with about equal SPH counts and
    every slab at least `ghost` layers wide (so that a ghost band lies inside
    the neighbouring slab)."""
    if world * ghost > n_layers:
        raise ValueError(f"{world} slabs of at least {ghost} layers do not fit in {n_layers} layers")
    hist = np.bincount(layers_of_sph, minlength=n_layers).astype(np.float64)
    cum = np.cumsum(hist)
    total = cum[-1] if len(cum) else 0.0
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left")) + 1
        b = max(b, bounds[-1] + ghost)
        b = min(b, n_layers - (world - r) * ghost)
        bounds.append(b)
    bounds.append(n_layers)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def _with_parked(d, idx, spare, ids_key, park_ids):
    """The rows idx of d followed by `spare` parked rows: copies of the first
    row with i_type 3 and their own ids (park_ids)."""
    out = {}
    src = idx[:1] if len(idx) else np.zeros(1, dtype=np.int64)
    for k, v in d.items():
        v = np.asarray(v)
        out[k] = np.concatenate([v[idx], np.repeat(v[src], spare, axis=0)])
    out["i_type"] = np.concatenate([np.asarray(d["i_type"])[idx], np.full(spare, 3, dtype=np.asarray(d["i_type"]).dtype)])
    if ids_key in out:
        out[ids_key] = np.concatenate([np.asarray(d[ids_key])[idx], park_ids]).astype(np.asarray(d[ids_key]).dtype)
    return out


class LocalExchange:
    """Records handed between the SlabBeds of one process (same device)."""

    def __init__(self, world):
        self.world = world
        self.box = {}

    def post(self, src, dst, payload):
        self.box[(src, dst)] = payload

    def take(self, src, dst):
        return self.box.pop((src, dst))


class DistExchange:
    """Records between ranks over torch.distributed: per neighbour first the
    record counts, then the records, as batched point-to-point operations.
    With a gloo group the records travel through host memory."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.host = dist.get_backend(group) == "gloo"

    def exchange(self, rank, sends):
        """sends: {neighbour rank: (sph uint8 tensor, dem uint8 tensor)};
        returns {neighbour rank: (sph, dem)} received."""
        import torch

        dist = self.dist
        dev = torch.device("cpu") if self.host else torch.device("cuda", torch.cuda.current_device())
        nbrs = sorted(sends)
        cnt_out = {q: torch.tensor([sends[q][0].numel(), sends[q][1].numel()], dtype=torch.int64, device=dev)
                   for q in nbrs}
        cnt_in = {q: torch.zeros(2, dtype=torch.int64, device=dev) for q in nbrs}
        ops = []
        for q in nbrs:
            ops.append(dist.P2POp(dist.isend, cnt_out[q], q, group=self.group))
            ops.append(dist.P2POp(dist.irecv, cnt_in[q], q, group=self.group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        out_buf, in_buf, ops = {}, {}, []
        for q in nbrs:
            a, b = sends[q]
            out_buf[q] = torch.cat([a.reshape(-1), b.reshape(-1)]).to(dev)
            na, nb = (int(v) for v in cnt_in[q].tolist())
            in_buf[q] = (torch.empty(na + nb, dtype=torch.uint8, device=dev), na)
            if out_buf[q].numel():
                ops.append(dist.P2POp(dist.isend, out_buf[q], q, group=self.group))
            if na + nb:
                ops.append(dist.P2POp(dist.irecv, in_buf[q][0], q, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        got = {}
        for q in nbrs:
            buf, na = in_buf[q]
            if self.host:
                buf = buf.cuda() if torch.cuda.is_available() else buf
            got[q] = (buf[:na], buf[na:])
        return got


class SlabBed:
    """One slab of a bed on this rank (see the module docstring).

    params, sph, dem: the whole bed, as for Engine (every rank passes the
    same arrays).  axis: 0 x, 1 y, 2 z.  ghost: ghost layers per side.
    spare: parked slots as a fraction of the slab's initial particles.
    engine: the engine class (tests substitute a model with the same slab
    calls)."""

    def __init__(self, params, sph, dem, rank, world, axis=2, ghost=GHOST_LAYERS, spare=0.5, engine=Engine):
        if params.ppe_mode != PPE_REFERENCE:
            raise ValueError("a sharded bed runs the reference PPE sweep (a Krylov solve needs global dot products)")
        self.rank, self.world, self.axis, self.ghost = rank, world, axis, ghost
        bbox, h0, t_ref = bed_domain(params, sph, dem) if engine is Engine else engine.bed_domain(params, sph, dem)
        # every particle keeps its row in the whole bed as its id; i_type 3
        # marks the parked spare slots (the others are tagged at commit)
        if sph:
            sph = dict(sph, pid=np.arange(len(sph["x"]), dtype=np.int32),
                       i_type=np.ones(len(sph["x"]), dtype=np.int32))
        if dem:
            dem = dict(dem, pid=np.arange(len(dem["x"]), dtype=np.int32),
                       i_type=np.ones(len(dem["x"]), dtype=np.int32))
        self.domain = (bbox, h0, t_ref)
        self.n_layers = grid_layers(params, bbox, h0, axis)
        lo_v, hi_v = bbox[2 * axis], bbox[2 * axis + 1]
        key = "xyz"[axis]
        ls = cell_layer(sph[key], lo_v, hi_v, self.n_layers) if sph else np.zeros(0, np.int64)
        ld = cell_layer(dem[key], lo_v, hi_v, self.n_layers) if dem else np.zeros(0, np.int64)
        self.slabs = split_layers(ls, self.n_layers, world, ghost)
        self.lo, self.hi = self.slabs[rank]
        glo, ghi = self.lo - ghost, self.hi + ghost
        si = np.flatnonzero((ls >= glo) & (ls < ghi))
        di = np.flatnonzero((ld >= glo) & (ld < ghi))
        ns_sp = int(np.ceil(len(si) * spare)) + 64
        nd_sp = int(np.ceil(len(di) * spare)) + 16 if dem else 0
        sph_r = _with_parked(sph, si, ns_sp, "pid", -1 - np.arange(ns_sp)) if sph else sph
        dem_r = None
        if dem:
            top = int(np.max(dem["dem_idx"])) if len(dem["dem_idx"]) else 0
            dem_r = _with_parked(dem, di, nd_sp, "dem_idx", top + 1 + np.arange(nd_sp))
        self.eng = engine(params, sph_r, dem_r, domain=self.domain)
        self.nbrs = [q for q in (rank - 1, rank + 1) if 0 <= q < world]

    def _band_to(self, q):
        """Layers of this slab that lie in neighbour q's ghost band."""
        return (self.hi - self.ghost, self.hi) if q > self.rank else (self.lo, self.lo + self.ghost)

    def exchange(self, transport):
        """Refresh the ghost bands and hand over the particles that crossed
        a slab boundary (after a step)."""
        sends = {}
        for q in self.nbrs:
            lo, hi = self._band_to(q)
            a = self.eng.slab_export(SPH, self.eng.slab_select(SPH, self.axis, lo, hi)) if self.eng.ns else None
            b = self.eng.slab_export(DEM, self.eng.slab_select(DEM, self.axis, lo, hi)) if self.eng.nd else None
            sends[q] = (a, b)
        if isinstance(transport, LocalExchange):
            for q, pay in sends.items():
                transport.post(self.rank, q, pay)
            return None
        got = transport.exchange(self.rank, {q: tuple(_empty_if_none(v) for v in pay) for q, pay in sends.items()})
        self.absorb(got)
        return got

    def absorb(self, got):
        """Park everything outside this slab's layers, then import the
        neighbours' records."""
        if self.eng.ns:
            self.eng.slab_keep(SPH, self.axis, self.lo, self.hi)
        if self.eng.nd:
            self.eng.slab_keep(DEM, self.axis, self.lo, self.hi)
        for q in sorted(got):
            a, b = got[q]
            if self.eng.ns and a is not None and a.numel():
                self.eng.slab_import(SPH, a)
            if self.eng.nd and b is not None and b.numel():
                self.eng.slab_import(DEM, b)

    def owned(self, which, fields):
        """{field: values} of the particles of this slab's own layers, with
        their rows in the whole bed ('pid'; spheres also 'dem_idx')."""
        key = "xyz"[self.axis]
        bbox = self.domain[0]
        it = self.eng.get(which, "i_type")
        lay = cell_layer(self.eng.get(which, key), bbox[2 * self.axis], bbox[2 * self.axis + 1], self.n_layers)
        m = (it != 3) & (lay >= self.lo) & (lay < self.hi)
        out = {f: self.eng.get(which, f)[m] for f in fields}
        out["pid"] = self.eng.get(which, "pid")[m]
        if which == DEM:
            out["dem_idx"] = self.eng.get(which, "dem_idx")[m]
        return out


def _empty_if_none(t):
    import torch

    if t is not None:
        return t
    return torch.empty(0, dtype=torch.uint8, device="cuda" if torch.cuda.is_available() else "cpu")


def step_local(beds, transport, n=1):
    """Advance the SlabBeds of one process n steps, exchanging after each."""
    for _ in range(n):
        for b in beds:
            b.eng.step(1)
        for b in beds:
            b.exchange(transport)
        for b in beds:
            got = {q: transport.take(q, b.rank) for q in b.nbrs}
            b.absorb(got)


def step_dist(bed, transport, n=1):
    """Advance this rank's SlabBed n steps, exchanging after each."""
    for _ in range(n):
        bed.eng.step(1)
        bed.exchange(transport)
