"""Spatial decomposition of one simulation box across ranks: slabs of whole cells along x.

Each rank owns a slab of cell layers [x0, x1) and its engine holds the slab's particles plus
one layer of ghost cells on each side (cells are no smaller than the cutoff, so one layer
holds every partner of a slab particle) -- the ghost-cell scheme of the reference's MPI
exchange (engine_exchange, src/mdcore/src/engine_exchange.cpp:767-964), which the reference
never built. One step:

1. ghosts: every rank sends the particles of its first and last cell layer to the ranks on
   either side, in the engine's own representation (cell, FP32 cell-relative position,
   velocity, type, id), so nothing is placed again;
2. the rank's engine is built over the whole box's grid from its particles and the ghosts, in
   ascending particle id, with the whole box's work-item split (the occupancy hint): every cell
   of the slab then holds the same particles in the same slots as in the undivided box, its
   cell pairs are the same work items, and the forces on its particles are the same sums in the
   same order, bit for bit (a ghost's own force misses its far partners and is discarded);
3. one engine step; the rank keeps the particles that stayed in its slab and sends the ones that
   left it (into a ghost layer) to the rank that owns their new cell.

Both exchanges are point-to-point with the two neighbouring slabs only (torch.distributed
isend / irecv: gloo with host tensors, or NCCL with device tensors), counts first, then the
records into the receiver's buffer; gather() collects the whole state with all-gathers. The engine is
rebuilt every step (a slab's particle count changes from step to step), so this path gives the
decomposition's results, not the speed of a resident multi-GPU engine. Not decomposed: bonds,
angles, dihedrals, exclusions, species, large particles and cuboids (refused), and the Philox
random streams (keyed on engine-local ids: refused); x must be periodic, and every slab at least
two cell layers wide.
"""
import ctypes

import numpy as np

from ._native import check, lib

# one particle as it crosses between ranks: the engine's own representation
RECORD = np.dtype([("dest", "<i4"), ("id", "<i4"), ("type", "<i4"), ("cell", "<i4"), ("xr", "<f4", (3,)),
                   ("v", "<f4", (3,))])


def slab_ranges(ncx, world):
    """The cell layers [x0, x1) of every rank: contiguous, in rank order, widths differing by at
    most one layer; every width at least 2 (a rank's first and last layers are then distinct, so
    that its ghosts reach each neighbour once)."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    if world > 1 and ncx < 2 * world:
        raise ValueError(f"{ncx} cell layers along x cannot give {world} slabs of two layers or more")
    base, extra = divmod(ncx, world)
    out, x0 = [], 0
    for r in range(world):
        w = base + (1 if r < extra else 0)
        out.append((x0, x0 + w))
        x0 += w
    return out


def owner_of_layers(ranges, ncx):
    """The rank owning each cell layer along x."""
    own = np.empty(ncx, dtype=np.int32)
    for r, (x0, x1) in enumerate(ranges):
        own[x0:x1] = r
    return own


def ghost_records(cell, layer_owner, rank, ranges, ncyz, ncx):
    """Destinations of a rank's boundary particles as ghosts: the first layer goes to the rank
    owning the layer below it, the last to the rank owning the layer above (periodic in x); a
    rank whose slab is the whole box (one rank) has its periodic neighbours in its own engine and
    sends nothing. Returns (index into the arrays, destination rank) pairs."""
    x0, x1 = ranges[rank]
    lx = cell // ncyz
    first = np.flatnonzero(lx == x0)
    last = np.flatnonzero(lx == x1 - 1)
    below, above = int(layer_owner[(x0 - 1) % ncx]), int(layer_owner[x1 % ncx])
    idx, dest = [np.zeros(0, dtype=np.int64)], [np.zeros(0, dtype=np.int32)]
    if below != rank:
        idx.append(first)
        dest.append(np.full(len(first), below, dtype=np.int32))
    if above != rank:
        idx.append(last)
        dest.append(np.full(len(last), above, dtype=np.int32))
    return np.concatenate(idx), np.concatenate(dest)


def pack(dest, ids, types, cells, xr, v):
    rec = np.zeros(len(ids), dtype=RECORD)
    rec["dest"], rec["id"], rec["type"], rec["cell"] = dest, ids, types, cells
    rec["xr"], rec["v"] = xr, v
    return rec


def exchange(records, rank, world, group=None, device=None):
    """All-gathers every rank's outgoing records and returns the ones addressed to this rank, in
    source-rank order (sizes first, then the records padded to the largest count)."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return records[records["dest"] == rank]
    dev = device or torch.device("cpu")
    size = records.dtype.itemsize
    n = torch.tensor([len(records)], dtype=torch.int64, device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    nmax = max(1, max(sizes))
    buf = torch.zeros(nmax * size, dtype=torch.uint8, device=dev)
    if len(records):
        buf[: len(records) * size] = torch.from_numpy(np.ascontiguousarray(records).view(np.uint8)).to(dev)
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    out = []
    for r in range(world):
        a = np.frombuffer(bufs[r][: sizes[r] * size].cpu().numpy().tobytes(), dtype=RECORD)
        out.append(a[a["dest"] == rank])
    return np.concatenate(out) if out else np.zeros(0, dtype=RECORD)


def exchange_neighbours(records, rank, world, peers, group=None, device=None):
    """Point-to-point exchange with the neighbouring slabs only (ghosts and leavers never go
    further: a particle moves less than one cell layer per step, and every slab is at least two
    layers wide). Every record must be addressed to one of `peers` (the distinct neighbour
    ranks). Each pair of neighbours swaps the count, then the records, straight into the
    receiver's buffer (torch.distributed isend / irecv: gloo with host tensors, NCCL with
    device tensors). Returns the records received, in ascending source rank."""
    import torch
    import torch.distributed as dist
    if world == 1 or not peers:
        return records[records["dest"] == rank]
    bad = ~np.isin(records["dest"], np.asarray(list(peers), dtype=np.int32))
    if bad.any():
        raise RuntimeError(f"slab rank {rank}: records addressed beyond the neighbouring slabs {sorted(peers)}")
    dev = device or torch.device("cpu")
    size = records.dtype.itemsize
    peers = sorted(peers)
    out_n = {p: torch.tensor([int((records["dest"] == p).sum())], dtype=torch.int64, device=dev) for p in peers}
    in_n = {p: torch.zeros(1, dtype=torch.int64, device=dev) for p in peers}
    reqs = [dist.irecv(in_n[p], src=p, group=group) for p in peers]
    reqs += [dist.isend(out_n[p], dst=p, group=group) for p in peers]
    for r in reqs:
        r.wait()
    sends, recvs, reqs = {}, {}, []
    for p in peers:
        n_in = int(in_n[p].item())
        if n_in:
            recvs[p] = torch.empty(n_in * size, dtype=torch.uint8, device=dev)
            reqs.append(dist.irecv(recvs[p], src=p, group=group))
    for p in peers:
        sel = records[records["dest"] == p]
        if len(sel):
            sends[p] = torch.from_numpy(np.ascontiguousarray(sel).view(np.uint8).copy()).to(dev)
            reqs.append(dist.isend(sends[p], dst=p, group=group))
    for r in reqs:
        r.wait()
    got = [np.frombuffer(recvs[p].cpu().numpy().tobytes(), dtype=RECORD) for p in peers if p in recvs]
    return np.concatenate(got) if got else np.zeros(0, dtype=RECORD)


class Slab:
    """This rank's slab of a universe built for the whole box (types, potentials, forces and all
    particles, as on a single GPU; every rank builds the same one). The whole box is placed once
    by the engine, each rank keeps the particles of its slab, and from then on steps(k) advances
    the decomposed system; gather() collects the whole state on every rank."""

    def __init__(self, universe, rank, world, group=None, device=None):
        u = universe
        if u.rng == "philox":
            raise ValueError("the slab path keeps the reference random term (Philox streams are keyed on "
                             "engine-local particle ids)")
        if u._bonds or u._angles or u._dihedrals or u._exclusions or u._species or u._cuboids or u._replicas:
            raise ValueError("the slab path decomposes nonbonded systems of one box (no bonds, angles, "
                             "dihedrals, exclusions, species, cuboids or extra replicas)")
        if any(float(np.float32(r)) > u.cutoff for (_, r, _, _) in u._types):
            raise ValueError("the slab path has no large particles (a type's radius above the cutoff)")
        self.u, self.rank, self.world, self.group, self.device = u, rank, world, group, device
        u._ensure()
        per = ctypes.c_uint()
        check(lib().mxg_engine_space_info(u._e, None, None, None, ctypes.byref(per)), "space_info")
        if not (per.value & 1):
            raise ValueError("the slab path cuts the box along x, which must be periodic")
        self.cdim, self.h = u.cell_grid()
        self.ncyz = int(self.cdim[1] * self.cdim[2])
        self.ncx = int(self.cdim[0])
        self.ranges = slab_ranges(self.ncx, world)
        self.layer_owner = owner_of_layers(self.ranges, self.ncx)
        x0, x1 = self.ranges[rank]
        self.peers = sorted({int(self.layer_owner[(x0 - 1) % self.ncx]), int(self.layer_owner[x1 % self.ncx])} - {rank})
        x, v, f, cell, xr = u.state()
        self.n_total = len(cell)
        mine = self.layer_owner[cell // self.ncyz] == rank
        self.ids = np.flatnonzero(mine).astype(np.int32)
        self.types = u._t[mine].astype(np.int32)
        self.cells = cell[mine].astype(np.int32)
        self.xr = xr[mine].astype(np.float32)
        self.v = v[mine].astype(np.float32)
        self.count = 0  # steps taken (the engine's step counter)

    def _build(self, ids, types, cells, xr, v):
        """The rank's engine over the whole grid with the given particles (ascending id)."""
        u = self.u
        order = np.argsort(ids, kind="stable")
        u._x = np.zeros((len(ids), 3))  # unused: every particle is added by cell
        u._v = v[order].astype(np.float32)
        u._t = types[order].astype(np.int32)
        u._r = np.zeros(len(ids), dtype=np.int32)
        u._c = cells[order].astype(np.int32)
        u._xr = xr[order].astype(np.float32)
        u._spec = np.zeros((len(ids), 0), dtype=np.float32)
        u.occupancy_hint = self.n_total
        u._dirty = True
        u._ensure()
        check(lib().mxg_engine_set_step_counter(u._e, self.count), "set_step_counter")
        return order

    def step(self):
        rank, world = self.rank, self.world
        # 1. ghosts from the neighbouring slabs
        gi, gd = ghost_records(self.cells, self.layer_owner, rank, self.ranges, self.ncyz, self.ncx)
        sent = pack(gd, self.ids[gi], self.types[gi], self.cells[gi], self.xr[gi], self.v[gi])
        ghosts = exchange_neighbours(sent, rank, world, self.peers, self.group, self.device)
        # 2. the rank's engine: own particles, then ghosts, placed in ascending id
        ids = np.concatenate([self.ids, ghosts["id"]])
        types = np.concatenate([self.types, ghosts["type"]])
        cells = np.concatenate([self.cells, ghosts["cell"]])
        xr = np.concatenate([self.xr, ghosts["xr"]])
        v = np.concatenate([self.v, ghosts["v"]])
        order = self._build(ids, types, cells, xr, v)
        # 3. one step; the slab's particles by their position in the engine (local id)
        self.u.steps(1)
        _, v1, _, c1, xr1 = self.u.state()
        local = np.empty(len(ids), dtype=np.int64)
        local[order] = np.arange(len(ids))
        own = local[: len(self.ids)]
        nc, nxr, nv = c1[own], xr1[own], v1[own]
        dest = self.layer_owner[nc // self.ncyz]
        stay = dest == rank
        leavers = pack(dest[~stay], self.ids[~stay], self.types[~stay], nc[~stay], nxr[~stay], nv[~stay])
        arrived = exchange_neighbours(leavers, rank, world, self.peers, self.group, self.device)
        self.ids = np.concatenate([self.ids[stay], arrived["id"]]).astype(np.int32)
        self.types = np.concatenate([self.types[stay], arrived["type"]]).astype(np.int32)
        self.cells = np.concatenate([nc[stay], arrived["cell"]]).astype(np.int32)
        self.xr = np.concatenate([nxr[stay], arrived["xr"]]).astype(np.float32)
        self.v = np.concatenate([nv[stay], arrived["v"]]).astype(np.float32)
        self.count += 1

    def steps(self, k):
        for _ in range(int(k)):
            self.step()

    def gather(self):
        """(cell, cell-relative position, velocity) of every particle by id, on every rank."""
        rec = pack(np.full(len(self.ids), -1, dtype=np.int32), self.ids, self.types, self.cells, self.xr, self.v)
        allr = []
        for r in range(self.world):
            rec["dest"] = r
            allr.append(rec.copy())
        got = exchange(np.concatenate(allr), self.rank, self.world, self.group, self.device)
        if len(got) != self.n_total or len(np.unique(got["id"])) != self.n_total:
            raise RuntimeError(f"slab gather: {len(got)} records for {self.n_total} particles")
        got = got[np.argsort(got["id"])]
        return got["cell"].copy(), got["xr"].copy(), got["v"].copy()
