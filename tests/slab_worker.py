"""One rank of a slab-decomposition test, launched by tests/test_slab.py and
tests/test_gpu_slab.py with RANK, WORLD_SIZE, MASTER_ADDR and MASTER_PORT in the
environment (gloo process group, host tensors).

  slab_worker.py routing OUT     exchange of seeded records only (CPU)
  slab_worker.py neighbours OUT  the neighbour-only exchange of seeded records (CPU)
  slab_worker.py engine OUT K N  the DPD box of N particles in 16 x 8 x 8 cells decomposed
                                 into slabs, K steps on cuda:0; rank 0 writes the gathered state
"""
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def routing(rank, world, out):
    from mechanica_b200 import slab
    recs = []
    for r in range(world):  # every rank can draw every rank's records from the shared seed
        rng = np.random.default_rng(100 + r)
        n = int(rng.integers(0, 50))
        recs.append(slab.pack(rng.integers(0, world, n).astype(np.int32), rng.integers(0, 10**6, n).astype(np.int32),
                              rng.integers(0, 3, n).astype(np.int32), rng.integers(0, 999, n).astype(np.int32),
                              rng.random((n, 3)).astype(np.float32), rng.random((n, 3)).astype(np.float32)))
    got = slab.exchange(recs[rank], rank, world)
    want = np.concatenate([r[r["dest"] == rank] for r in recs])
    ok = got.tobytes() == want.tobytes()
    with open(f"{out}.{rank}", "w") as f:
        f.write("ok" if ok else f"mismatch {len(got)} {len(want)}")


def neighbours(rank, world, out):
    """Every rank sends seeded records to its two neighbours on the ring of slabs (below and
    above, periodic) and must receive exactly the records addressed to it, in source-rank order."""
    from mechanica_b200 import slab

    def peers(r):
        return sorted({(r - 1) % world, (r + 1) % world} - {r})

    recs = []
    for r in range(world):
        rng = np.random.default_rng(200 + r)
        n = int(rng.integers(0, 60))
        p = np.asarray(peers(r), dtype=np.int32)
        dest = p[rng.integers(0, len(p), n)] if len(p) else np.zeros(0, dtype=np.int32)
        recs.append(slab.pack(dest.astype(np.int32), rng.integers(0, 10**6, n).astype(np.int32),
                              rng.integers(0, 3, n).astype(np.int32), rng.integers(0, 999, n).astype(np.int32),
                              rng.random((n, 3)).astype(np.float32), rng.random((n, 3)).astype(np.float32)))
    got = slab.exchange_neighbours(recs[rank], rank, world, peers(rank))
    want = np.concatenate([recs[r][recs[r]["dest"] == rank] for r in range(world) if r in peers(rank)] +
                          [np.zeros(0, dtype=slab.RECORD)])
    ok = got.tobytes() == want.tobytes()
    with open(f"{out}.{rank}", "w") as f:
        f.write("ok" if ok else f"mismatch {len(got)} {len(want)}")


def engine(rank, world, out, K, N):
    import torch
    torch.cuda.set_device(0)
    import mechanica_b200 as m
    from mechanica_b200 import slab
    from mechanica_b200 import workloads as W
    scn = W.dpd(n=N, dims=(16.0, 8.0, 8.0), seed=7)
    W.build_gpu(scn)
    s = slab.Slab(m.universe, rank, world)
    s.steps(K)
    c, xr, v = s.gather()
    if rank == 0:
        np.savez(out, cell=c, xr=xr, v=v, ranges=np.array(s.ranges))
    m.universe.close()


if __name__ == "__main__":
    import torch.distributed as dist
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        if sys.argv[1] == "routing":
            routing(rank, world, sys.argv[2])
        elif sys.argv[1] == "neighbours":
            neighbours(rank, world, sys.argv[2])
        else:
            engine(rank, world, sys.argv[2], int(sys.argv[3]), int(sys.argv[4]))
    finally:
        dist.destroy_process_group()
