"""Slab decomposition on the GPU: a DPD box (4,000 particles, 16 x 8 x 8 cells, periodic in x
and y, no-slip walls in z, the reference random term, a body force) split along x into 1, 2 and
3 slabs, each rank a separate process with its own engine on the same GPU (gloo exchanges
through host memory; no kernel of one rank waits on another's). After 5 steps every particle's
cell, FP32 cell-relative position and velocity are bit-identical to the undivided box stepped
by one engine: the ghosts carry the engine's own representation, the slab engines place
particles in ascending id and split their work items as the whole box does, so every force
sum on a slab particle has the same terms in the same order."""
import numpy as np
import pytest

import mechanica_b200 as m
from mechanica_b200 import workloads as W
from slab_launch import run_ranks

pytestmark = pytest.mark.gpu

K, N = 5, 4000


def _single():
    scn = W.dpd(n=N, dims=(16.0, 8.0, 8.0), seed=7)
    W.build_gpu(scn)
    start = m.universe.state()[3]
    m.universe.steps(K)
    x, v, f, c, xr = m.universe.state()
    m.universe.close()
    return start, c, xr, v


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slabs_match_the_undivided_box(tmp_path, world):
    from mechanica_b200 import slab
    start, c0, xr0, v0 = _single()
    out = str(tmp_path / "slab.npz")
    res = run_ranks(world, ["engine", out, K, N], timeout=600)
    assert all(rc == 0 for rc, _ in res), res
    z = np.load(out)
    assert len(z["ranges"]) == world
    assert np.array_equal(z["cell"], c0)
    assert np.array_equal(z["xr"].view(np.uint32), xr0.view(np.uint32))
    assert np.array_equal(z["v"].view(np.uint32), v0.view(np.uint32))
    if world > 1:
        # particles crossed slab faces in these steps: the migration path was taken
        own = slab.owner_of_layers(slab.slab_ranges(16, world), 16)
        assert (own[start // 64] != own[c0 // 64]).sum() > 0
