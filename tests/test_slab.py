"""Slab decomposition bookkeeping on the CPU (mechanica_b200.slab): the slab ranges, the
owners of the cell layers, which particles go to which neighbour as ghosts, and the record
exchange between gloo ranks (world sizes 2 and 3) -- every rank receives exactly the records
addressed to it, in source-rank order -- and the step's neighbour-only point-to-point exchange
(world sizes 2, 3 and 4)."""
import numpy as np
import pytest

from mechanica_b200 import slab
from slab_launch import run_ranks


def test_slab_ranges():
    assert slab.slab_ranges(16, 1) == [(0, 16)]
    assert slab.slab_ranges(16, 2) == [(0, 8), (8, 16)]
    assert slab.slab_ranges(16, 3) == [(0, 6), (6, 11), (11, 16)]
    assert slab.slab_ranges(4, 2) == [(0, 2), (2, 4)]
    for ncx in range(2, 40):
        for world in range(1, ncx // 2 + 1):
            r = slab.slab_ranges(ncx, world)
            assert r[0][0] == 0 and r[-1][1] == ncx
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            widths = [b - a for a, b in r]
            assert max(widths) - min(widths) <= 1 and (world == 1 or min(widths) >= 2)
    with pytest.raises(ValueError):
        slab.slab_ranges(5, 3)


def test_ghost_destinations_periodic():
    ranges = slab.slab_ranges(12, 3)  # (0,4) (4,8) (8,12)
    own = slab.owner_of_layers(ranges, 12)
    ncyz = 6
    cells = np.arange(12 * ncyz, dtype=np.int32)
    for rank, (x0, x1) in enumerate(ranges):
        mine = cells[(cells // ncyz >= x0) & (cells // ncyz < x1)]
        idx, dest = slab.ghost_records(mine, own, rank, ranges, ncyz, 12)
        lx = mine[idx] // ncyz
        # first layer to the rank below (periodic), last layer to the rank above
        assert set(lx[dest == (rank - 1) % 3]) == {x0}
        assert set(lx[dest == (rank + 1) % 3]) == {x1 - 1}
        assert len(idx) == 2 * ncyz


def test_one_slab_sends_no_ghosts():
    """With one rank the periodic neighbours of the slab are in its own engine: a ghost sent to
    itself would duplicate its boundary particles."""
    ranges = slab.slab_ranges(8, 1)
    own = slab.owner_of_layers(ranges, 8)
    idx, dest = slab.ghost_records(np.arange(8 * 4, dtype=np.int32), own, 0, ranges, 4, 8)
    assert len(idx) == 0 and len(dest) == 0


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo(tmp_path, world):
    out = str(tmp_path / "route")
    res = run_ranks(world, ["routing", out], timeout=180)
    assert all(rc == 0 for rc, _ in res), res
    for r in range(world):
        assert open(f"{out}.{r}").read() == "ok"


@pytest.mark.parametrize("world", [2, 3, 4])
def test_neighbour_exchange_over_gloo(tmp_path, world):
    """The slab step's exchange: point-to-point with the two neighbouring slabs only, counts then
    records; every rank receives exactly what its neighbours addressed to it."""
    out = str(tmp_path / "nb")
    res = run_ranks(world, ["neighbours", out], timeout=180)
    assert all(rc == 0 for rc, _ in res), res
    for r in range(world):
        assert open(f"{out}.{r}").read() == "ok"
