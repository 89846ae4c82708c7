"""Space set-up: cell grid and the cell-pair task list (type, sort ID, cells
after the flip), integer bit-exact against the reference's space_init."""
import os

import numpy as np
import pytest

import mechanica_b200 as m
from oracle import refengine

import scenarios as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["argon_small", "argon_default_cells", "dpd_small", "lattice_small", "morse2_small"]


def _load(name):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import load_scenario
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, load_scenario(z)


def _init_only(scn):
    bc = {"x": scn["bc"][0], "y": scn["bc"][1], "z": scn["bc"][2]}
    m.init(dim=scn["dim"], cells=scn["cells"], cutoff=scn["cutoff"], dt=scn["dt"], bc=bc)
    return m.universe


@pytest.mark.parametrize("name", CASES)
def test_task_list_matches_golden(name):
    z, scn = _load(name)
    u = _init_only(scn)
    cdim, h, nc, per = u.space_info()
    assert np.array_equal(cdim, z["force_cdim"])
    assert np.array_equal(h, z["force_h"])
    ref = z["force_tasks"]
    ref = ref[(ref[:, 0] == 1) | (ref[:, 0] == 2)]  # the reference also lists one sort task per cell
    assert np.array_equal(u.tasks(), ref)


GEOMS = [
    # dim, cells, cutoff, bc
    ((10.0, 10.0, 10.0), (4, 4, 4), 1.0, ("periodic", "periodic", "periodic")),
    ((10.0, 10.0, 10.0), (10, 10, 10), 1.0, ("periodic", "periodic", "periodic")),
    ((7.3, 5.1, 9.9), (7, 5, 9), 1.0, ("periodic", "free_slip", "no_slip")),
    ((16.0, 16.0, 18.0), (10, 10, 12), 1.5, ("free_slip", "free_slip", "free_slip")),
    ((12.0, 12.0, 12.0), (6, 6, 6), 2.5, ("periodic", "periodic", "periodic")),   # span 2
    ((5.0, 5.0, 5.0), (2, 2, 2), 1.0, ("periodic", "periodic", "periodic")),      # raised to 3 cells
    ((40.0, 20.0, 20.0), (40, 20, 20), 1.0, ("periodic", "periodic", "no_slip")),
]


@pytest.mark.skipif(not refengine.available(), reason="reference not built here")
@pytest.mark.parametrize("geom", GEOMS)
def test_task_list_live(geom):
    dim, cells, cutoff, bc = geom
    scn = dict(dim=list(dim), cells=list(cells), cutoff=cutoff, dt=0.01, bc=bc, types=[(1.0, 0.1, 0)], pots=[],
               forces=[], x=np.array([[0.5, 0.5, 0.5]]), v=np.zeros((1, 3)), t=np.zeros(1, dtype=np.int32))
    ref = refengine.run(dict(scn, action="force", runners=1))
    u = _init_only(scn)
    cdim, h, nc, per = u.space_info()
    assert np.array_equal(cdim, ref["cdim"])
    assert np.array_equal(h, ref["h"])
    assert per == int(ref["period"]) & 7
    rt = ref["tasks"]
    assert np.array_equal(u.tasks(), rt[(rt[:, 0] == 1) | (rt[:, 0] == 2)])
