"""engine_load / engine_unload on the device (mxg_engine_load, mxg_engine_unload): the
placement of global positions by id into cells (space_addpart's arithmetic and the
first shuffle, space.cpp:431-451 and 352-371) gives the same cells, the same FP32
cell-relative positions and the same slot order as the host placement of a freshly
built engine; unload returns global positions cell origin + x_rel in double."""
import numpy as np
import pytest
import torch

import scenarios as S
from golden_util import load
from mechanica_b200._native import EngineError, lib

pytestmark = pytest.mark.gpu


def _slots(u):
    st = u.device_state()
    return (st["pos"].cpu().numpy().view(np.uint32).copy(), st["vel"].cpu().numpy().view(np.uint32).copy(),
            st["cell"].cpu().numpy().copy())


@pytest.mark.parametrize("name", ["argon_small", "dpd_small", "morse2_small"])
def test_device_load_matches_host_placement(name):
    z, scn = load(name)
    u = S.build_gpu(scn)
    u.steps(4)
    x, v, f, c, xr = u.state()
    # the same positions loaded into the running engine: the device placement
    u.load(x, v)
    xl, vl, fl, cl, xrl = u.state()
    pl, wl, cellsl = _slots(u)
    u.steps(2)
    after_load = u.state()[4].copy()
    # an engine built from those positions: the host placement at engine start
    u = S.build_gpu(dict(scn, x=x, v=v))
    x2, v2, f2, c2, xr2 = u.state()
    p2, w2, cells2 = _slots(u)
    # the same step counter (it keys the random direction of pairs closer than a table minimum)
    assert lib().mxg_engine_set_step_counter(u._e, 4) == 0
    u.steps(2)
    after_host = u.state()[4].copy()
    u.close()
    assert np.array_equal(cl, c2)
    assert np.array_equal(xrl.view(np.uint32), xr2.view(np.uint32))
    assert np.array_equal(xl, x2) and np.array_equal(vl, v2)
    assert np.array_equal(pl, p2) and np.array_equal(wl, w2) and np.array_equal(cellsl, cells2)
    # the next steps agree bit for bit
    assert np.array_equal(after_load.view(np.uint32), after_host.view(np.uint32))


def test_device_load_matches_host_placement_on_a_large_grid():
    """16,000 cells (two tiles of the device scan of the occupancy), a few of them empty,
    velocities given (their copy overlaps the placement)."""
    from mechanica_b200 import workloads as W
    scn = W.dpd(n=60000, dims=(40.0, 20.0, 20.0), seed=4)
    u = W.build_gpu(scn)
    u.steps(3)
    x, v, f, c, xr = u.state()
    assert np.bincount(np.asarray(c), minlength=16000).min() == 0
    u.load(x, v)
    xl, vl, fl, cl, xrl = u.state()
    pl, wl, cellsl = _slots(u)
    u.close()
    u = W.build_gpu(dict(scn, x=x, v=v))
    x2, v2, f2, c2, xr2 = u.state()
    p2, w2, cells2 = _slots(u)
    u.close()
    assert np.array_equal(cl, c2)
    assert np.array_equal(xrl.view(np.uint32), xr2.view(np.uint32))
    assert np.array_equal(xl, x2) and np.array_equal(vl, v2)
    assert np.array_equal(pl, p2) and np.array_equal(wl, w2) and np.array_equal(cellsl, cells2)


def test_load_keeps_velocities_and_rejects_outside_positions():
    z, scn = load("argon_small")
    u = S.build_gpu(scn)
    u.steps(2)
    x, v, f, c, xr = u.state()
    L = np.asarray(scn["dim"])
    u.load(np.mod(x + 0.01, L))  # velocities kept
    x4, v4, _, _, _ = u.state()
    assert np.array_equal(v4, v)
    bad = x.copy()
    bad[3] = [-5.0, 1.0, 1.0]
    with pytest.raises(EngineError) as exc:
        u.load(bad)
    assert exc.value.code == -3  # the state is left as it was
    x5, v5, _, c5, xr5 = u.state()
    assert np.array_equal(x5, x4) and np.array_equal(v5, v4)
    u.close()
