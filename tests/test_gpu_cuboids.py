"""Cuboids (static boxes particles are pushed from; potential_eval_cuboid_particle,
src/mdcore/src/cuboid_eval.hpp:73-188, from runner_doself) against the reference engine
compiled in place. The reference's cuboid constructor file is not compiled there, so the
test driver builds the cuboid as cuboid_init does (oracle/ref_driver.cpp) and adds it with
the reference's own engine_addcuboid; the quaternion arithmetic is that of the Magnum
stand-in the oracle is compiled against (Magnum itself is absent from the reference
checkout), so parity at that boundary is pinned to the stand-in.

Workload: 1,500 particles in a periodic box of 8 with a weak Morse pair term, one rotated
cuboid (size 2 x 1.5 x 1, angles 0.3, 0.5, 0.2) near the centre bound to the type with a
shifted Morse potential; some particles start inside it."""
import numpy as np
import pytest

import mechanica_b200 as m
from mechanica_b200 import workloads as W
from oracle import refengine

from golden_util import rel_rms

pytestmark = pytest.mark.gpu


def _scenario(seed=4):
    rng = np.random.default_rng(seed)
    L, n = 8.0, 1500
    x = rng.uniform(0, L, size=(n, 3)).astype(np.float32).astype(np.float64)
    return dict(dim=[L, L, L], cells=[8, 8, 8], cutoff=1.0, dt=0.002, bc=("periodic",) * 3,
                types=[(1.0, 0.1, m.Newtonian)], pots=[("morse", (0.2, 4.0, 0.2, 1e-4, 1.0, 1e-3), 0, 0)], forces=[],
                x=x, v=np.zeros_like(x), t=np.zeros(n, dtype=np.int32),
                cuboids=[((4.0, 4.1, 3.9), (2.0, 1.5, 1.0), (0.3, 0.5, 0.2))],
                cuboid_pots=[(0, "morse", (1.0, 6.0, 0.0, 1e-4, 3.0, 1e-3))])


@pytest.mark.skipif(not refengine.available(), reason="reference library not built")
def test_cuboid_forces_match_reference():
    scn = _scenario()
    u = W.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    ref = refengine.run(dict(scn, action="force", runners=2))
    assert np.array_equal(c, ref["cell"])
    assert rel_rms(f, ref["f"]) <= 1e-5
    # the cuboid acts on the particles it reaches, and only on them
    bare = dict(scn)
    bare.pop("cuboids")
    bare.pop("cuboid_pots")
    ref0 = refengine.run(dict(bare, action="force", runners=2))
    touched = np.abs(ref["f"] - ref0["f"]).sum(1) > 0
    assert touched.sum() > 20
    assert rel_rms(f[touched], ref["f"][touched]) <= 1e-5
    u.close()


@pytest.mark.skipif(not refengine.available(), reason="reference library not built")
def test_cuboid_steps_match_reference():
    scn = _scenario(seed=5)
    u = W.build_gpu(scn)
    for nsteps in (1, 2):
        u.steps(1)
        x, v, f, c, xr = u.state()
        ref = refengine.run(dict(scn, action="steps", nsteps=nsteps, runners=2))
        assert np.array_equal(c, ref["cell"])
        assert np.abs(x - ref["xabs"]).max() < 1e-5
        assert rel_rms(v, ref["v"]) <= 1e-5
    u.close()


def test_cuboid_geometry():
    """The cuboid's frame and bounding box: the orientation is a unit quaternion, and the
    box holds the eight rotated corners."""
    scn = _scenario()
    u = W.build_gpu(scn)
    pos, size, q, lo, hi = u.cuboid_info(0)
    assert abs(float((q.astype(np.float64) ** 2).sum()) - 1.0) < 1e-6
    x, y, z, w = q.astype(np.float64)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    corners = np.array([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]) * size / 2
    pts = corners @ R.T + pos
    assert np.allclose(pts.min(0), lo, atol=1e-5) and np.allclose(pts.max(0), hi, atol=1e-5)
    u.close()
