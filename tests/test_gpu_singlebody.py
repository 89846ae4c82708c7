"""The forces module's Berendsen, friction and random single-body forces
(MxForce.cpp:308-419) against the reference engine.

Berendsen and friction without noise are deterministic functions of the
velocities and are compared pair-force-pass to pair-force-pass; the random
force draws from the reference's global mt19937 there and from a Philox stream
here, so its magnitude distribution is compared statistically, including the
reference module's exchange of `std` and `mean`."""
import numpy as np
import pytest

import scenarios as S
from golden_util import rel_rms
from oracle import refengine

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not refengine.available(), reason="reference library not built")]


def _argon():
    return S.argon(n=2000, L=10.0, cells=10, seed=51, dt=0.002)


def _ke_sum(scn):
    v = np.asarray(scn["v"], dtype=np.float32).astype(np.float64)
    return float(0.5 * 39.4 * (v ** 2).sum())


def test_berendsen_force_matches_reference():
    scn = _argon()
    scn["sbforces"] = [(0, "berendsen", (0.5,))]
    scn["target_temperature"] = {0: 1.5 * _ke_sum(scn)}
    ref = refengine.run(dict(scn, action="force", runners=4))
    u = _build(scn)
    u.force()
    f = u.state()[2]
    assert rel_rms(f, ref["f"]) <= 1e-5


def test_friction_force_matches_reference():
    scn = _argon()
    scn["sbforces"] = [(0, "friction", (0.3, 0.0, 0.0, 0.002))]
    ref = refengine.run(dict(scn, action="force", runners=4))
    u = _build(scn)
    u.force()
    assert rel_rms(u.state()[2], ref["f"]) <= 1e-5
    ref1 = refengine.run(dict(scn, action="steps", nsteps=1, runners=4))
    u = _build(scn)
    u.steps(1)
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, ref1["cell"])
    assert rel_rms(v, ref1["v"]) <= 1e-5


def _free(n=20000, seed=52, dt=0.01):
    """Particles without pair forces (one type, no potential): the force on each
    is its single-body force alone."""
    rng = np.random.default_rng(seed)
    L = 20.0
    x = rng.uniform(0, L, size=(n, 3)).astype(np.float32).astype(np.float64)
    import mechanica_b200 as m
    return dict(dim=[L, L, L], cells=[10, 10, 10], cutoff=1.0, dt=dt, bc=("periodic",) * 3,
                types=[(1.0, 0.5, m.Newtonian)], pots=[], forces=[], x=x, v=np.zeros((n, 3), np.float32),
                t=np.zeros(n, dtype=np.int32))


def test_random_force_statistics_match_reference():
    """forces.random(std=2, mean=0.3): in the reference the magnitude is drawn
    with mean 2 and standard deviation 0.3 (the module exchanges the two); the
    direction is uniform, and a force persists until its particle's next redraw."""
    scn = _free()
    scn["sbforces"] = [(0, "random", (2.0, 0.3, 0.01))]  # durration = dt: every step
    ref = refengine.run(dict(scn, action="steps", nsteps=1, runners=4))
    u = _build(scn)
    u.steps(1)
    f = u.state()[2].astype(np.float64)
    for ff in (f, ref["f"].astype(np.float64)):
        mag = np.linalg.norm(ff, axis=1)
        assert abs(mag.mean() - 2.0) < 0.01 and abs(mag.std() - 0.3) < 0.01, (mag.mean(), mag.std())
        assert np.abs(ff.mean(axis=0)).max() < 0.05  # isotropic
    # a force is redrawn when (time + id) is a multiple of ceil(durration / dt), the
    # interval computed as the reference does it (float duration, double dt:
    # ceil(float(0.04) / 0.01) = 4, while ceil(float(0.05) / 0.01) = 6)
    scn = _free(n=2000, seed=53)
    scn["sbforces"] = [(0, "random", (1.0, 0.1, 0.04))]
    every = int(np.ceil(float(np.float32(0.04)) / scn["dt"]))
    assert every == 4
    u = _build(scn)
    fs = []
    for _ in range(6):
        u.steps(1)
        fs.append(u.state()[2].copy())
    ids = np.arange(2000)
    for t in range(1, 6):  # step t+1 runs at time t+1
        same = np.all(fs[t] == fs[t - 1], axis=1)
        redrawn = (t + 1 + ids) % every == 0
        assert np.array_equal(~same, redrawn)


def _build(scn):
    import mechanica_b200 as m
    u = S.build_gpu(scn)
    types = list(m.universe._types)
    for (t, kind, params) in scn.get("sbforces", []):
        f = {"berendsen": m.forces.berenderson_tstat, "random": m.forces.random, "friction": m.forces.friction}[kind]
        u.bind(f(*params), t)
    for t, temp in scn.get("target_temperature", {}).items():
        u._targets[t] = temp
        u._dirty = True
    return u
