"""Runge-Kutta 4 (engine_advance_runge_kutta_4, engine_advance.cpp:443-698)
against the reference engine, and its accuracy against forward Euler.

The reference re-bins particles between the four stages but keeps the stage
origin p0 in the old cell's frame, so a particle that crosses a cell face
mid-step lands a cell edge away there; this engine keeps the step's cell frame.
The parity scenarios therefore keep every particle at least `margin` from its
cell's faces, more than any stage moves it, so the two agree; particles may
still cross a face at the end of the step, where both re-bin the same way."""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import rel_rms
from oracle import refengine

pytestmark = pytest.mark.gpu


def _margin(scn, margin):
    x = scn["x"].copy()
    h = np.asarray(scn["dim"]) / np.asarray(scn["cells"])
    base = np.floor(x / h) * h
    scn["x"] = (base + np.clip(x - base, margin, h - margin)).astype(np.float32).astype(np.float64)
    scn["integrator"] = m.RUNGE_KUTTA_4
    return scn


def _argon():
    return _margin(S.argon(n=2000, L=10.0, cells=10, seed=41, dt=0.002), 0.02)


def _morse_lattice(n_side=12, density=0.6, seed=42, dt=0.002, dynamics=m.Overdamped):
    """Two-type Morse mixture (d 0.5 / 0.3 / 0.7, a = 5, r0 = 1, cutoff 2.5) on a
    jittered simple-cubic lattice: nearest neighbours near the Morse minimum, so
    forces stay moderate (a random start would put pairs deep in the repulsive
    wall; the reference's RK4 has no displacement clamp and stops with a
    too-fast error there)."""
    rng = np.random.default_rng(seed)
    n = n_side ** 3
    L = (n / density) ** (1.0 / 3.0)
    sp = L / n_side
    g = (np.arange(n_side) + 0.5) * sp
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = np.mod(x + rng.uniform(-0.1, 0.1, size=x.shape) * sp, L)
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    t = (np.arange(n) % 2).astype(np.int32)
    v = (rng.normal(0, 0.3, size=(n, 3)) if dynamics == m.Newtonian else np.zeros((n, 3))).astype(np.float32)
    cut = 2.5
    pots = [("morse", (dd, 5.0, 1.0, 1e-4, cut, 1e-3), a, b) for (dd, a, b) in ((0.5, 0, 0), (0.3, 0, 1), (0.7, 1, 1))]
    return dict(dim=[L, L, L], cells=[int(L // cut)] * 3, cutoff=cut, dt=dt, bc=("periodic",) * 3,
                types=[(1.0, 1.0, dynamics), (1.0, 1.0, dynamics)], pots=pots, forces=[], x=x, v=v, t=t)


def _morse_overdamped():
    return _margin(_morse_lattice(), 0.02)


@pytest.mark.skipif(not refengine.available(), reason="reference library not built")
@pytest.mark.parametrize("build", [_argon, _morse_overdamped], ids=["lj_newtonian", "morse_overdamped"])
def test_rk4_step_matches_reference(build):
    scn = build()
    ref = refengine.run(dict(scn, action="steps", nsteps=1, runners=4))
    u = S.build_gpu(scn)
    u.steps(1)
    assert m.universe.integrator == m.RUNGE_KUTTA_4
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, ref["cell"])
    L = np.asarray(scn["dim"])
    d = x - ref["xabs"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5
    if scn["types"][0][2] == m.Newtonian:
        assert rel_rms(v, ref["v"]) <= 1e-5


def test_rk4_is_fourth_order_where_euler_is_first():
    """Newtonian Morse mixture over 0.2 time units: the final positions with
    dt = 0.01 against a run with dt = 0.00125; the RK4 error is a small fraction
    of forward Euler's."""
    def final(integ, dt, nsteps):
        scn = _morse_lattice(dt=dt, dynamics=m.Newtonian)
        scn["integrator"] = integ
        u = S.build_gpu(scn)
        u.steps(nsteps)
        return u.state()[0], np.asarray(scn["dim"])

    exact, L = final(m.RUNGE_KUTTA_4, 0.00125, 160)
    err = {}
    for integ in (m.FORWARD_EULER, m.RUNGE_KUTTA_4):
        x, _ = final(integ, 0.01, 20)
        d = x - exact
        d -= L * np.round(d / L)
        err[integ] = np.sqrt((d ** 2).sum(1).mean())
    assert err[m.RUNGE_KUTTA_4] < 0.05 * err[m.FORWARD_EULER], err
