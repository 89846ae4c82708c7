"""Failure detection and degenerate inputs, with the faults made on the host
(no GPU fault is provoked): the engine's device status word reports a particle
that moved more than one cell in a step (the reference's engine_err_toofast,
engine_advance.cpp:171) and more particles entering one cell in a step than its
movers bucket holds; both are raised as EngineError after the step. Empty and
single-particle universes step normally."""
import numpy as np
import pytest

import mechanica_b200 as m
from mechanica_b200._native import EngineError

pytestmark = pytest.mark.gpu


def _box(**kw):
    m.init(dim=[6.0, 6.0, 6.0], cells=[6, 6, 6], cutoff=1.0, dt=0.01, **kw)

    class A(m.Particle):
        mass = 1.0
        radius = 0.1

    return A


def test_empty_universe_steps():
    _box()
    u = m.universe
    u.steps(3)
    u.force()
    ep, ek = u.energies()
    assert ep == 0.0 and ek == 0.0


def test_single_particle_crosses_cells():
    A = _box()
    A.factory(positions=np.array([[0.95, 2.5, 2.5]]), velocities=np.array([[2.0, 0.0, 0.0]]))
    u = m.universe
    u.steps(20)
    x, v, f, c, xr = u.state()
    # 20 steps of dt 0.01 at speed 2 (below the clamp h frac / dt = 5): x = 0.95 + 0.4
    assert abs(x[0, 0] - 1.35) < 1e-5
    assert np.all(v[0] == np.float32([2.0, 0.0, 0.0]))
    assert 0.0 <= xr[0, 0] < 1.0


def test_too_fast_particle_is_reported():
    """Runge-Kutta 4 has no speed clamp (as in the reference), so a particle at
    speed 300 moves three cells in one step of dt 0.01."""
    A = _box(integrator=m.RUNGE_KUTTA_4)
    A.factory(positions=np.array([[2.5, 2.5, 2.5]]), velocities=np.array([[300.0, 0.0, 0.0]]))
    with pytest.raises(EngineError) as exc:
        m.universe.steps(1)
    assert exc.value.code == -29  # engine_err_toofast


def test_cell_bucket_overflow_is_reported():
    """40 particles cross the same cell face in one step; a cell takes at most
    32 newcomers per step."""
    A = _box()
    g = (np.arange(40) % 8 + 0.5) / 8.0
    h = (np.arange(40) // 8 + 0.5) / 5.0
    pos = np.stack([np.full(40, 1.995), 2.0 + g, 2.0 + h], axis=1)
    A.factory(positions=pos, velocities=np.tile([1.0, 0.0, 0.0], (40, 1)))
    with pytest.raises(EngineError) as exc:
        m.universe.steps(1)
    assert exc.value.code == -101
