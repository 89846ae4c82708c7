"""Failure detection and degenerate inputs, with the faults made on the host
(no GPU fault is provoked): the engine's device status word reports a particle
that moved more than one cell in a step (the reference's engine_err_toofast,
engine_advance.cpp:171), raised as EngineError after the step. Many particles
entering one cell in a step are not a failure (the reference has no limit,
space_cell.cpp:260-290): beyond a cell's 32-entry movers bucket they go through
the step's overflow list, and the cells and positions match the reference
engine. Empty and single-particle universes step normally."""
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


def _crossing(counts):
    """counts[k] particles just left of the face x = 2 of cell (1, 2 + k, 2), moving +x."""
    pos = []
    for k, n in enumerate(counts):
        side = int(np.ceil(np.sqrt(n)))
        g = (np.arange(n) % side + 0.5) / side
        h = (np.arange(n) // side + 0.5) / side
        pos.append(np.stack([np.full(n, 1.995), 2.0 + k + g, 2.0 + h], axis=1))
    x = np.concatenate(pos)
    return x, np.tile([1.0, 0.0, 0.0], (len(x), 1))


@pytest.mark.parametrize("counts", [(40,), (100, 100)])
def test_many_particles_entering_one_cell(counts):
    """40 particles cross one cell face in a step, then 100 into each of two neighbouring
    cells (both beyond the bucket, so the overflow list holds movers of two cells): no
    error, every particle in the reference's cell at the reference's position, over three
    steps; the cells stay sorted by id."""
    from oracle import refengine
    if not refengine.available():
        pytest.skip("reference library not built")
    x, v = _crossing(counts)
    A = _box()
    A.factory(positions=x, velocities=v)
    u = m.universe
    scn = dict(dim=[6.0, 6.0, 6.0], cells=[6, 6, 6], cutoff=1.0, dt=0.01, bc=("periodic",) * 3,
               types=[(1.0, 0.1, m.Newtonian)], pots=[], forces=[], x=x, v=v, t=np.zeros(len(x), dtype=np.int32))
    for nsteps in (1, 2, 3):
        u.steps(1)
        xg, vg, fg, cg, xrg = u.state()
        ref = refengine.run(dict(scn, action="steps", nsteps=nsteps, runners=2))
        assert np.array_equal(cg, ref["cell"])
        assert np.abs(xg - ref["xabs"]).max() < 1e-5
    # slot order: ascending id inside every cell
    import torch
    st = u.device_state()
    ids = st["vel"][:, 3].contiguous().view(torch.int32).cpu().numpy()
    cells = st["cell"].cpu().numpy()
    assert np.array_equal(np.lexsort((ids, cells)), np.arange(len(x)))
