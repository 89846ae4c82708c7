"""Species fluxes (flux_eval_ex, src/mdcore/src/flux_eval.hpp:33-84; the state
update MxFluxes_Integrate, src/mdcore/src/Flux.cpp:261-285) against the
reference engine compiled in place, with its own Flux.cpp: Fick, secretion and
uptake fluxes and a constant species over a moving fluid. The species values
after one, two and ten steps agree with the reference's to FP32 summation
order, including the reference's rule that a particle which changed cells in
a step keeps its values and carries its rates into the next step."""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import load, rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsteps", [1, 2])
def test_species_after_steps_match_reference(nsteps):
    z, scn = load("species_fluxes")
    u = S.build_gpu(scn)
    u.steps(nsteps)
    sp = u.species_values()
    ref = z[f"step{nsteps}_species"]
    assert sp.shape == ref.shape
    err = np.abs(sp - ref).max()
    assert err <= 2e-6, err
    # the constant species does not move
    assert np.array_equal(sp[scn["t"] == 0, 2], scn["sp_values"][scn["t"] == 0, 2])
    changed = np.abs(sp - scn["sp_values"]).max(axis=1) > 0
    assert changed.mean() > 0.5


def test_species_trajectory_matches_reference():
    z, scn = load("species_fluxes")
    u = S.build_gpu(scn)
    u.steps(int(z["traj_nsteps"]))
    sp = u.species_values()
    assert rel_rms(sp, z["traj_species"]) <= 1e-5


def test_fick_flux_conserves_and_relaxes():
    """A pure Fick flux among static particles moves species between
    neighbours, conserving the total (up to FP32 rounding) and shrinking the
    spread; an untouched species keeps its values."""
    rng = np.random.default_rng(3)
    m.init(dim=[6.0, 6.0, 6.0], cells=[6, 6, 6], cutoff=1.0, dt=0.01)

    class A(m.Particle):
        mass = 1.0
        radius = 0.1
        frozen = 28
        species = ["S1", "S2"]

    assert A.species == ["S1", "S2"]
    A.factory(positions=rng.uniform(0, 6, size=(600, 3)))
    m.flux(A, A, "S1", 3.0)
    u = m.universe
    vals = np.zeros((600, 2), dtype=np.float32)
    vals[:, 0] = rng.uniform(0, 1, 600)
    vals[:, 1] = rng.uniform(0, 1, 600)
    u.set_species_values(vals)
    u.steps(50)
    sp = u.species_values()
    assert abs(sp[:, 0].sum() - vals[:, 0].sum()) <= 1e-4 * vals[:, 0].sum()
    assert sp[:, 0].std() < 0.9 * vals[:, 0].std()
    assert np.array_equal(sp[:, 1], vals[:, 1])


def test_particle_species_attribute():
    m.init(dim=[6.0, 6.0, 6.0], cells=[3, 3, 3], cutoff=1.0, dt=0.01)

    class A(m.Particle):
        mass = 1.0
        radius = 0.1
        species = ["S1", "$S2"]

    a1 = A(position=[3.0, 3.0, 3.0])
    a2 = A(position=[3.0, 3.5, 3.0])
    m.flux(A, A, "S1", 5.0)
    m.flux(A, A, "S2", 5.0)
    a1.species.S1 = 0.0
    a2.species.S1 = 1.0
    a1.species.S2 = 2.0
    m.universe.steps(1)
    # one pair at r = 0.5: q = 5 (s1 - s2) (1 - 0.5)^2, dt 0.01; S2 is constant
    assert a1.species.S1 == pytest.approx(0.0125, rel=1e-5)
    assert a2.species.S1 == pytest.approx(1.0 - 0.0125, rel=1e-5)
    assert a1.species.S2 == 2.0 and a2.species.S2 == 0.0
    with pytest.raises(ValueError):
        m.flux(A, A, "S9", 1.0)
