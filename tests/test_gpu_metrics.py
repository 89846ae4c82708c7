"""Particle-group metrics on the device (ParticleList.center_of_mass / centroid /
radius_of_gyration / moment_of_inertia; MxParticleList.cpp:406-458 over
metrics.cpp:330-466) against the oracle's restatement of the reference's formulas,
on the global positions of a stepped LJ fluid: FP64 sums within 1e-10 of the FP64
restatement, and within the reference's own FP32 running-sum error (1e-5) of the
FP32 restatement."""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import load
from oracle import restatement as R

pytestmark = pytest.mark.gpu


def _masses(scn, ids):
    mt = np.array([t[0] for t in scn["types"]], dtype=np.float64)
    return mt[np.asarray(scn["t"])[ids]]


def _check(pl, x, mass):
    got = (pl.center_of_mass(), pl.centroid(), pl.radius_of_gyration(), pl.moment_of_inertia())
    M, com, cen, rog, I = R.group_metrics(x, mass)
    assert np.abs(got[0] - com).max() <= 1e-10 * np.abs(com).max()
    assert np.abs(got[1] - cen).max() <= 1e-10 * np.abs(cen).max()
    assert abs(got[2] - rog) <= 1e-10 * rog
    assert np.abs(got[3] - I).max() <= 1e-10 * np.abs(I).max()
    M32, com32, cen32, rog32, I32 = R.group_metrics(x, mass, fp32=True)
    assert np.abs(got[0] - com32).max() <= 1e-5 * np.abs(com).max()
    assert abs(got[2] - rog32) <= 1e-5 * rog
    assert np.abs(got[3] - I32).max() <= 1e-5 * np.abs(I).max()


def test_group_metrics_match_restatement():
    z, scn = load("morse2_small")
    u = S.build_gpu(scn)
    u.steps(5)
    x = u.state()[0]
    rng = np.random.default_rng(12)
    ids = rng.choice(len(x), size=300, replace=False).astype(np.int32)
    _check(m.ParticleList(ids), x[ids], _masses(scn, ids))


def test_type_items_are_a_particle_list():
    m.init(dim=[8.0, 8.0, 8.0], cells=[4, 4, 4], cutoff=2.0, dt=0.01)

    class A(m.Particle):
        mass = 2.0
        radius = 0.2

    class B(m.Particle):
        mass = 5.0
        radius = 0.2

    rng = np.random.default_rng(5)
    A.factory(positions=rng.uniform(0, 8, size=(200, 3)))
    B.factory(positions=rng.uniform(0, 8, size=(100, 3)))
    pl = B.items()
    assert isinstance(pl, m.ParticleList) and len(pl) == 100
    assert np.array_equal(np.asarray(pl), np.arange(200, 300, dtype=np.int32))
    x = m.universe.state()[0]
    _check(pl, x[200:300], np.full(100, 5.0))
    with pytest.raises(ValueError):
        m.ParticleList([]).center_of_mass()
    with pytest.raises(m.EngineError):
        m.ParticleList([0, 300]).centroid()
