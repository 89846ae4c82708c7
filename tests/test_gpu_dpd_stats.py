"""The DPD random term in Philox mode, checked statistically (the random
streams of a reference implementation and of this one cannot agree draw by
draw; the reference's own term has no random number, dpd_eval.hpp:57).

1. Kinetic temperature of a DPD fluid (a=25, gamma=4.5, sigma=3, so
   kT = sigma^2 / (2 gamma) = 1) within 1 % of kT. A random start releases
   the overlap energy of the conservative force as heat (T reaches ~1.7),
   which the thermostat removes over ~3 time units; the test equilibrates for
   6 and averages over the next 8. At dt = 0.002 the forward-Euler bias of the
   thermostat is ~0.2 %.
2. Momentum: the pair forces are exact negations, so the total momentum
   stays at its initial value up to FP32 rounding of the sums.
3. Velocity autocorrelation: the same initial state and the same Philox
   stream (keyed on the step and the particle ids) run by the FP64
   restatement of the model; the two autocorrelation curves agree.
"""
import numpy as np
import pytest

import mechanica_b200 as m
from mechanica_b200 import workloads as W
from oracle import adjoint_ref as R

pytestmark = pytest.mark.gpu


def _dpd_fluid(n, L, seed, dt):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, L, size=(n, 3))
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    v = rng.normal(0, 1.0, size=(n, 3))
    v -= v.mean(axis=0)
    cells = int(L // 1.0)
    return dict(dim=[L, L, L], cells=[cells] * 3, cutoff=1.0, dt=dt, bc=("periodic",) * 3,
                types=[(1.0, 0.5, m.Newtonian)], pots=[("dpd", (25.0, 4.5, 3.0, 1.0), 0, 0)], forces=[],
                x=x, v=v.astype(np.float32), t=np.zeros(n, dtype=np.int32))


def _temperature(v):
    v = v.astype(np.float64)
    return (v ** 2).sum() / (3 * (len(v) - 1))


def test_philox_dpd_temperature_and_momentum():
    scn = _dpd_fluid(n=24000, L=20.0, seed=31, dt=0.002)
    u = W.build_gpu(scn, rng_mode="philox")
    u.steps(1)
    p0 = u.state()[1].astype(np.float64).sum(0)
    u.steps(3000)  # 6 time units
    temps = []
    for _ in range(100):
        u.steps(40)
        v = u.state()[1]
        temps.append(_temperature(v))
    T = float(np.mean(temps))
    assert abs(T - 1.0) <= 0.01, T
    p = u.state()[1].astype(np.float64).sum(0)
    assert np.abs(p - p0).max() <= 1e-3 * np.sqrt(len(v)), (p, p0)


def test_philox_dpd_velocity_autocorrelation_matches_fp64():
    n, L, dt, nsteps = 1500, 7.9, 0.002, 150
    scn = _dpd_fluid(n=n, L=L, seed=32, dt=dt)
    u = W.build_gpu(scn, rng_mode="philox")
    vs = [u.state()[1].astype(np.float64)]
    for _ in range(nsteps // 10):
        u.steps(10)
        vs.append(u.state()[1].astype(np.float64))
    vg = np.array(vs)
    box = np.asarray(scn["dim"])
    h = box[0] / scn["cells"][0]
    maxv = float(np.float32(np.float32(h) * np.float32(0.05)) / np.float32(dt))
    delta = float(np.float32(1.0 / np.sqrt(dt)))
    terms = {(0, 0): [R.Dpd(25.0, 4.5, 3.0, 1.0, delta)]}
    vr = R.run_velocities(scn["x"], scn["v"].astype(np.float64), scn["t"], np.arange(n), box, np.array([1.0]),
                          np.array([0.5]), terms, 1.0, dt, nsteps, 0, maxv, every=10)
    cg = (vg * vg[0]).sum(axis=(1, 2)) / (vg[0] ** 2).sum()
    cr = (vr * vr[0]).sum(axis=(1, 2)) / (vr[0] ** 2).sum()
    assert cg[0] == 1.0 and cr[0] == 1.0
    assert np.all(np.diff(cr[:6]) < 0)  # the correlation decays
    assert np.abs(cg - cr).max() <= 2e-3, (cg, cr)
