"""Large particles (radius > cutoff: the reference's PARTICLE_LARGE,
MxParticle.cpp:2091-2093) against the reference engine compiled in place:
they stay put, take no part in the cell-pair loop, and every other particle
interacts with them through the potential of the type pair
(particle_largecell_force, runner_dopair.cpp:342-434). The small particles'
forces, energies and one and two steps are compared; the large particles'
cells are not (the reference keeps them in a separate cell)."""
import numpy as np
import pytest

import scenarios as S
from golden_util import load, rel_rms

pytestmark = pytest.mark.gpu


def test_large_particle_force_pass_matches_reference():
    z, scn = load("large_fluid")
    small = scn["t"] == 0
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert np.array_equal(c[small], z["force_cell"][small])
    assert rel_rms(f[small], z["force_f"][small]) <= 1e-5



def test_large_particle_energy_is_the_sum_of_pair_energies():
    """The reference's energy for these pairs is undefined: particle_largecell_force
    adds a running sum through a local that is never initialised
    (runner_dopair.cpp:343,425-427). Here each (small, large) pair's table energy
    counts once: the energy with the large-particle potential minus the energy
    without it equals the sum over pairs of potential_eval_ex on the host table."""
    import ctypes
    import mechanica_b200 as m
    from mechanica_b200._native import lib
    z, scn = load("large_fluid")
    u = S.build_gpu(scn)
    u.force()
    ep_with, _ = u.energies()
    x = u.state()[0]
    scn2 = dict(scn)
    scn2["pots"] = [p for p in scn["pots"] if not (p[2] == 0 and p[3] == 1)]
    u2 = S.build_gpu(scn2)
    u2.force()
    ep_without, _ = u2.energies()
    kind, params, _, _ = [p for p in scn["pots"] if p[2] == 0 and p[3] == 1][0]
    pot = S.make_potential(kind, params)
    r_small, r_large = scn["types"][0][1], scn["types"][1][1]
    xs = x[scn["t"] == 0].astype(np.float32)
    total = 0.0
    for xl in scn["x"][scn["t"] == 1].astype(np.float32):
        d = xs - xl
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        for q in r2:
            e, f = ctypes.c_float(), ctypes.c_float()
            if lib().mxg_potential_eval(pot._h, r_small, r_large, float(q), ctypes.byref(e), ctypes.byref(f)):
                total += e.value
    assert total < 0
    assert abs((ep_with - ep_without) - total) <= 1e-5 * abs(total)


@pytest.mark.parametrize("nsteps", [1, 2])
def test_large_particles_stay_and_small_ones_step_like_reference(nsteps):
    z, scn = load("large_fluid")
    small = scn["t"] == 0
    u = S.build_gpu(scn)
    u.steps(nsteps)
    x, v, f, c, xr = u.state()
    k = f"step{nsteps}_"
    L = np.asarray(scn["dim"])
    d = x - z[k + "xabs"]
    d -= L * np.round(d / L)
    assert np.abs(d[small]).max() < 1e-5
    assert rel_rms(v[small], z[k + "v"][small]) <= 1e-5
    assert np.abs(x[~small] - scn["x"][~small]).max() < 1e-6
    assert np.array_equal(z[k + "xabs"][~small], scn["x"][~small])
