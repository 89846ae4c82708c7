"""Wall potentials (boundary_eval, src/mdcore/src/boundary_eval.hpp:124-223)
against the reference engine compiled in place (golden fixtures from
tests/golden/make_golden.py): LJ and Morse walls bound per face and type on
"potential" z faces, and DPD walls on no-slip faces bound to every face.
Bars as for the other force passes: cells and cell-relative positions exact,
forces within 1e-5 relative RMS, energy within 1e-5, one and two steps within
1e-5 in position."""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import load, rel_rms

pytestmark = pytest.mark.gpu

CASES = ["walls_lj", "walls_dpd"]


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", CASES)
def test_wall_force_pass_matches_reference(name):
    z, scn = load(name)
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["force_cell"])
    assert np.array_equal(_bits(xr), _bits(z["force_xrel"]))
    assert rel_rms(f, z["force_f"]) <= 1e-5
    ep, _ = u.energies()
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-5 * abs(ref) + 1e-9


@pytest.mark.parametrize("nsteps", [1, 2])
@pytest.mark.parametrize("name", CASES)
def test_wall_steps_match_reference(name, nsteps):
    z, scn = load(name)
    u = S.build_gpu(scn)
    u.steps(nsteps)
    x, v, f, c, xr = u.state()
    k = f"step{nsteps}_"
    assert (c == z[k + "cell"]).mean() >= 0.999
    L = np.asarray(scn["dim"])
    d = x - z[k + "xabs"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5
    assert rel_rms(v, z[k + "v"]) <= 1e-5


def test_walls_push_particles_away():
    """Without the wall potentials the same fluid has no wall forces: the
    difference of the two force passes acts only within the potentials' range
    of a bound face, along the face normal."""
    z, scn = load("walls_lj")
    u = S.build_gpu(scn)
    u.force()
    f_w = u.state()[2].astype(np.float64)
    scn2 = dict(scn)
    scn2["wall_pots"] = []
    u2 = S.build_gpu(scn2)
    u2.force()
    x, _, f0, _, _ = u2.state()
    d = f_w - f0.astype(np.float64)
    moved = np.abs(d).max(axis=1) > 1e-4 * np.abs(f_w).max()
    zpos = x[:, 2]
    L = scn["dim"][2]
    assert moved.any()
    assert np.all((zpos[moved] <= 1.0 + 1e-6) | (zpos[moved] >= L - 1.0 - 1e-6))
    assert np.abs(d[moved][:, :2]).max() <= 1e-4 * np.abs(d[moved][:, 2]).max()
    bottom = moved & (zpos < L / 2) & (scn["t"] == 0)
    assert np.all(d[bottom, 2] > 0)  # the r^-12 wall pushes +z at the bottom face
