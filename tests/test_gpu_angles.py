"""Angle forces (angle_eval, src/mdcore/src/angle.cpp:92-352) in the bonded pass,
against the reference engine compiled in place (golden fixtures from
tests/golden/make_golden.py).

chains_bonded has bonds and angles and no pair potential: every particle's
force is the same sequence of FP32 updates as in the reference's serial
bonded loops, so forces and trajectories are compared bit for bit.
chains_morse adds a Morse pair potential: forces within the 1e-5 relative
RMS bar, energies within 1e-6.
"""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import load, rel_rms

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_bonded_force_pass_is_bit_exact():
    z, scn = load("chains_bonded")
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["force_cell"])
    assert np.array_equal(_bits(f), _bits(z["force_f"]))
    ep, _ = u.energies()
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-12 * abs(ref)


def test_bonded_trajectory_is_bit_exact():
    """Ten forward-Euler steps with bonds and angles across periodic faces."""
    z, scn = load("chains_bonded")
    u = S.build_gpu(scn)
    u.steps(int(z["traj_nsteps"]))
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["traj_cell"])
    assert np.array_equal(_bits(xr), _bits(z["traj_xrel"]))
    assert np.array_equal(_bits(v), _bits(z["traj_v"]))


def test_angles_with_pair_potential():
    z, scn = load("chains_morse")
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["force_cell"])
    assert rel_rms(f, z["force_f"]) <= 1e-5
    ep, _ = u.energies()
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-6 * abs(ref)
    u.steps(int(z["traj_nsteps"]))
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["traj_cell"])
    L = np.asarray(scn["dim"])
    d = x - z["traj_xabs"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5
    assert rel_rms(v, z["traj_v"]) <= 1e-5


def _eval_r(p, r):
    """potential_eval_r (potential_eval.hpp:180-207) in FP32 on the table."""
    info = p._info()
    c = p.coefficients.reshape(-1, 8)
    a = info["alpha"]
    f32 = np.float32
    r = f32(r)
    ind = min(int(max(f32(0), a[0] + r * (a[1] + r * a[2]))), info["n"])
    q = c[ind]
    x = (r - q[0]) * q[1]
    ee = q[2] * x + q[3]
    eff = q[2]
    for k in range(4, 8):
        eff = eff * x + ee
        ee = ee * x + q[k]
    return float(ee), float(eff * q[1])


@pytest.mark.parametrize("geometry", ["right", "straight"])
def test_degenerate_angle_uses_one_random_direction(geometry):
    """At cos(theta) = 0 or -1 the reference puts both outer particles' force
    along one random unit vector (angle.cpp:184-196): f_i = f_k = -eff * u,
    f_j = -(f_i + f_k), |f_i| = |eff|."""
    pot = m.Potential.harmonic_angle(k=3.0, theta0=2.2)
    m.init(dim=[6.0, 6.0, 6.0], cells=[3, 3, 3], cutoff=2.0, dt=0.001)

    class Bead(m.Particle):
        mass = 1.0
        radius = 0.1

    # exactly representable offsets, so the cosine is exactly 0 or -1
    xj = np.array([3.0, 3.0, 3.0])
    xi = xj + [-0.5, 0.0, 0.0]
    xk = xj + ([0.0, 0.5, 0.0] if geometry == "right" else [0.5, 0.0, 0.0])
    u = m.universe
    u._add_particles(np.stack([xi, xj, xk]), np.zeros((3, 3), dtype=np.float32), np.zeros(3, dtype=np.int32))
    m.Angle(pot, 0, 1, 2)
    u.force()
    f = u.state()[2].astype(np.float64)
    ct = 0.0 if geometry == "right" else -1.0
    ee, eff = _eval_r(pot, max(ct, pot.min))
    assert np.array_equal(f[0], f[2])
    assert np.allclose(f[1], -(f[0] + f[2]), rtol=0, atol=1e-6 * abs(eff))
    assert abs(np.linalg.norm(f[0]) - abs(eff)) <= 1e-5 * abs(eff)
    ep, _ = u.energies()
    assert abs(ep - ee) <= 1e-6 * abs(ee)


def test_angle_energy_matches_analytic():
    """A single angle away from the degenerate points: the table energy and the
    force along the bisector plane against k (theta - theta0)^2 in FP64."""
    k, th0 = 4.0, 1.9
    pot = m.Potential.harmonic_angle(k=k, theta0=th0)
    m.init(dim=[6.0, 6.0, 6.0], cells=[3, 3, 3], cutoff=2.0, dt=0.001)

    class Bead(m.Particle):
        mass = 1.0
        radius = 0.1

    th = 2.4
    xj = np.array([2.9, 3.05, 3.1])
    xi = xj + 0.6 * np.array([1.0, 0.0, 0.0])
    xk = xj + 0.5 * np.array([np.cos(th), np.sin(th), 0.0])
    u = m.universe
    u._add_particles(np.stack([xi, xj, xk]), np.zeros((3, 3), dtype=np.float32), np.zeros(3, dtype=np.int32))
    m.Angle(pot, 0, 1, 2)
    u.force()
    f = u.state()[2].astype(np.float64)
    x = u.state()[0]
    rji, rjk = x[0] - x[1], x[2] - x[1]
    c = rji @ rjk / np.linalg.norm(rji) / np.linalg.norm(rjk)
    theta = np.arccos(c)
    ep, _ = u.energies()
    assert abs(ep - k * (theta - th0) ** 2) <= 2e-3 * k * (theta - th0) ** 2
    # the force on i is -dV/dx_i = 2k (theta - theta0) dtheta/dx_i
    dth = -(rjk / np.linalg.norm(rjk) - c * rji / np.linalg.norm(rji)) / np.linalg.norm(rji) / np.sqrt(1 - c * c)
    fi = -2 * k * (theta - th0) * dth
    assert np.linalg.norm(f[0] - fi) <= 5e-3 * np.linalg.norm(fi)
    assert np.abs(f.sum(axis=0)).max() <= 1e-5 * np.abs(f).max()


# ---- dihedrals (dihedral_eval, src/mdcore/src/dihedral.cpp:81-392) ----

def test_dihedral_force_pass_and_trajectory_are_bit_exact():
    """Bonds, angles and n = 3 dihedrals on every consecutive quadruple, no pair
    term: forces of one pass and a 10-step trajectory bit for bit."""
    z, scn = load("chains_dihedral")
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["force_cell"])
    assert np.array_equal(_bits(f), _bits(z["force_f"]))
    ep, _ = u.energies()
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-12 * abs(ref)
    u.steps(int(z["traj_nsteps"]))
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["traj_cell"])
    assert np.array_equal(_bits(xr), _bits(z["traj_xrel"]))
    assert np.array_equal(_bits(v), _bits(z["traj_v"]))


def test_phase_shifted_dihedrals_with_pair_potential():
    z, scn = load("chains_dihedral_shift")
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert rel_rms(f, z["force_f"]) <= 1e-5
    ep, _ = u.energies()
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-6 * abs(ref)
    u.steps(int(z["traj_nsteps"]))
    x, v, f, c, xr = u.state()
    assert np.array_equal(c, z["traj_cell"])
    L = np.asarray(scn["dim"])
    d = x - z["traj_xabs"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5


def _dihedral_energy(x, K, n, delta):
    b1, b2, b3 = x[0] - x[1], x[2] - x[1], x[3] - x[2]
    n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
    c = -(n1 @ n2) / np.linalg.norm(n1) / np.linalg.norm(n2)
    phi = np.arccos(np.clip(c, -1, 1))
    return K * (1 + np.cos(n * phi - delta)), c


def test_single_dihedral_against_central_differences():
    """Energy and forces of one dihedral against K (1 + cos(n phi - delta)) and
    its FP64 central-difference gradient; momentum is conserved (the k end
    takes the negated sum)."""
    K, n, delta = 2.0, 2, 0.0
    pot = m.Potential.harmonic_dihedral(K, n, delta)
    m.init(dim=[6.0, 6.0, 6.0], cells=[3, 3, 3], cutoff=2.0, dt=0.001)

    class Bead(m.Particle):
        mass = 1.0
        radius = 0.1

    x0 = np.array([[2.6, 2.5, 3.0], [3.0, 3.1, 3.05], [3.5, 3.0, 2.9], [3.7, 3.3, 2.4]])
    u = m.universe
    u._add_particles(x0, np.zeros((4, 3), dtype=np.float32), np.zeros(4, dtype=np.int32))
    m.Dihedral(pot, 0, 1, 2, 3)
    u.force()
    x = u.state()[0].astype(np.float64)
    f = u.state()[2].astype(np.float64)
    e_ref, c = _dihedral_energy(x, K, n, delta)
    ep, _ = u.energies()
    assert abs(ep - e_ref) <= 1e-3 * K
    h = 1e-6
    g = np.zeros_like(x)
    for p in range(4):
        for q in range(3):
            xp, xm = x.copy(), x.copy()
            xp[p, q] += h
            xm[p, q] -= h
            g[p, q] = (_dihedral_energy(xp, K, n, delta)[0] - _dihedral_energy(xm, K, n, delta)[0]) / (2 * h)
    assert np.abs(f + g).max() <= 2e-3 * np.abs(g).max(), (f, -g)
    assert np.abs(f.sum(axis=0)).max() <= 1e-5 * np.abs(f).max()


# ---- exclusions (exclusion_eval, src/mdcore/src/exclusion.cpp:83-282) ----

def test_exclusions_match_reference():
    """LJ chains with the bonded neighbours excluded from the pair potential:
    the force pass and one step against the reference engine. Beads
    of different chains that start closer than the table minimum get a random
    pair direction (a Philox draw here, an mt19937 draw there) and are left
    out, as in the other parity tests."""
    from test_gpu_parity import _close_pairs
    z, scn = load("chains_excl")
    keep = ~_close_pairs(scn, scn["x"])
    assert keep.mean() > 0.9
    u = S.build_gpu(scn)
    u.force()
    x, v, f, c, xr = u.state()
    assert rel_rms(f[keep], z["force_f"][keep]) <= 1e-5
    ep, _ = u.energies()  # a random direction keeps the pair at distance a: same energy
    ref = float(z["force_epot"])
    assert abs(ep - ref) <= 1e-6 * abs(ref)
    scn_no = dict(scn)
    scn_no.pop("ex_i")
    scn_no.pop("ex_j")
    u2 = S.build_gpu(scn_no)
    u2.force()
    # the exclusions change the forces
    assert rel_rms(u2.state()[2][keep], z["force_f"][keep]) > 1e-3
    L = np.asarray(scn["dim"])
    for nsteps in (1,):
        u = S.build_gpu(scn)
        u.steps(nsteps)
        x, v, f, c, xr = u.state()
        k = f"step{nsteps}_"
        d = x - z[k + "xabs"]
        d -= L * np.round(d / L)
        assert np.abs(d[keep]).max() < 1e-5
