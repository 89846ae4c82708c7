"""Oracle pins: tier B (own restatement, FP32 and FP64) against the golden
vectors produced by the reference engine compiled in place (tier A)."""
import numpy as np
import pytest

from oracle import restatement as R

from golden_util import CASES, fp64_total, load, ref_tasks, rel_rms

NONBONDED = [c for c in CASES if not c.startswith("lattice")]


@pytest.mark.parametrize("name", NONBONDED)
def test_tier_b_fp32_matches_reference(name):
    z, scn = load(name)
    f, ep, cnt = R.nonbond(scn, z["force_xrel"], scn["v"], z["force_cell"], ref_tasks(z), z["force_cdim"],
                           precision=32)
    # same per-pair arithmetic; only the order of the per-particle sums differs
    assert rel_rms(f, z["force_f"]) < 1e-6
    if float(z["force_epot"]) != 0.0:
        assert abs(ep - float(z["force_epot"])) <= 1e-6 * abs(float(z["force_epot"])) + 1e-9
    assert cnt[2] == 0  # no pair below the table minimum in these inputs


@pytest.mark.parametrize("name", NONBONDED)
def test_tier_b_fp64_close_to_reference(name):
    """FP32 rounding of the reference stated against the FP64 oracle."""
    z, scn = load(name)
    f64, ep64, _ = R.nonbond(scn, z["force_xrel"], scn["v"], z["force_cell"], ref_tasks(z), z["force_cdim"],
                             precision=64)
    assert rel_rms(z["force_f"], f64) < 1e-5


BONDED = ["lattice_small", "lattice_break", "lattice_noisy", "chains_bonded", "chains_morse", "chains_dihedral",
          "chains_dihedral_shift", "chains_excl"]


@pytest.mark.parametrize("name", BONDED)
def test_fp64_bonded_restatement_matches_reference(name):
    """The FP64 oracle with bonded terms (tier B nonbonded + the bonded restatement) against
    the reference engine's FP32 force pass: forces within the reference's own FP32 error
    (1e-5 relative RMS), energies within 1e-6. Particles in pairs closer than the table
    minimum (a random direction in the reference) are left out of the force comparison;
    their energy is not restated, so the energy check skips cases that have them."""
    from test_gpu_parity import _close_pairs
    z, scn = load(name)
    f64, ep64 = fp64_total(scn, z["force_xrel"], scn["v"], z["force_cell"], z, z["force_bond_flags"])
    keep = ~_close_pairs(scn, scn["x"])
    assert rel_rms(z["force_f"][keep], f64[keep]) < 1e-5
    if keep.all():
        ref = float(z["force_epot"])
        assert abs(ep64 - ref) <= 1e-6 * abs(ref)


def test_tier_b_bonds_excluded_lattice_nonbonded():
    """Lattice nonbonded part: reference forces minus tier B nonbonded are the
    bond forces, which vanish for intact bonds at rest length."""
    z, scn = load("lattice_small")
    f, ep, cnt = R.nonbond(scn, z["force_xrel"], scn["v"], z["force_cell"], ref_tasks(z), z["force_cdim"],
                           precision=32)
    bond = np.asarray(z["force_f"], dtype=np.float64) - f
    # bonds at (nearly) rest length contribute little compared with the Morse forces
    assert np.sqrt((bond ** 2).mean()) < 0.5 * np.sqrt((f ** 2).mean())


@pytest.mark.parametrize("name", ["pw_morse_short", "pw_morse_long_ab", "pw_lattice"])
def test_pairlist_restatement_matches_reference(name):
    """The numpy restatement of make_pairlist reproduces the reference's
    pairwise bonds (ids and order) on the fixture's placement."""
    import os
    from golden_util import GOLDEN
    z = np.load(os.path.join(GOLDEN, "pairwise.npz"))
    origins = R.cell_origins(z[f"{name}__dim"], z[f"{name}__cdim"])
    pairs = [tuple(p) for p in z[f"{name}__pairs"]] or None
    fi, fj = R.pairlist(z[f"{name}__ids"], z[f"{name}__xrel"], z[f"{name}__cell"], origins, z[f"{name}__t"],
                        float(z[f"{name}__cutoff"]), pairs)
    assert np.array_equal(fi, z[f"{name}__i"])
    assert np.array_equal(fj, z[f"{name}__j"])


def test_flux_restatement_matches_reference():
    """The FP64 restatement of one species step (fluxes, then the update of the
    particles that kept their cell) reproduces the reference engine's."""
    import os
    from golden_util import GOLDEN
    from make_golden import load_scenario
    z = np.load(os.path.join(GOLDEN, "species_fluxes.npz"))
    scn = load_scenario(z)
    t = scn["t"]
    konst = np.zeros_like(scn["sp_values"])
    for ty in range(len(scn["sp_nspec"])):
        konst[t == ty] = (scn["sp_flags"][ty] & 4) != 0
    moved = z["force_cell"] != z["step1_cell"]
    out = R.flux_step(scn["x"], t, np.asarray(scn["dim"]), scn["cutoff"], scn["dt"], scn["sp_values"],
                      scn["fluxes"], konst, moved)
    assert moved.sum() > 0
    assert np.abs(out - z["step1_species"]).max() <= 1e-6


def test_group_metrics_restatement_known_answer():
    """Two particles at x = 0 and 2 with masses 1 and 3 (metrics.cpp:330-466): centroid
    1, centre of mass 1.5, radius of gyration sqrt(|1 - 0| + |1 - 2|) = sqrt(2) (the
    reference sums distances, not squares), inertia about the centre of mass
    diag(0, 3, 3); the FP32 running sums give the same values here."""
    import numpy as np
    from oracle import restatement as R
    x = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]])
    m = np.array([1.0, 3.0])
    for fp32 in (False, True):
        M, com, cen, rog, I = R.group_metrics(x, m, fp32=fp32)
        assert M == 4.0
        assert np.allclose(com, [1.5, 0, 0]) and np.allclose(cen, [1.0, 0, 0])
        assert abs(rog - np.sqrt(2.0)) < 1e-7
        assert np.allclose(I, np.diag([0.0, 3.0, 3.0]))
    # an off-diagonal term keeps the reference's + sign
    x = np.array([[1.0, 1.0, 0.0], [-1.0, -1.0, 0.0]])
    I = R.group_metrics(x, np.ones(2))[4]
    assert I[0, 1] == 2.0 and I[1, 0] == 2.0


def test_group_metrics_fp32_close_to_fp64():
    import numpy as np
    from oracle import restatement as R
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 10, size=(400, 3))
    m = rng.uniform(1, 3, size=400)
    a, b = R.group_metrics(x, m), R.group_metrics(x, m, fp32=True)
    assert abs(a[0] - b[0]) <= 1e-6 * a[0]
    assert np.abs(a[1] - b[1]).max() <= 1e-6 * np.abs(a[1]).max()
    assert np.abs(a[2] - b[2]).max() <= 1e-6 * np.abs(a[2]).max()
    assert abs(a[3] - b[3]) <= 1e-6 * a[3]
    assert np.abs(a[4] - b[4]).max() <= 1e-5 * np.abs(a[4]).max()
