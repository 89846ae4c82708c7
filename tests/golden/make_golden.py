"""Generates the golden fixtures in tests/golden/ from the reference engine
compiled in place (oracle/_ref/libmxref.so, built by `make -C oracle reference`
from the reference sources).

Run from the repository root:  python tests/golden/make_golden.py
Fixtures: small seeded cases of each workload shape (forces after one
engine_force, state after a few engine_steps, task lists, potential tables).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import scenarios as S  # noqa: E402
from oracle import refengine  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, scenario factory, steps for the trajectory fixture)
CASES = [
    ("argon_small", lambda: S.argon(n=1000, L=4.641588833612778, cells=4, seed=11), 10),
    ("argon_default_cells", lambda: S.argon(n=1000, L=10.0, cells=4, seed=12, dmin=0.3), 10),
    ("dpd_small", lambda: S.dpd(n=4000, dims=(8.0, 6.0, 7.0), seed=13), 10),
    # the bonded lattice (k=200, dissociation 2.0, dt=0.005) breaks within a few
    # steps under the reference's eff >= dissociation rule: partial break states
    ("lattice_small", lambda: S.lattice(nx=8, seed=14, pull=0.05), 3),
    ("lattice_break", lambda: S.lattice(nx=6, seed=15, pull=0.05), 2),
    ("morse2_small", lambda: S.morse2(n=1500, seed=16), 10),
    # bond lengths spread around the break threshold: one force pass on
    # identical inputs decides the flags
    ("lattice_noisy", lambda: S.lattice(nx=8, seed=17, noise=5e-3), 1),
    # bead-spring chains with harmonic angles: bonded forces only (bit-exact
    # forces and trajectories), and with a Morse pair potential
    ("chains_bonded", lambda: S.chains(nchains=16, length=24, seed=21), 10),
    ("chains_morse", lambda: S.chains(nchains=16, length=24, seed=22, pair=(0.2, 6.0, 0.5, 1e-4, 1.0, 1e-3)), 10),
    # the same with harmonic dihedrals on consecutive quadruples: n = 3, delta = 0;
    # and n = 2, delta = 1 with a Morse pair term (a phase that is not a multiple
    # of pi needs tol 0.01: at the default 0.001 the fit exceeds its interval limit
    # in the reference and here alike)
    ("chains_dihedral", lambda: S.chains(nchains=16, length=24, seed=23, dihedral=(1.5, 3, 0.0, 0.001)), 10),
    ("chains_dihedral_shift", lambda: S.chains(nchains=16, length=24, seed=24, dihedral=(0.8, 2, 1.0, 0.01),
                                               pair=(0.2, 6.0, 0.5, 1e-4, 1.0, 1e-3)), 10),
    # exclusions between bonded neighbours of the Morse chains
    ("chains_excl", lambda: S.chains(nchains=16, length=24, seed=25,
                                     pair=("lj126", (0.2, 1.0, 1e-8, 1e-4, 1e-3)), exclude_bonded=True), 10),
    # wall potentials: LJ and Morse walls on "potential" z faces; DPD walls on no-slip z faces
    ("walls_lj", lambda: S.walls(kind="lj", bc_z="potential", seed=41), 10),
    ("walls_dpd", lambda: S.walls(kind="dpd", bc_z="no_slip", seed=42), 10),
    # a fluid around three static large particles (radius > cutoff)
    ("large_fluid", lambda: S.large(seed=51), 10),
    # species fluxes (Fick, secretion, uptake, a constant species) over a Morse fluid
    ("species_fluxes", lambda: S.species(seed=61), 10),
]

TABLES = [
    ("lj_argon", "lj126", (0.275, 1.0, 9.5075e-6, 6.1545e-3, 1e-3)),
    ("lj_argon_example", "lj126", (0.275, 3.0, 9.5075e-6, 6.1545e-3, 1e-3)),
    ("morse_lattice", "morse", (0.5, 6.0, 0.5, 1e-4, 1.5, 1e-3)),
    ("morse_sorting", "morse", (0.37, 5.0, 1.0, 1e-4, 2.5, 1e-3)),
    ("morse_default", "morse", (1.0, 6.0, 0.0, 1e-4, 3.0, 1e-3)),
    ("harmonic_lattice", "harmonic", (200.0, 0.5, 0.1, 1.0, 0.009)),
    ("harmonic_unit", "harmonic", (1.0, 1.0, 0.2, 2.0, 0.018)),
    ("power_sq", "power", (1.0, 1.0, 2.0, 0.1, 3.0, 1e-3)),
    ("angle_default", "harmonic_angle", (5.0, 2.0, 0.0, 3.141592653589793, 0.005 * 3.141592653589793)),
    ("angle_narrow", "harmonic_angle", (20.0, 1.9, 1.0, 2.8, 0.009)),
    ("dihedral_n3", "harmonic_dihedral", (1.5, 3, 0.0, 0.001)),
    ("dihedral_shift", "harmonic_dihedral", (0.8, 2, 1.0, 0.01)),
    ("dihedral_pi", "harmonic_dihedral", (2.0, 1, 3.141592653589793, 0.001)),
]


def make_tables():
    import ctypes
    L = ctypes.PyDLL(refengine.LIB)
    vp, cd = ctypes.c_void_p, ctypes.c_double
    out = {}
    for name, kind, params in TABLES:
        fn = getattr(L, f"mxref_potential_{kind}")
        fn.restype = vp
        fn.argtypes = [cd] * len(params)
        if kind == "harmonic_dihedral":  # (k, n, delta, tol) with an int multiplicity
            fn.argtypes = [cd, ctypes.c_int, cd, cd]
        p = fn(*params)
        if not p:
            raise RuntimeError(f"reference table {name} failed")
        n = ctypes.c_int()
        a4 = (ctypes.c_float * 4)()
        a, b, r0 = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        fl, k = ctypes.c_uint(), ctypes.c_int()
        L.mxref_potential_info(vp(p), ctypes.byref(n), a4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(fl),
                               ctypes.byref(r0), ctypes.byref(k))
        buf = np.zeros((n.value + 1) * 8, dtype=np.float32)
        L.mxref_potential_coeffs(vp(p), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), buf.size)
        # a sweep of potential_eval_ex values across the domain
        r = np.linspace(max(a.value * 0.9, 1e-3), b.value * 1.05, 257).astype(np.float32)
        e = np.zeros_like(r)
        f = np.zeros_like(r)
        ok = np.zeros(r.shape, dtype=np.int32)
        L.mxref_potential_eval_ex.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                              ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        for q, rr in enumerate(r):
            ee, ff = ctypes.c_float(), ctypes.c_float()
            ok[q] = L.mxref_potential_eval_ex(vp(p), ctypes.c_float(0.5), ctypes.c_float(0.5),
                                              ctypes.c_float(np.float32(rr) * np.float32(rr)), ctypes.byref(ee),
                                              ctypes.byref(ff))
            e[q], f[q] = ee.value, ff.value
        out[f"{name}__kind"] = np.array(kind)
        out[f"{name}__params"] = np.array(params, dtype=np.float64)
        out[f"{name}__info"] = np.array([n.value, fl.value], dtype=np.int64)
        out[f"{name}__alpha"] = np.array(a4, dtype=np.float32)
        out[f"{name}__ab"] = np.array([a.value, b.value, r0.value], dtype=np.float32)
        out[f"{name}__coef"] = buf
        out[f"{name}__r"] = r
        out[f"{name}__e"] = e
        out[f"{name}__f"] = f
        out[f"{name}__ok"] = ok
    np.savez_compressed(os.path.join(OUT, "tables.npz"), **out)


# pairwise bond constructor cases: (name, scenario, list-order seed, list size,
# cutoff, type pairs or None)
PAIRWISE = [
    ("pw_morse_short", lambda: S.morse2(n=2000, seed=31), 1, 1500, 1.2, None),
    ("pw_morse_long_ab", lambda: S.morse2(n=2000, seed=32), 2, 2000, 3.0, [(0, 1)]),
    ("pw_lattice", lambda: S.lattice(nx=6, seed=33, noise=2e-2), 3, 216, 0.55, None),
]


def make_pairwise():
    out = {}
    for name, fac, seed, n, cutoff, tp in PAIRWISE:
        scn = fac()
        ids = np.random.default_rng(seed).permutation(len(scn["t"]))[:n].astype(np.int32)
        extra = dict(action="pairwise", pw_ids=ids, pw_cutoff=cutoff)
        if tp:
            extra.update(pw_ta=[a for a, _ in tp], pw_tb=[b for _, b in tp])
        r = refengine.run(dict(scn, **extra))
        out[f"{name}__ids"] = ids
        out[f"{name}__cutoff"] = np.float64(cutoff)
        out[f"{name}__pairs"] = np.array(tp if tp else [], dtype=np.int32).reshape(-1, 2)
        out[f"{name}__i"] = r["pw_i"]
        out[f"{name}__j"] = r["pw_j"]
        out[f"{name}__xrel"] = r["xrel"]
        out[f"{name}__cell"] = r["cell"]
        out[f"{name}__cdim"] = r["cdim"]
        out[f"{name}__dim"] = np.asarray(scn["dim"], dtype=np.float64)
        out[f"{name}__t"] = np.asarray(scn["t"], dtype=np.int32)
    np.savez_compressed(os.path.join(OUT, "pairwise.npz"), **out)


def scenario_arrays(scn):
    d = {}
    for k, v in scn.items():
        if k in ("types", "pots", "forces", "bond_pot", "angle_pot", "dihedral_pot", "bc", "wall_pots", "fluxes",
                 "sp_names"):
            d["scn_" + k] = np.array(repr(v))
        else:
            d["scn_" + k] = np.asarray(v)
    return d


def make_case(name, factory, nsteps):
    scn = factory()
    f1 = refengine.run(dict(scn, action="force", runners=1))
    tr = refengine.run(dict(scn, action="steps", nsteps=nsteps, runners=1))
    out = scenario_arrays(scn)
    for k in ("f", "cell", "xrel", "epot", "ekin", "tasks", "cdim", "h", "bond_flags", "epot_angle",
              "epot_dihedral"):
        out["force_" + k] = f1[k]
    for k in ("xrel", "xabs", "v", "cell", "epot", "ekin", "bond_flags", "species"):
        if k in tr:
            out["traj_" + k] = tr[k]
    out["traj_nsteps"] = np.int64(nsteps)
    for ns in (1, 2):
        t = refengine.run(dict(scn, action="steps", nsteps=ns, runners=1))
        for k in ("xrel", "xabs", "v", "cell", "epot", "ekin", "bond_flags", "species"):
            if k in t:
                out[f"step{ns}_" + k] = t[k]
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)


def load_scenario(z):
    scn = {}
    for k in z.files:
        if not k.startswith("scn_"):
            continue
        v = z[k]
        key = k[4:]
        if key in ("types", "pots", "forces", "bond_pot", "angle_pot", "dihedral_pot", "bc", "wall_pots", "fluxes",
                   "sp_names"):
            scn[key] = eval(str(v))  # plain literals written by scenario_arrays
        elif v.shape == ():
            scn[key] = v.item()
        else:
            scn[key] = v
    return scn


if __name__ == "__main__":
    # no arguments: everything; otherwise the named cases ("tables" for the tables)
    want = set(sys.argv[1:])
    if not want or "tables" in want:
        make_tables()
    if not want or "pairwise" in want:
        make_pairwise()
    for name, fac, ns in CASES:
        if not want or name in want:
            make_case(name, fac, ns)
            print("wrote", name)
