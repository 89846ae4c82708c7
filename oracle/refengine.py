"""Runs a scenario through the reference engine compiled in place (oracle tier A).

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU-baseline leg.
The product never imports this module.

The reference engine is a process-wide singleton (src/mdcore/include/engine.h:708),
so every scenario runs in a fresh Python process: ``run(scenario)`` writes the
scenario to a temporary .npz, runs ``python -m oracle.refengine in out`` and
reads the results back.

A scenario is a dict:
    dim, cells, cutoff, dt, bc (x, y, z strings: periodic | free_slip | no_slip),
    max_distance (-1 = default fraction), types [(mass, radius, dynamics)],
    pots [(kind, params, ti, tj)] with kind in lj126/morse/harmonic/power/dpd,
    forces [(type, fx, fy, fz)], x (N,3) float64, v (N,3), t (N,) int,
    bonds (optional): bi, bj, bond_pot (kind, params), dissociation,
    angles (optional): ai, aj, ak (vertex aj), angle_pot ("harmonic_angle", (k, theta0, min, max, tol)),
    dihedrals (optional): di, dj, dk, dl, dihedral_pot ("harmonic_dihedral", (k, n, delta, tol)),
    exclusions (optional): ex_i, ex_j (engine_exclusion_add pairs),
    action: "force" | "steps" | "pairwise", nsteps, runners (threads), time_it (bool),
    pairwise (action "pairwise"): pw_ids (list order), pw_cutoff, pw_ta/pw_tb (type pairs, optional)
        -> pw_i, pw_j: the bonds MxBond_PairwiseNew creates, in order,
    integrator (0 forward Euler, 1 Runge-Kutta 4),
    sbforces [(type, "berendsen" | "random" | "friction", params)] with the forces module's
    arguments: berenderson_tstat(tau), random(std, mean, durration),
    friction(coef, std, mean, durration) (MxForce.cpp:213-259),
    target_temperature {type: T},
    wall_pots [(face or -1, type, kind, params)] (bind(pot, boundary condition, type)),
    cuboids [(pos, size, angles)] (static cuboids), cuboid_pots [(type, kind, params)] (bind(pot, Cuboid, type)),
    species (optional): sp_nspec (per type), sp_flags (types x smax), sp_values (N x smax),
    fluxes [(kind 0 fick | 1 secrete | 2 uptake, type a, type b, species a, species b, k, decay, target)]
Results: xabs, xrel, v, f, cell, number_density (per id), tasks (rows type, sid, i, j),
    cdim, h, epot, epot_angle, epot_dihedral, ekin, bond_flags, seconds (wall time of the steps).
"""
import ctypes
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libmxref.so")


def available():
    return os.path.exists(LIB)


def _pack(scn):
    flat = {}
    for k, v in scn.items():
        if k in ("types", "pots", "forces", "bond_pot", "angle_pot", "dihedral_pot", "bc", "sbforces",
                 "target_temperature", "wall_pots", "fluxes",
                 "sp_names", "cuboids", "cuboid_pots"):
            flat[k] = np.array(repr(v))
        else:
            flat[k] = np.asarray(v)
    return flat


def _unpack(npz):
    out = {}
    for k in npz.files:
        v = npz[k]
        if k in ("types", "pots", "forces", "bond_pot", "angle_pot", "dihedral_pot", "bc", "sbforces",
                 "target_temperature", "wall_pots", "fluxes",
                 "sp_names", "cuboids", "cuboid_pots"):
            out[k] = eval(str(v))  # written by _pack from plain literals
        elif v.shape == ():
            out[k] = v.item()
        else:
            out[k] = v
    return out


def run(scn, timeout=3600):
    """Runs a scenario in a subprocess and returns the result dict."""
    if not available():
        raise RuntimeError("oracle/_ref/libmxref.so is not built (make -C oracle reference)")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        np.savez(fin, **_pack(scn))
        root = os.path.dirname(HERE)
        env = dict(os.environ)
        env["PYTHONPATH"] = root + os.pathsep + env.get("PYTHONPATH", "")
        r = subprocess.run([sys.executable, "-m", "oracle.refengine", fin, fout], cwd=root, env=env,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference engine failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-4000:]}")
        with np.load(fout, allow_pickle=False) as z:
            return {k: z[k] for k in z.files}


def _execute(scn):
    L = ctypes.PyDLL(LIB)
    cd, ci, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    P = ctypes.POINTER
    L.mxref_init.argtypes = [P(cd), P(cd), P(ci), cd, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, cd, cd, ci]
    L.mxref_add_type.argtypes = [cd, cd, ci]
    L.mxref_add_particles.argtypes = [ci, P(cd), P(cd), P(ci)]
    for fn, n in (("mxref_potential_lj126", 5), ("mxref_potential_morse", 6), ("mxref_potential_harmonic", 5),
                  ("mxref_potential_power", 6), ("mxref_potential_harmonic_angle", 5)):
        getattr(L, fn).restype = vp
        getattr(L, fn).argtypes = [cd] * n
    L.mxref_potential_dpd.restype = vp
    L.mxref_potential_dpd.argtypes = [cd, cd, cd, cd, ci]
    L.mxref_bind.argtypes = [vp, ci, ci]
    L.mxref_bind_force.argtypes = [ci, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    L.mxref_add_bonds.argtypes = [ci, P(ci), P(ci), vp, cd]
    L.mxref_get_state.argtypes = [ci, P(ctypes.c_float), P(cd), P(ctypes.c_float), P(ctypes.c_float), P(ci), P(ci)]
    L.mxref_space_info.argtypes = [P(ci), P(cd), P(ci), P(ci), P(ctypes.c_uint)]
    L.mxref_get_tasks.argtypes = [P(ci), ci]
    L.mxref_bond_flags.argtypes = [P(ctypes.c_uint), ci]
    L.mxref_energies.argtypes = [P(cd)] * 4

    def a(x, t):
        return np.ascontiguousarray(x, dtype={cd: np.float64, ci: np.int32}[t]).ctypes.data_as(P(t))

    bc = scn.get("bc", ("periodic", "periodic", "periodic"))
    origin = np.zeros(3)
    rc = L.mxref_init(a(origin, cd), a(scn["dim"], cd), a(scn["cells"], ci), float(scn["cutoff"]),
                      bc[0].encode(), bc[1].encode(), bc[2].encode(), float(scn["dt"]),
                      float(scn.get("max_distance", -1.0)), 64)
    if rc != 0:
        raise RuntimeError(f"mxref_init {rc}")
    if scn.get("integrator", 0):
        L.mxref_set_integrator(int(scn["integrator"]))
    for (m, r, d) in scn["types"]:
        L.mxref_add_type(float(m), float(r), int(d))

    def make_pot(kind, params):
        fn = {"lj126": L.mxref_potential_lj126, "morse": L.mxref_potential_morse,
              "harmonic": L.mxref_potential_harmonic, "power": L.mxref_potential_power,
              "harmonic_angle": L.mxref_potential_harmonic_angle, "dpd": L.mxref_potential_dpd,
              "harmonic_dihedral": L.mxref_potential_harmonic_dihedral}[kind]
        if kind == "dpd":
            return fn(*[float(p) for p in params[:4]], int(params[4]) if len(params) > 4 else 0)
        if kind == "harmonic_dihedral":
            fn.restype = vp
            fn.argtypes = [cd, ci, cd, cd]
            return fn(float(params[0]), int(params[1]), float(params[2]), float(params[3]))
        return fn(*[float(p) for p in params])

    keep = []
    for (kind, params, ti, tj) in scn.get("pots", []):
        p = make_pot(kind, params)
        keep.append(p)
        if L.mxref_bind(p, int(ti), int(tj)) != 0:
            raise RuntimeError("mxref_bind")
    for (t, fx, fy, fz) in scn.get("forces", []):
        if L.mxref_bind_force(int(t), float(fx), float(fy), float(fz)) < 0:
            raise RuntimeError("mxref_bind_force")
    L.mxref_bind_singlebody.argtypes = [ci] * 2 + [ctypes.c_float] * 4
    L.mxref_set_target_temperature.argtypes = [ci, cd]
    for (t, kind, params) in scn.get("sbforces", []):
        code = {"berendsen": 1, "random": 2, "friction": 3}[kind]
        q = list(params) + [0.0] * (4 - len(params))
        if L.mxref_bind_singlebody(int(t), code, *[float(v) for v in q]) < 0:
            raise RuntimeError("mxref_bind_singlebody")
    L.mxref_bind_boundary_potential.argtypes = [ci, ci, vp]
    for (face, t, kind, params) in scn.get("wall_pots", []):
        wp = make_pot(kind, params)
        keep.append(wp)
        if L.mxref_bind_boundary_potential(int(face), int(t), wp) != 0:
            raise RuntimeError("mxref_bind_boundary_potential")
    for t, temp in scn.get("target_temperature", {}).items():
        L.mxref_set_target_temperature(int(t), float(temp))
    fp = ctypes.POINTER(ctypes.c_float)
    L.mxref_add_cuboid.argtypes = [fp, fp, fp]
    L.mxref_bind_cuboid.argtypes = [vp, ci]
    for (pos, size, ang) in scn.get("cuboids", []):
        pa, sa, aa = (np.ascontiguousarray(q, dtype=np.float32) for q in (pos, size, ang))
        if L.mxref_add_cuboid(pa.ctypes.data_as(fp), sa.ctypes.data_as(fp), aa.ctypes.data_as(fp)) != 0:
            raise RuntimeError("mxref_add_cuboid")
    for (t, kind, params) in scn.get("cuboid_pots", []):
        cp = make_pot(kind, params)
        keep.append(cp)
        if L.mxref_bind_cuboid(cp, int(t)) != 0:
            raise RuntimeError("mxref_bind_cuboid")
    x = np.ascontiguousarray(scn["x"], dtype=np.float64)
    v = np.ascontiguousarray(scn["v"], dtype=np.float64)
    t = np.ascontiguousarray(scn["t"], dtype=np.int32)
    n = len(t)
    rc = L.mxref_add_particles(n, a(x, cd), a(v, cd), a(t, ci))
    if rc < 0:
        raise RuntimeError(f"mxref_add_particles {rc}")
    if "bi" in scn and len(scn["bi"]):
        bp = make_pot(*scn["bond_pot"])
        keep.append(bp)
        L.mxref_add_bonds(len(scn["bi"]), a(scn["bi"], ci), a(scn["bj"], ci), bp, float(scn["dissociation"]))
    if "ai" in scn and len(scn["ai"]):
        ap = make_pot(*scn["angle_pot"])
        keep.append(ap)
        L.mxref_add_angles.argtypes = [ci, P(ci), P(ci), P(ci), vp]
        if L.mxref_add_angles(len(scn["ai"]), a(scn["ai"], ci), a(scn["aj"], ci), a(scn["ak"], ci), ap) != 0:
            raise RuntimeError("mxref_add_angles")
    if "ex_i" in scn and len(scn["ex_i"]):
        L.mxref_add_exclusions.argtypes = [ci, P(ci), P(ci)]
        if L.mxref_add_exclusions(len(scn["ex_i"]), a(scn["ex_i"], ci), a(scn["ex_j"], ci)) != 0:
            raise RuntimeError("mxref_add_exclusions")
    if "di" in scn and len(scn["di"]):
        dp = make_pot(*scn["dihedral_pot"])
        keep.append(dp)
        L.mxref_add_dihedrals.argtypes = [ci, P(ci), P(ci), P(ci), P(ci), vp]
        if L.mxref_add_dihedrals(len(scn["di"]), a(scn["di"], ci), a(scn["dj"], ci), a(scn["dk"], ci),
                                 a(scn["dl"], ci), dp) != 0:
            raise RuntimeError("mxref_add_dihedrals")
    if scn.get("action") == "pairwise":
        hp = make_pot("harmonic", (1.0, 0.5, 0.1, 1.0, 0.009))
        keep.append(hp)
        ta = np.asarray(scn.get("pw_ta", []), dtype=np.int32)
        tb = np.asarray(scn.get("pw_tb", []), dtype=np.int32)
        ids = np.asarray(scn["pw_ids"], dtype=np.int32)
        L.mxref_pairwise.argtypes = [ci, P(ci), ctypes.c_float, vp, ci, P(ci), P(ci)]
        t0 = time.perf_counter()
        cnt = L.mxref_pairwise(len(ids), a(ids, ci), float(scn["pw_cutoff"]), hp, len(ta), a(ta, ci), a(tb, ci))
        seconds = time.perf_counter() - t0
        if cnt < 0:
            raise RuntimeError("mxref_pairwise")
        nb0 = len(scn["bi"]) if "bi" in scn else 0
        tot = nb0 + cnt
        bi = np.zeros(max(tot, 1), dtype=np.int32)
        bj = np.zeros(max(tot, 1), dtype=np.int32)
        L.mxref_bond_ids.argtypes = [P(ci), P(ci), ci]
        L.mxref_bond_ids(a(bi, ci), a(bj, ci), len(bi))
        n = len(scn["t"])
        xr = np.zeros((n, 3), dtype=np.float32)
        xa = np.zeros((n, 3))
        vv = np.zeros((n, 3), dtype=np.float32)
        ff = np.zeros((n, 3), dtype=np.float32)
        cc = np.zeros(n, dtype=np.int32)
        tt = np.zeros(n, dtype=np.int32)
        L.mxref_get_state(n, xr.ctypes.data_as(P(ctypes.c_float)), xa.ctypes.data_as(P(cd)),
                          vv.ctypes.data_as(P(ctypes.c_float)), ff.ctypes.data_as(P(ctypes.c_float)),
                          cc.ctypes.data_as(P(ci)), tt.ctypes.data_as(P(ci)))
        cdim = np.zeros(3, dtype=np.int32)
        h = np.zeros(3)
        nc, nt, per = ci(), ci(), ctypes.c_uint()
        L.mxref_space_info(cdim.ctypes.data_as(P(ci)), h.ctypes.data_as(P(cd)), ctypes.byref(nc), ctypes.byref(nt),
                           ctypes.byref(per))
        return {"pw_i": bi[nb0:tot].copy(), "pw_j": bj[nb0:tot].copy(), "seconds": np.float64(seconds),
                "xrel": xr, "cell": cc, "cdim": cdim}
    L.mxref_add_flux.argtypes = [ci] * 5 + [ctypes.c_float] * 3
    for (kind, ta, tb, ia, ib, kk, dec, tgt) in scn.get("fluxes", []):
        if L.mxref_add_flux(int(kind), int(ta), int(tb), int(ia), int(ib), float(kk), float(dec), float(tgt)) != 0:
            raise RuntimeError("mxref_add_flux")
    smax = 0
    if "sp_values" in scn:
        sv = np.ascontiguousarray(scn["sp_values"], dtype=np.float32)
        smax = sv.shape[1]
        L.mxref_set_species.argtypes = [ci, ci, P(ci), P(ctypes.c_uint), P(ctypes.c_float)]
        L.mxref_set_species(n, smax, a(scn["sp_nspec"], ci),
                            np.ascontiguousarray(scn["sp_flags"], dtype=np.uint32).ctypes.data_as(P(ctypes.c_uint)),
                            sv.ctypes.data_as(P(ctypes.c_float)))
    L.mxref_start(int(scn.get("runners", 1)))
    t0 = time.perf_counter()
    if scn.get("action", "force") == "force":
        rc = L.mxref_force()
    else:
        warm = int(scn.get("warmup", 0))
        if warm:
            L.mxref_step(warm)
        t0 = time.perf_counter()
        rc = L.mxref_step(int(scn["nsteps"]))
    seconds = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"reference step/force returned {rc}")
    out = {"seconds": np.float64(seconds)}
    xr = np.zeros((n, 3), dtype=np.float32)
    xa = np.zeros((n, 3))
    vv = np.zeros((n, 3), dtype=np.float32)
    ff = np.zeros((n, 3), dtype=np.float32)
    cc = np.zeros(n, dtype=np.int32)
    tt = np.zeros(n, dtype=np.int32)
    L.mxref_get_state(n, xr.ctypes.data_as(P(ctypes.c_float)), xa.ctypes.data_as(P(cd)),
                      vv.ctypes.data_as(P(ctypes.c_float)), ff.ctypes.data_as(P(ctypes.c_float)),
                      cc.ctypes.data_as(P(ci)), tt.ctypes.data_as(P(ci)))
    out.update(xrel=xr, xabs=xa, v=vv, f=ff, cell=cc)
    nd = np.zeros(n, dtype=np.float32)
    L.mxref_number_density(n, nd.ctypes.data_as(P(ctypes.c_float)))
    out["number_density"] = nd
    cdim = np.zeros(3, dtype=np.int32)
    h = np.zeros(3)
    nc, nt, per = ci(), ci(), ctypes.c_uint()
    L.mxref_space_info(cdim.ctypes.data_as(P(ci)), h.ctypes.data_as(P(cd)), ctypes.byref(nc), ctypes.byref(nt),
                       ctypes.byref(per))
    tasks = np.zeros(4 * nt.value, dtype=np.int32)
    L.mxref_get_tasks(tasks.ctypes.data_as(P(ci)), tasks.size)
    out.update(cdim=cdim, h=h, tasks=tasks.reshape(-1, 4), period=np.uint32(per.value))
    nb = len(scn["bi"]) if "bi" in scn else 0
    bf = np.zeros(max(nb, 1), dtype=np.uint32)
    L.mxref_bond_flags(bf.ctypes.data_as(P(ctypes.c_uint)), bf.size)
    out["bond_flags"] = bf[:nb]
    e = [cd() for _ in range(4)]
    L.mxref_energies(*[ctypes.byref(q) for q in e])
    # total potential energy of the last force pass: bonded part (in s->epot after
    # engine_force) plus the per-cell nonbonded energies
    if scn.get("action", "force") == "force":
        out["epot"] = np.float64(e[0].value + e[1].value)
    else:
        out["epot"] = np.float64(e[0].value)
    out["epot_nonbond"] = np.float64(e[1].value)
    out["epot_bond"] = np.float64(e[2].value)
    out["ekin"] = np.float64(e[3].value)
    if smax:
        spo = np.zeros((n, smax), dtype=np.float32)
        L.mxref_get_species.argtypes = [ci, ci, P(ctypes.c_float)]
        L.mxref_get_species(n, smax, spo.ctypes.data_as(P(ctypes.c_float)))
        out["species"] = spo
    L.mxref_epot_angle.restype = cd
    out["epot_angle"] = np.float64(L.mxref_epot_angle())
    L.mxref_epot_dihedral.restype = cd
    out["epot_dihedral"] = np.float64(L.mxref_epot_dihedral())
    return out


if __name__ == "__main__":
    with np.load(sys.argv[1], allow_pickle=False) as z:
        scn = _unpack(z)
    res = _execute(scn)
    np.savez(sys.argv[2], **res)
    sys.stdout.flush()
    os._exit(0)  # runner threads of the reference engine never exit on their own
