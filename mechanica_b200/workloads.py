"""Seeded synthetic workloads shaped like the benchmark configurations, and a
helper that builds a workload in the engine through the Python surface. The
same dict describes the workload to the reference engine in the tests.

Shapes follow the five workloads of the force-and-step path:
  argon   LJ 12-6 fluid, one type, mass 39.4, periodic cube, density 10
  dpd     DPD fluid with a constant body force, periodic x/y, no-slip z walls
  lattice simple-cubic harmonic-bonded lattice with Morse nonbonded, overdamped
  morse2  two-type Morse mixture, overdamped, periodic (batched replicas)
Sizes are parameters so tests run small cases and the bench runs full ones.
"""
import numpy as np

import mechanica_b200 as m


def _reject_close(x, L, dmin, rng):
    """Replaces points closer than dmin to an earlier point (periodic cube)."""
    n = len(x)
    ncell = max(1, int(L // max(dmin, 1e-9)))
    h = L / ncell
    for _ in range(200):
        idx = np.floor(x / h).astype(np.int64) % ncell
        key = (idx[:, 0] * ncell + idx[:, 1]) * ncell + idx[:, 2]
        order = np.argsort(key, kind="stable")
        bad = np.zeros(n, dtype=bool)
        # compare against the 27 neighbouring cells
        buckets = {}
        for p in order:
            buckets.setdefault(int(key[p]), []).append(p)
        for p in range(n):
            i, j, k = idx[p]
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    for dk in (-1, 0, 1):
                        kk = (((i + di) % ncell) * ncell + (j + dj) % ncell) * ncell + (k + dk) % ncell
                        for q in buckets.get(int(kk), ()):
                            if q < p:
                                d = x[p] - x[q]
                                d -= L * np.round(d / L)
                                if d @ d < dmin * dmin:
                                    bad[p] = True
                                    break
                        if bad[p]:
                            break
                    if bad[p]:
                        break
                if bad[p]:
                    break
        if not bad.any():
            return x
        x[bad] = rng.uniform(0, L, size=(int(bad.sum()), 3))
    raise RuntimeError("rejection sampling did not converge")


def argon(n=10000, L=10.0, cells=10, seed=1, dmin=0.3, temperature=100.0, mass=39.4, dt=0.01):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, L, size=(n, 3))
    if dmin > 0:
        x = _reject_close(x, L, dmin, rng)
    x = x.astype(np.float32).astype(np.float64)
    v = rng.normal(0, np.sqrt(temperature / mass), size=(n, 3))
    v -= v.mean(axis=0)
    v = v.astype(np.float32).astype(np.float64)
    return dict(dim=[L, L, L], cells=[cells] * 3, cutoff=1.0, dt=dt, bc=("periodic", "periodic", "periodic"),
                types=[(mass, 0.1, m.Newtonian)],
                pots=[("lj126", (0.275, 1.0, 9.5075e-6, 6.1545e-3, 1e-3), 0, 0)],
                forces=[], x=x, v=v, t=np.zeros(n, dtype=np.int32))


def dpd(n=200000, dims=(40.0, 20.0, 20.0), seed=2, body=0.02, dt=0.01):
    rng = np.random.default_rng(seed)
    d = np.asarray(dims)
    x = rng.uniform(0, 1, size=(n, 3)) * d
    x = np.minimum(x, d * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    v = rng.normal(0, 1.0, size=(n, 3))
    v -= v.mean(axis=0)
    v = v.astype(np.float32).astype(np.float64)
    cells = [int(c) for c in d]  # cutoff 1.0
    return dict(dim=list(d), cells=cells, cutoff=1.0, dt=dt, bc=("periodic", "periodic", "no_slip"),
                types=[(1.0, 0.5, m.Newtonian)],
                pots=[("dpd", (25.0, 4.5, 3.0, 1.0, 0), 0, 0)],
                forces=[(0, body, 0.0, 0.0)], x=x, v=v, t=np.zeros(n, dtype=np.int32))


def lattice(nx=32, spacing=0.5, seed=3, dt=0.005, pull=0.05, dissociation=2.0, k=200.0, margin=2.0, noise=1e-4,
            radius=0.5):
    """nx^3 simple-cubic lattice, harmonic bonds to the 6 nearest neighbours,
    Morse nonbonded (d=0.5, a=6, r0=0.5, cutoff 1.5); the top layer is a
    separate type pulled by a constant force in +z. Free-slip walls."""
    rng = np.random.default_rng(seed)
    g = np.arange(nx) * spacing + spacing / 2 + margin / 2
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    x += rng.normal(0, noise * spacing, size=x.shape)
    x = x.astype(np.float32).astype(np.float64)
    n = len(x)
    idx = np.arange(n).reshape(nx, nx, nx)
    t = np.zeros(n, dtype=np.int32)
    t[idx[:, :, -1].ravel()] = 1
    bi, bj = [], []
    for ax in range(3):
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[ax] = slice(0, nx - 1)
        sl_b[ax] = slice(1, nx)
        bi.append(idx[tuple(sl_a)].ravel())
        bj.append(idx[tuple(sl_b)].ravel())
    bi = np.concatenate(bi).astype(np.int32)
    bj = np.concatenate(bj).astype(np.int32)
    L = nx * spacing + margin
    cut = 1.5
    cells = int(L // cut)
    return dict(dim=[L, L, L + 2.0], cells=[cells, cells, int((L + 2.0) // cut)], cutoff=cut, dt=dt,
                bc=("free_slip", "free_slip", "free_slip"),
                types=[(1.0, radius, m.Overdamped), (1.0, radius, m.Overdamped)],
                pots=[("morse", (0.5, 6.0, 0.5, 1e-4, cut, 1e-3), 0, 0), ("morse", (0.5, 6.0, 0.5, 1e-4, cut, 1e-3), 0, 1),
                      ("morse", (0.5, 6.0, 0.5, 1e-4, cut, 1e-3), 1, 1)],
                forces=[(1, 0.0, 0.0, pull)], x=x, v=np.zeros_like(x), t=t,
                bi=bi, bj=bj, bond_pot=("harmonic", (k, spacing, 0.1, 1.0, 0.009)), dissociation=dissociation)


def walls(n=3000, L=8.0, seed=6, dt=0.005, kind="lj", bc_z="potential", temperature=0.5):
    """A two-type fluid between z walls with wall potentials (the box's other
    axes periodic). kind "lj": Morse pairs, a repulsive r^-12 wall on both z
    faces for type 0 and a Morse wall on the top face only for type 1.
    kind "dpd": a DPD fluid with a DPD wall potential on every face (only the
    non-periodic z faces act)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, L, size=(n, 3))
    x[:, 2] = rng.uniform(0.05, L - 0.05, size=n)
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    t = (np.arange(n) % 2).astype(np.int32)
    v = rng.normal(0, np.sqrt(temperature), size=(n, 3))
    v -= v.mean(axis=0)
    v = v.astype(np.float32).astype(np.float64)
    cut = 1.0
    cells = [int(L // cut)] * 3
    if kind == "dpd":
        pots = [("dpd", (25.0, 4.5, 3.0, cut, 0), 0, 0), ("dpd", (25.0, 4.5, 3.0, cut, 0), 0, 1),
                ("dpd", (25.0, 4.5, 3.0, cut, 0), 1, 1)]
        wall = [(-1, 0, "dpd", (25.0, 4.5, 3.0, cut, 0)), (-1, 1, "dpd", (40.0, 4.5, 3.0, cut, 0))]
        types = [(1.0, 0.5, m.Newtonian), (1.0, 0.5, m.Newtonian)]
    else:
        # shifted Morse tables span r - (ri + rj) + r0 + 1, so max covers the cutoff
        morse = (0.3, 5.0, 0.6, 1e-4, 2.0, 1e-3)
        pots = [("morse", morse, 0, 0), ("morse", morse, 0, 1), ("morse", morse, 1, 1)]
        wall = [(4, 0, "lj126", (0.3, 1.0, 1e-6, 0.0, 1e-3)), (5, 0, "lj126", (0.3, 1.0, 1e-6, 0.0, 1e-3)),
                (5, 1, "morse", (0.5, 4.0, 0.3, 1e-4, 2.0, 1e-3))]
        types = [(1.0, 0.3, m.Newtonian), (1.0, 0.3, m.Newtonian)]
    return dict(dim=[L, L, L], cells=cells, cutoff=cut, dt=dt, bc=("periodic", "periodic", bc_z), types=types,
                pots=pots, forces=[], x=x, v=v, t=t, wall_pots=wall)


def large(n=3000, L=10.0, nlarge=3, seed=7, dt=0.005, big=2.0, temperature=0.3):
    """A fluid of small particles (radius 0.3, Morse pairs) around a few large
    particles (radius big > cutoff 1.0: the reference's PARTICLE_LARGE), which
    stay put and act on every small particle through a shifted Morse
    potential. Small particles start outside the large ones' radius."""
    rng = np.random.default_rng(seed)
    xl = rng.uniform(big + 0.5, L - big - 0.5, size=(nlarge, 3))
    x = rng.uniform(0, L, size=(4 * n, 3))
    keep = np.ones(len(x), dtype=bool)
    for c in xl:
        keep &= np.linalg.norm(x - c, axis=1) > big + 0.3
    x = x[keep][:n]
    x = np.concatenate([x, xl])
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    t = np.concatenate([np.zeros(len(x) - nlarge, dtype=np.int32), np.ones(nlarge, dtype=np.int32)])
    v = rng.normal(0, np.sqrt(temperature), size=x.shape)
    v[t == 1] = 0.0
    v = v.astype(np.float32).astype(np.float64)
    cut = 1.0
    small = (0.3, 5.0, 0.6, 1e-4, 2.0, 1e-3)
    return dict(dim=[L, L, L], cells=[int(L // cut)] * 3, cutoff=cut, dt=dt, bc=("periodic", "periodic", "periodic"),
                types=[(1.0, 0.3, m.Newtonian), (10.0, big, m.Newtonian)],
                pots=[("morse", small, 0, 0), ("morse", (0.5, 3.0, 0.2, 1e-4, 3.0, 1e-3), 0, 1)],
                forces=[], x=x, v=v, t=t)


def species(n=2000, L=8.0, seed=8, dt=0.01, temperature=0.3):
    """Two particle types carrying species (A: S1, S2, S3 with S3 constant; B:
    S1, S2), with a Fick flux of S1 among A particles, secretion of S2 from B to
    A and uptake of S1 by B from A, over a Morse fluid in a periodic box.
    sp_* arrays describe the state vectors; fluxes lists (kind, type a, type b,
    species index in a, species index in b, k, decay, target)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, L, size=(n, 3))
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    t = (rng.uniform(size=n) < 0.3).astype(np.int32)  # 0: A, 1: B
    v = rng.normal(0, np.sqrt(temperature), size=(n, 3))
    v = v.astype(np.float32).astype(np.float64)
    cut = 1.0
    morse = (0.2, 5.0, 0.6, 1e-4, 2.0, 1e-3)
    smax = 3
    values = rng.uniform(0, 1, size=(n, smax)).astype(np.float32)
    values[t == 1, 2] = 0.0
    return dict(dim=[L, L, L], cells=[int(L // cut)] * 3, cutoff=cut, dt=dt, bc=("periodic", "periodic", "periodic"),
                types=[(1.0, 0.3, m.Newtonian), (1.0, 0.3, m.Newtonian)],
                pots=[("morse", morse, 0, 0), ("morse", morse, 0, 1), ("morse", morse, 1, 1)],
                forces=[], x=x, v=v, t=t,
                sp_nspec=np.array([3, 2], dtype=np.int32), sp_names=[["S1", "S2", "$S3"], ["S1", "S2"]],
                sp_flags=np.array([[0, 0, 4], [0, 0, 0]], dtype=np.uint32), sp_values=values,
                fluxes=[(0, 0, 0, 0, 0, 2.0, 0.1, 0.0), (1, 1, 0, 1, 1, 1.0, 0.0, 0.5),
                        (2, 0, 1, 0, 0, 0.5, 0.05, 1.0), (0, 0, 0, 2, 2, 1.0, 0.0, 0.0)])


def chains(nchains=64, length=32, bond=0.5, L=8.0, seed=5, dt=0.002, k_bond=100.0, k_angle=5.0, theta0=2.0,
           pair=None, cut=1.0, temperature=0.1, dihedral=None, exclude_bonded=False):
    """Bead-spring chains in a periodic cube: harmonic bonds between consecutive
    beads (k_bond (r - bond)^2, never breaking) and harmonic angles on
    consecutive triples (k_angle (theta - theta0)^2, vertex at the middle bead).
    Chains are random walks with bond-length steps whose turning angle stays
    near pi - theta0, wrapped into the box, so bonds and angles cross the
    periodic faces. pair: None (bonded forces only), the parameters of a Morse
    potential bound on the bead type, or (kind, parameters). dihedral: None or (k, n, delta, tol) of a
    harmonic dihedral on consecutive quadruples. exclude_bonded: exclusions
    between bonded neighbours (the pair potential taken back). Newtonian, mass 1."""
    rng = np.random.default_rng(seed)
    xs = []
    for _ in range(nchains):
        p = rng.uniform(0, L, size=3)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        pts = [p]
        for _ in range(length - 1):
            # turn by pi - theta0 (jittered) about a random axis perpendicular to d
            ax = np.cross(d, rng.normal(size=3))
            ax /= np.linalg.norm(ax)
            turn = (np.pi - theta0) + rng.normal(0, 0.15)
            d = d * np.cos(turn) + np.cross(ax, d) * np.sin(turn)
            d /= np.linalg.norm(d)
            p = p + bond * (1 + rng.normal(0, 0.05)) * d
            pts.append(p)
        xs.append(np.array(pts))
    x = np.mod(np.concatenate(xs), L)
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    n = len(x)
    idx = np.arange(n).reshape(nchains, length)
    bi = idx[:, :-1].ravel().astype(np.int32)
    bj = idx[:, 1:].ravel().astype(np.int32)
    ai = idx[:, :-2].ravel().astype(np.int32)
    aj = idx[:, 1:-1].ravel().astype(np.int32)
    ak = idx[:, 2:].ravel().astype(np.int32)
    v = rng.normal(0, np.sqrt(temperature), size=(n, 3))
    v -= v.mean(axis=0)
    cells = int(L // cut)
    if pair is None:
        pots = []
    elif isinstance(pair[0], str):  # (kind, params)
        pots = [(pair[0], tuple(pair[1]), 0, 0)]
    else:
        pots = [("morse", tuple(pair), 0, 0)]
    extra = {}
    if exclude_bonded:
        extra.update(ex_i=bi.copy(), ex_j=bj.copy())
    if dihedral is not None:
        kd, nd, dd, tol = dihedral
        extra = dict(di=idx[:, :-3].ravel().astype(np.int32), dj=idx[:, 1:-2].ravel().astype(np.int32),
                     dk=idx[:, 2:-1].ravel().astype(np.int32), dl=idx[:, 3:].ravel().astype(np.int32),
                     dihedral_pot=("harmonic_dihedral", (float(kd), int(nd), float(dd), float(tol))))
    return dict(**extra, dim=[L, L, L], cells=[cells] * 3, cutoff=cut, dt=dt, bc=("periodic", "periodic", "periodic"),
                types=[(1.0, 0.25, m.Newtonian)], pots=pots, forces=[], x=x, v=v, t=np.zeros(n, dtype=np.int32),
                bi=bi, bj=bj, bond_pot=("harmonic", (k_bond, bond, 0.1, 1.0, 0.009)),
                dissociation=float(np.finfo(np.float64).max),
                ai=ai, aj=aj, ak=ak, angle_pot=("harmonic_angle", (k_angle, theta0, 0.0, np.pi, 0.005 * np.pi)))


def morse2(n=4000, density=0.8, seed=4, dt=0.01, d=(0.6, 0.3, 0.8), cut=2.5):
    rng = np.random.default_rng(seed)
    L = (n / density) ** (1.0 / 3.0)
    x = rng.uniform(0, L, size=(n, 3))
    x = _reject_close(x, L, 0.6, rng).astype(np.float32).astype(np.float64)
    t = (np.arange(n) % 2).astype(np.int32)
    cells = max(3, int(L // cut))
    dAA, dAB, dBB = d
    return dict(dim=[L, L, L], cells=[cells] * 3, cutoff=cut, dt=dt, bc=("periodic", "periodic", "periodic"),
                types=[(1.0, 1.0, m.Overdamped), (1.0, 1.0, m.Overdamped)],
                pots=[("morse", (dAA, 5.0, 1.0, 1e-4, cut, 1e-3), 0, 0), ("morse", (dAB, 5.0, 1.0, 1e-4, cut, 1e-3), 0, 1),
                      ("morse", (dBB, 5.0, 1.0, 1e-4, cut, 1e-3), 1, 1)],
                forces=[], x=x, v=np.zeros_like(x), t=t)


def make_potential(kind, params):
    if kind == "lj126":
        return m.Potential.lennard_jones_12_6(*params)
    if kind == "morse":
        return m.Potential.morse(*params)
    if kind == "harmonic":
        k, r0, mn, mx, tol = params
        return m.Potential.harmonic(k, r0, mn, mx, tol)
    if kind == "power":
        return m.Potential.power(*params)
    if kind == "dpd":
        return m.Potential.dpd(*params[:4], shifted=bool(params[4]) if len(params) > 4 else False)
    if kind == "harmonic_angle":
        return m.Potential.harmonic_angle(*params)
    if kind == "harmonic_dihedral":
        k, n, delta, tol = params
        return m.Potential.harmonic_dihedral(k, int(n), delta, tol)
    raise ValueError(kind)


def build_gpu(scn, rng_mode="reference"):
    """Builds the scenario in the B200 engine through the Python surface."""
    bc = {"x": scn["bc"][0], "y": scn["bc"][1], "z": scn["bc"][2]}
    m.init(dim=scn["dim"], cells=scn["cells"], cutoff=scn["cutoff"], dt=scn["dt"], bc=bc, rng=rng_mode,
           max_distance=scn.get("max_distance"), integrator=scn.get("integrator", m.FORWARD_EULER))
    types = []
    for k, (mass, radius, dyn) in enumerate(scn["types"]):
        attrs = {"mass": mass, "radius": radius, "dynamics": dyn}
        if "sp_names" in scn and scn["sp_nspec"][k] > 0:
            attrs["species"] = list(scn["sp_names"][k])
        types.append(type(f"T{k}", (m.Particle,), attrs))
    for (kind, params, ti, tj) in scn["pots"]:
        m.bind(make_potential(kind, params), types[ti], types[tj])
    for (ti, fx, fy, fz) in scn["forces"]:
        m.bind(m.forces.ConstantForce([fx, fy, fz]), types[ti])
    for (pos, size, ang) in scn.get("cuboids", []):
        m.Cuboid(pos, size, ang)
    for (ti, kind, params) in scn.get("cuboid_pots", []):
        m.bind(make_potential(kind, params), m.Cuboid, types[ti])
    for (face, ti, kind, params) in scn.get("wall_pots", []):
        bcs = m.universe.boundary_conditions
        m.bind(make_potential(kind, params), bcs if face < 0 else getattr(bcs, m._FACES[face]), types[ti])
    x, v, t = scn["x"], scn["v"], scn["t"]
    # create in id order, type by type, keeping ids equal to the scenario's indices
    assert np.all(np.diff(np.flatnonzero(t == t[0])) >= 1)
    u = m.universe
    u._add_particles(np.asarray(x), np.asarray(v, dtype=np.float32), np.asarray(t, dtype=np.int32))
    if "bi" in scn and len(scn["bi"]):
        kind, params = scn["bond_pot"]
        u._add_bonds(make_potential(kind, params), scn["bi"], scn["bj"], scn["dissociation"])
    if "ai" in scn and len(scn["ai"]):
        u._add_angles(make_potential(*scn["angle_pot"]), scn["ai"], scn["aj"], scn["ak"])
    for (kind, ta, tb, ia, ib, k, decay, target) in scn.get("fluxes", []):
        name = scn["sp_names"][ta][ia].lstrip("$")
        assert scn["sp_names"][tb][ib].lstrip("$") == name
        u._add_flux(kind, types[ta], types[tb], name, k, decay, target)
    if "sp_values" in scn:
        u.set_species_values(np.asarray(scn["sp_values"], dtype=np.float32))
    if "ex_i" in scn and len(scn["ex_i"]):
        u.add_exclusions(scn["ex_i"], scn["ex_j"])
    if "di" in scn and len(scn["di"]):
        u._add_dihedrals(make_potential(*scn["dihedral_pot"]), scn["di"], scn["dj"], scn["dk"], scn["dl"])
    return u


def cell_sorting_specs(nrep=256, seed=5, nmin=1000, nmax=20000, density=0.8, cut=2.5, dt=0.01, a=5.0, r0=1.0):
    """Replicas of the two-type cell-sorting mixture: particle counts uniform in
    [nmin, nmax], cubic periodic boxes at the given density, 50/50 types, Morse
    per type pair with d_AA, d_BB ~ U(0.2, 1.0), d_AB ~ U(0.05, 0.5), overdamped."""
    rng = np.random.default_rng(seed)
    specs = []
    for r in range(nrep):
        n = int(rng.integers(nmin, nmax + 1))
        L = (n / density) ** (1.0 / 3.0)
        x = rng.uniform(0, L, size=(n, 3)).astype(np.float32).astype(np.float64)
        x = np.minimum(x, np.float32(L) * (1 - 1e-6))
        t = np.zeros(n, dtype=np.int32)
        t[rng.permutation(n)[: n // 2]] = 1
        cells = max(3, int(L // cut))
        dAA, dBB = rng.uniform(0.2, 1.0, size=2)
        dAB = rng.uniform(0.05, 0.5)
        specs.append(dict(dim=[L, L, L], cells=[cells] * 3, cutoff=cut, dt=dt, bc=("periodic", "periodic", "periodic"),
                          types=[(1.0, 1.0, m.Overdamped), (1.0, 1.0, m.Overdamped)],
                          pots=[("morse", (float(dAA), a, r0, 1e-4, cut, 1e-3), 0, 0),
                                ("morse", (float(dAB), a, r0, 1e-4, cut, 1e-3), 0, 1),
                                ("morse", (float(dBB), a, r0, 1e-4, cut, 1e-3), 1, 1)],
                          forces=[], x=x, v=np.zeros_like(x), t=t))
    return specs


def build_gpu_batch(specs, stream=None):
    """All replicas in one engine (one set of kernel launches per step). Types
    come from the first spec and are shared; potentials are per replica."""
    s0 = specs[0]
    bc0 = {"x": s0["bc"][0], "y": s0["bc"][1], "z": s0["bc"][2]}
    m.init(dim=s0["dim"], cells=s0["cells"], cutoff=s0["cutoff"], dt=s0["dt"], bc=bc0, stream=stream)
    u = m.universe
    types = [type(f"T{k}", (m.Particle,), {"mass": ms, "radius": rad, "dynamics": dyn})
             for k, (ms, rad, dyn) in enumerate(s0["types"])]
    for r, sc in enumerate(specs):
        rep = 0 if r == 0 else u.add_replica(sc["dim"], sc["cells"],
                                             bc={"x": sc["bc"][0], "y": sc["bc"][1], "z": sc["bc"][2]})
        for (kind, params, ti, tj) in sc["pots"]:
            u.bind(make_potential(kind, params), types[ti], types[tj], replica=rep)
        u._add_particles(np.asarray(sc["x"]), np.asarray(sc["v"], dtype=np.float32),
                         np.asarray(sc["t"], dtype=np.int32), rep)
    return u


def adjoint_spec(n=32768, seed=7, density=0.8, cut=2.5, dt=0.01, a=5.0, r0=1.0, gamma=1.0, sigma=1.0, jitter=0.15):
    """Two-type Morse mixture (parameters drawn as the cell-sorting replicas') plus
    a DPD thermostat summed on every type pair (alpha 0, gamma, sigma; kT =
    sigma^2 / (2 gamma)), Newtonian, mass 1, periodic cube at the given density.
    Positions: a jittered simple-cubic lattice of k^3 >= n sites, first n kept."""
    rng = np.random.default_rng(seed)
    k = int(np.ceil(n ** (1.0 / 3.0) - 1e-9))
    L = (n / density) ** (1.0 / 3.0)
    sp = L / k
    g = (np.arange(k) + 0.5) * sp
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:n]
    x = x + rng.uniform(-jitter, jitter, size=x.shape) * sp
    x = np.mod(x, L)
    x = np.minimum(x, L * (1 - 1e-6)).astype(np.float32).astype(np.float64)
    t = np.zeros(n, dtype=np.int32)
    t[rng.permutation(n)[: n // 2]] = 1
    kT = sigma * sigma / (2 * gamma)
    v = rng.normal(0, np.sqrt(kT), size=(n, 3))
    v -= v.mean(axis=0)
    dAA, dBB = rng.uniform(0.2, 1.0, size=2)
    dAB = rng.uniform(0.05, 0.5)
    cells = max(3, int(L // cut))
    morse = {(0, 0): [float(dAA), a, r0, 1e-4, cut, 1e-3], (0, 1): [float(dAB), a, r0, 1e-4, cut, 1e-3],
             (1, 1): [float(dBB), a, r0, 1e-4, cut, 1e-3]}
    return dict(dim=[L, L, L], cells=[cells] * 3, cutoff=cut, dt=dt, bc=("periodic",) * 3,
                types=[(1.0, 1.0, m.Newtonian), (1.0, 1.0, m.Newtonian)], morse=morse,
                dpd=[0.0, float(gamma), float(sigma), cut, 0.0], x=x, v=v.astype(np.float32), t=t)


def rdf_target(nbins=64, rmax=2.5, seed=11):
    """A seeded smooth target for the A-B radial distribution: 1 plus a few
    random sine modes, damped near r = 0."""
    rng = np.random.default_rng(seed)
    c = (np.arange(nbins) + 0.5) * rmax / nbins
    g = 1.0 + sum(rng.normal(0, 0.3) * np.sin((k + 1) * np.pi * c / rmax) for k in range(4))
    return np.clip(g, 0.0, None) * (1 - np.exp(-(c / 0.9) ** 8))


def build_adjoint(spec, stream=None):
    """The adjoint workload in the engine (Philox DPD stream); returns the
    universe and the ten differentiated parameters: Morse (d, a, r0) of AA, AB,
    BB and the DPD gamma shared by the three pairs."""
    from . import adjoint as A
    bc = {"x": spec["bc"][0], "y": spec["bc"][1], "z": spec["bc"][2]}
    m.init(dim=spec["dim"], cells=spec["cells"], cutoff=spec["cutoff"], dt=spec["dt"], bc=bc, rng="philox",
           stream=stream)
    types = [type(f"T{k}", (m.Particle,), {"mass": ms, "radius": rad, "dynamics": dyn})
             for k, (ms, rad, dyn) in enumerate(spec["types"])]
    u = m.universe
    slots, dpds = [], []
    for (ti, tj), q in spec["morse"].items():
        mp = m.Potential.morse(*q)
        dp = m.Potential.dpd(*spec["dpd"][:4], shifted=bool(spec["dpd"][4]))
        u.bind(mp + dp, types[ti], types[tj])
        slots += [[(mp, 0)], [(mp, 1)], [(mp, 2)]]
        dpds.append((dp, 1))
    slots.append(dpds)
    u._add_particles(np.asarray(spec["x"]), np.asarray(spec["v"], dtype=np.float32), np.asarray(spec["t"], dtype=np.int32))
    return u, A.Parameters(u, slots)


def bonded_block(nx=32, spacing=0.51, r0=0.5, k=20.0, d=0.05, a=6.0, margin=3.0, seed=17, noise=0.005, dt=0.002):
    """A simple-cubic block of nx^3 particles with harmonic bonds to the six nearest
    neighbours (k, r0; the block starts at `spacing`, stretched when spacing > r0) and a weak
    form of the lattice's Morse nonbonded term (d, a, r0 = 0.5, radius 0.5; its table ends at
    r = 0.95, between the third and fourth neighbour shells), overdamped, in the middle of a
    periodic box with `margin` of free space on each side. dt keeps overdamped Euler inside
    its stability limit dt 8 (2k + V''_Morse) < 2. Returns a spec dict (x, bonds, potentials'
    construction parameters, box)."""
    rng = np.random.default_rng(seed)
    L = nx * spacing + 2 * margin
    g = (np.arange(nx) - (nx - 1) / 2) * spacing + L / 2
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = (x + rng.normal(0, noise, size=x.shape)).astype(np.float32).astype(np.float64)
    idx = np.arange(len(x)).reshape(nx, nx, nx)
    bi, bj = [], []
    for ax in range(3):
        sa, sb = [slice(None)] * 3, [slice(None)] * 3
        sa[ax], sb[ax] = slice(0, nx - 1), slice(1, nx)
        bi.append(idx[tuple(sa)].ravel())
        bj.append(idx[tuple(sb)].ravel())
    cut = 1.0
    cells = int(L // cut)
    return dict(dim=[L, L, L], cells=[cells] * 3, cutoff=cut, dt=dt, bc=("periodic",) * 3, x=x,
                t=np.zeros(len(x), dtype=np.int32), bi=np.concatenate(bi).astype(np.int32),
                bj=np.concatenate(bj).astype(np.int32), morse=(d, a, 0.5, 1e-4, 1.45, 1e-3),
                harmonic=(k, r0, 0.1, 1.2, 0.009), radius=0.5)


def build_bonded_adjoint(spec, stream=None):
    """The bonded block in the engine; returns the universe and the four differentiated
    parameters: harmonic k and r0 of the bonds, Morse d and a."""
    from . import adjoint as A
    bc = {"x": spec["bc"][0], "y": spec["bc"][1], "z": spec["bc"][2]}
    m.init(dim=spec["dim"], cells=spec["cells"], cutoff=spec["cutoff"], dt=spec["dt"], bc=bc, stream=stream)
    Tp = type("Bead", (m.Particle,), {"mass": 1.0, "radius": spec["radius"], "dynamics": m.Overdamped})
    u = m.universe
    mp = m.Potential.morse(*spec["morse"])
    m.bind(mp, Tp, Tp)
    hp = m.Potential.harmonic(*spec["harmonic"])
    x = np.asarray(spec["x"])
    u._add_particles(x, np.zeros_like(x, dtype=np.float32), np.asarray(spec["t"], dtype=np.int32))
    u._add_bonds(hp, spec["bi"], spec["bj"], 1e30)
    return u, A.Parameters(u, [[(hp, 0)], [(hp, 1)], [(mp, 0)], [(mp, 1)]])
