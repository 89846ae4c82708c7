"""Python wrapper of oracle tier B (oracle/liboracle.so, built from oracle.cpp).

TEST INFRASTRUCTURE ONLY. Computes the nonbonded forces and energy of a
configuration in FP32 (reference operation order) or FP64 on the same FP32
table coefficients. Tables come from the reference's own table builder
(oracle/_ref/libmxref.so) when it is built, else from the committed golden
tables.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class _OrcInput(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("xrel", ctypes.c_void_p), ("vel", ctypes.c_void_p), ("cell", ctypes.c_void_p),
        ("type", ctypes.c_void_p), ("ncells", ctypes.c_int), ("cell_origin", ctypes.c_void_p),
        ("dim", ctypes.c_double * 3), ("cutoff", ctypes.c_double), ("tasks", ctypes.c_void_p),
        ("ntasks", ctypes.c_int), ("ntypes", ctypes.c_int), ("radius", ctypes.c_void_p),
        ("pot_of_pair", ctypes.c_void_p), ("dpd_of_pair", ctypes.c_void_p), ("npots", ctypes.c_int),
        ("pot_kind", ctypes.c_void_p), ("pot_flags", ctypes.c_void_p), ("pot_n", ctypes.c_void_p),
        ("pot_alpha", ctypes.c_void_p), ("pot_abr", ctypes.c_void_p), ("pot_coef_off", ctypes.c_void_p),
        ("coef", ctypes.c_void_p), ("dpd", ctypes.c_void_p), ("body", ctypes.c_void_p),
        ("cdim", ctypes.c_int * 3), ("pruning", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import subprocess
            subprocess.run(["make", "-C", HERE, "restatement"], check=True, capture_output=True)
        _lib = ctypes.CDLL(LIB)
        _lib.orc_nonbond.argtypes = [ctypes.c_int, ctypes.POINTER(_OrcInput), ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
        _lib.orc_nonbond.restype = ctypes.c_int
        _lib.orc_nonbond_virial.argtypes = [ctypes.c_int, ctypes.POINTER(_OrcInput), ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.orc_nonbond_virial.restype = ctypes.c_int
    return _lib


def reference_table(kind, params):
    """(info dict, coefficients) from the reference's table builder (in process)."""
    from . import refengine
    L = ctypes.PyDLL(refengine.LIB)
    vp, cd = ctypes.c_void_p, ctypes.c_double
    if kind == "dpd":
        L.mxref_potential_dpd.restype = vp
        L.mxref_potential_dpd.argtypes = [cd, cd, cd, cd, ctypes.c_int]
        p = L.mxref_potential_dpd(*[float(q) for q in params[:4]], int(params[4]) if len(params) > 4 else 0)
    else:
        fn = getattr(L, f"mxref_potential_{kind}")
        fn.restype = vp
        if kind == "harmonic_dihedral":  # (k, n, delta, tol) with an int multiplicity
            fn.argtypes = [cd, ctypes.c_int, cd, cd]
            p = fn(float(params[0]), int(params[1]), float(params[2]), float(params[3]))
        else:
            fn.argtypes = [cd] * len(params)
            p = fn(*[float(q) for q in params])
    if not p:
        return None, None  # the reference's potential_init failed
    n = ctypes.c_int()
    a4 = (ctypes.c_float * 4)()
    a, b, r0 = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    fl, k = ctypes.c_uint(), ctypes.c_int()
    L.mxref_potential_info(vp(p), ctypes.byref(n), a4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(fl),
                           ctypes.byref(r0), ctypes.byref(k))
    coef = np.zeros(max(1, (n.value + 1) * 8), dtype=np.float32)
    if k.value == 0:
        L.mxref_potential_coeffs(vp(p), coef.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), coef.size)
    return dict(kind=k.value, flags=fl.value, n=n.value, alpha=np.array(a4[:3], dtype=np.float32), a=a.value,
                b=b.value, r0p1=r0.value), coef


def cell_origins(dim, cdim, origin=(0.0, 0.0, 0.0)):
    h = np.asarray(dim, dtype=np.float64) / np.asarray(cdim)
    out = np.zeros((int(np.prod(cdim)), 3))
    c = 0
    for i in range(cdim[0]):
        for j in range(cdim[1]):
            for k in range(cdim[2]):
                out[c] = (origin[0] + i * h[0], origin[1] + j * h[1], origin[2] + k * h[2])
                c += 1
    return out


def pairlist(ids, xrel, cell, origins, types, cutoff, type_pairs=None):
    """make_pairlist (src/mdcore/src/bond.cpp:892-942) restated: for list
    entries a = 1..n-1 and b = 0..a-1, global positions float(x_rel + cell
    origin), r2 = (dx*dx + dy*dy) + dz*dz in FP32 against float(cutoff)^2, type
    pair accepted by pair_check (bond.cpp:1134-1152). Returns (ids[a], ids[b])
    in the double loop's order."""
    f32 = np.float32
    g = (xrel.astype(np.float64) + origins[cell]).astype(f32)[ids]
    t = np.asarray(types)[ids]
    c2 = f32(cutoff) * f32(cutoff)
    allowed = None
    if type_pairs:
        allowed = {(int(a), int(b)) for a, b in type_pairs} | {(int(b), int(a)) for a, b in type_pairs}
    fi, fj = [], []
    for a in range(1, len(ids)):
        d = g[a] - g[:a]
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        ok = r2 <= c2
        if allowed is not None:
            ok &= np.array([(int(t[a]), int(tb)) in allowed for tb in t[:a]], dtype=bool)
        b = np.flatnonzero(ok)
        fi.extend([ids[a]] * len(b))
        fj.extend(ids[b].tolist())
    return np.array(fi, dtype=np.int32), np.array(fj, dtype=np.int32)


def flux_step(x, t, L, cutoff, dt, values, fluxes, konst, moved):
    """One forward-Euler species update under fluxes, in FP64 (flux_eval_ex,
    src/mdcore/src/flux_eval.hpp:33-84; MxFluxes_Integrate, src/mdcore/src/
    Flux.cpp:261-285): for every pair within the cutoff (minimum image in a
    periodic box L) and every flux entry (kind, type a, type b, species a,
    species b, k, decay, target) of its type pair, q = (1 - r/cutoff)^2 times
    k (s_a - s_b) (Fick), max(k (s_a - target), 0) (secrete) or
    max(k (target - s_b) s_a, 0) (uptake); rate_a -= q + decay/2 s_a,
    rate_b += q - decay/2 s_b. values += dt * rate where konst is 0 and the
    particle did not change cells (moved), else the values stay. Pairs of one
    type take the lower id as a, which matters only for secretion and uptake
    within one type."""
    x = np.asarray(x, dtype=np.float64)
    sv = np.asarray(values, dtype=np.float64)
    rate = np.zeros_like(sv)
    n = len(t)
    for a in range(n - 1):
        d = x[a] - x[a + 1:]
        d -= L * np.round(d / L)
        r2 = (d ** 2).sum(1)
        for bb in np.flatnonzero(r2 <= cutoff * cutoff):
            b = a + 1 + bb
            w = (1 - np.sqrt(r2[bb]) / cutoff) ** 2
            for (kind, ta, tb, ia, ib, k, dec, tgt) in fluxes:
                if sorted((t[a], t[b])) != sorted((ta, tb)):
                    continue
                if ta == tb:
                    pi, pj = a, b
                else:
                    pi, pj = (a, b) if t[a] == ta else (b, a)
                si, sj = sv[pi, ia], sv[pj, ib]
                if kind == 0:
                    g = k * (si - sj)
                elif kind == 1:
                    g = max(k * (si - tgt), 0.0)
                else:
                    g = max(k * (tgt - sj) * si, 0.0)
                rate[pi, ia] += -w * g - dec / 2 * si
                rate[pj, ib] += w * g - dec / 2 * sj
    out = sv + dt * rate * (1 - np.asarray(konst))
    out[np.asarray(moved)] = sv[np.asarray(moved)]
    return out


def group_metrics(x, mass, fp32=False):
    """Particle-group metrics as the reference computes them (src/mdcore/src/metrics.cpp):
    centre of mass (:366-389), centroid (:391-412), radius of gyration (:330-364: the
    square root of the SUM of the distances to the centroid) and moment of inertia about
    the centre of mass (:414-466: diagonal sum m (dy^2 + dz^2) ..., off-diagonal + sum m
    dx dy ...). x: global positions in list order (the reference's p->x[k] + o[k], in
    double); mass: per entry. fp32=True repeats the reference's FP32 running sums in list
    order (Magnum float vectors, `float m`); otherwise every sum is FP64.
    Returns (total mass, com[3], centroid[3], rog, inertia[3x3])."""
    x = np.asarray(x, dtype=np.float64)
    mass = np.asarray(mass, dtype=np.float64)
    n = len(x)
    if not fp32:
        M = mass.sum()
        com = (mass[:, None] * x).sum(axis=0) / M
        cen = x.sum(axis=0) / n
        rog = np.sqrt(np.linalg.norm(cen - x, axis=1).sum())
        d = x - com
        I = np.zeros((3, 3))
        I[0, 0] = ((d[:, 1] ** 2 + d[:, 2] ** 2) * mass).sum()
        I[1, 1] = ((d[:, 0] ** 2 + d[:, 2] ** 2) * mass).sum()
        I[2, 2] = ((d[:, 1] ** 2 + d[:, 0] ** 2) * mass).sum()
        I[0, 1] = I[1, 0] = (d[:, 0] * d[:, 1] * mass).sum()
        I[1, 2] = I[2, 1] = (d[:, 1] * d[:, 2] * mass).sum()
        I[0, 2] = I[2, 0] = (d[:, 0] * d[:, 2] * mass).sum()
        return M, com, cen, float(rog), I
    f = np.float32
    r = [f(0)] * 3
    M = f(0)
    for i in range(n):  # `r[k] += p->mass * (x + o)`: double product, rounded on the float store
        M = f(float(M) + mass[i])
        for k in range(3):
            r[k] = f(float(r[k]) + mass[i] * x[i, k])
    com = np.array([f(r[k] / M) for k in range(3)], dtype=np.float32)
    c = [f(0)] * 3
    for i in range(n):
        for k in range(3):
            c[k] = f(float(c[k]) + x[i, k])
    cen = np.array([f(c[k] / f(n)) for k in range(3)], dtype=np.float32)
    r2 = f(0)
    for i in range(n):
        dx = [f(float(cen[k]) - x[i, k]) for k in range(3)]
        r2 = f(r2 + f(np.sqrt(f(f(dx[0] * dx[0] + dx[1] * dx[1]) + dx[2] * dx[2]))))
    rog = float(np.sqrt(r2))
    I = np.zeros((3, 3), dtype=np.float32)
    for i in range(n):
        d = [f(f(x[i, k]) - com[k]) for k in range(3)]  # pix is a float vector: rounded first
        m = mass[i]
        I[0, 0] = f(float(I[0, 0]) + float(f(d[1] * d[1] + d[2] * d[2])) * m)
        I[1, 1] = f(float(I[1, 1]) + float(f(d[0] * d[0] + d[2] * d[2])) * m)
        I[2, 2] = f(float(I[2, 2]) + float(f(d[1] * d[1] + d[0] * d[0])) * m)
        I[0, 1] = f(float(I[0, 1]) + float(f(d[0] * d[1])) * m)
        I[1, 2] = f(float(I[1, 2]) + float(f(d[1] * d[2])) * m)
        I[0, 2] = f(float(I[0, 2]) + float(f(d[0] * d[2])) * m)
    I[1, 0], I[2, 1], I[2, 0] = I[0, 1], I[1, 2], I[0, 2]
    return float(M), com.astype(np.float64), cen.astype(np.float64), rog, I.astype(np.float64)


def nonbond(scn, xrel, vel, cell, tasks, cdim, precision=64, tables=None, second=None, pruning=0, virial=False):
    """Forces (N,3) float64, energy, counts for a configuration.

    tables: {pot index: (info, coef)} for scn["pots"] order (defaults to the
    reference builder); second: optional list of (kind, params, ti, tj) DPD
    terms summed with the first potential of each pair.
    """
    N = len(scn["t"])
    ntypes = len(scn["types"])
    pots = list(scn["pots"]) + list(second or [])
    infos = []
    coefs = []
    for q, (kind, params, ti, tj) in enumerate(pots):
        if tables is not None and q in tables:
            infos.append(tables[q][0])
            coefs.append(tables[q][1])
        else:
            inf, cf = reference_table(kind, params)
            infos.append(inf)
            coefs.append(cf)
    off = np.cumsum([0] + [len(c) for c in coefs])[:-1].astype(np.int32)
    coef = np.concatenate(coefs).astype(np.float32)
    pot_of_pair = -np.ones(ntypes * ntypes, dtype=np.int32)
    dpd_of_pair = -np.ones(ntypes * ntypes, dtype=np.int32)
    for q, (kind, params, ti, tj) in enumerate(pots):
        tgt = pot_of_pair if q < len(scn["pots"]) else dpd_of_pair
        tgt[ti * ntypes + tj] = q
        tgt[tj * ntypes + ti] = q
    kinds = np.array([i["kind"] for i in infos], dtype=np.int32)
    flags = np.array([i["flags"] for i in infos], dtype=np.uint32)
    ns = np.array([i["n"] for i in infos], dtype=np.int32)
    alpha = np.concatenate([i["alpha"] for i in infos]).astype(np.float32)
    abr = np.array([[i["a"], i["b"], i["r0p1"]] for i in infos], dtype=np.float32).ravel()
    dt = float(scn["dt"])
    dpd = np.zeros(4 * len(pots), dtype=np.float32)
    for q, (kind, params, ti, tj) in enumerate(pots):
        if kind == "dpd":
            dpd[4 * q:4 * q + 3] = np.float32(params[0]), np.float32(params[1]), np.float32(params[2])
            dpd[4 * q + 3] = np.float32(1.0 / np.sqrt(dt))
    radius = np.array([r for (_, r, _) in scn["types"]], dtype=np.float32)
    body = np.zeros(3 * ntypes, dtype=np.float32)
    for (t, fx, fy, fz) in scn.get("forces", []):
        body[3 * t:3 * t + 3] = fx, fy, fz
    tasks = np.ascontiguousarray(tasks, dtype=np.int32)
    origins = cell_origins(scn["dim"], cdim)
    keep = dict(xrel=np.ascontiguousarray(xrel, dtype=np.float32), vel=np.ascontiguousarray(vel, dtype=np.float32),
                cell=np.ascontiguousarray(cell, dtype=np.int32), type=np.ascontiguousarray(scn["t"], dtype=np.int32),
                origins=origins, tasks=tasks, radius=radius, pop=pot_of_pair, dop=dpd_of_pair, kinds=kinds,
                flags=flags, ns=ns, alpha=alpha, abr=abr, off=off, coef=coef, dpd=dpd, body=body)
    inp = _OrcInput()
    inp.N = N
    inp.xrel = keep["xrel"].ctypes.data
    inp.vel = keep["vel"].ctypes.data
    inp.cell = keep["cell"].ctypes.data
    inp.type = keep["type"].ctypes.data
    inp.ncells = len(origins)
    inp.cell_origin = origins.ctypes.data
    for k in range(3):
        inp.dim[k] = float(scn["dim"][k])
    inp.cutoff = float(scn["cutoff"])
    inp.tasks = tasks.ctypes.data
    inp.ntasks = len(tasks)
    inp.ntypes = ntypes
    inp.radius = radius.ctypes.data
    inp.pot_of_pair = pot_of_pair.ctypes.data
    inp.dpd_of_pair = dpd_of_pair.ctypes.data if second else None
    inp.npots = len(pots)
    inp.pot_kind = kinds.ctypes.data
    inp.pot_flags = flags.ctypes.data
    inp.pot_n = ns.ctypes.data
    inp.pot_alpha = alpha.ctypes.data
    inp.pot_abr = abr.ctypes.data
    inp.pot_coef_off = off.ctypes.data
    inp.coef = coef.ctypes.data
    inp.dpd = dpd.ctypes.data
    inp.body = body.ctypes.data
    for k in range(3):
        inp.cdim[k] = int(cdim[k])
    inp.pruning = int(pruning)
    f = np.zeros((N, 3))
    ep = ctypes.c_double()
    counts = np.zeros(3, dtype=np.int64)
    if virial:
        vir = np.zeros(9)
        rc = lib().orc_nonbond_virial(int(precision), ctypes.byref(inp), f.ctypes.data, ctypes.addressof(ep),
                                      counts.ctypes.data, vir.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"orc_nonbond_virial {rc}")
        return f, ep.value, counts, vir.reshape(3, 3)
    rc = lib().orc_nonbond(int(precision), ctypes.byref(inp), f.ctypes.data, ctypes.addressof(ep), counts.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_nonbond {rc}")
    return f, ep.value, counts


def _table_index(info, s):
    """The interval of s as the FP32 code picks it (potential_eval.hpp:83-86: the quadratic
    map in float, truncated, at most n): an integer decision of the tabulated model, so the
    FP64 evaluation uses the same polynomial piece as the FP32 one."""
    f32 = np.float32
    a = np.asarray(info["alpha"], dtype=f32)
    s32 = np.asarray(s, dtype=f32)
    t = a[0] + s32 * (a[1] + s32 * a[2])
    return np.minimum(np.maximum(f32(0), t).astype(np.int64), info["n"])


def _table_poly(coef, ind, s):
    """Value and derivative of the table's interval polynomial at s, in FP64
    (the Horner scheme of potential_eval.hpp:67-104 without its rounding)."""
    c = np.asarray(coef, dtype=np.float64).reshape(-1, 8)[ind]
    x = (s - c[..., 0]) * c[..., 1]
    ee = c[..., 2] * x + c[..., 3]
    eff = c[..., 2].copy()
    for k in range(4, 8):
        eff = eff * x + ee
        ee = ee * x + c[..., k]
    return ee, eff * c[..., 1]


def _min_image(d, dim, periodic):
    d = np.array(d, dtype=np.float64)
    for k in range(3):
        if periodic[k]:
            d[..., k] -= dim[k] * np.round(d[..., k] / dim[k])
    return d


def _cos_grad(u, w):
    """c = u.w / (|u| |w|) and its gradients with respect to u and w."""
    nu, nw = np.linalg.norm(u, axis=-1, keepdims=True), np.linalg.norm(w, axis=-1, keepdims=True)
    c = (u * w).sum(-1, keepdims=True) / (nu * nw)
    return c[..., 0], (w / nw - c * u / nu) / nu, (u / nu - c * w / nw) / nw


def bonded(scn, xabs, bond_flags=None, tables=None, virial=False):
    """FP64 bonded forces (N, 3) and energy of a configuration, in the order of
    engine_bonded_eval (src/mdcore/src/engine_bonded.cpp:1373-1543) on the
    reference builder's FP32 tables:
      exclusions (exclusion.cpp:83-282): the pair's table potential without the
        radius shift taken back for excluded pairs within the cutoff;
      bonds (bond.cpp:99-312): r^2 clamped to [a^2, b^2], F_i = -V'(r)/r d; bond_flags
        (after the pass) select the bonds that acted;
      angles (angle.cpp:92-352): V(cos theta) at the vertex j, cos clamped to [a, b],
        F = -V'(c) dc/dx;
      dihedrals (dihedral.cpp:81-392): V(c), c = -(b1 x b2).(b2 x b3) / (|b1 x b2| |b2 x b3|)
        with b1 = x_i - x_j, b2 = x_k - x_j, b3 = x_l - x_k, clamped to [a, b].
    Positions are global (FP64), pairs by minimum image on periodic axes.
    tables: optional {"bond"/"angle"/"dihedral"/(ti, tj): (info, coef)}.
    virial: also return the terms' virial sum (x_m - x_ref) (x) F_m (bonds and
    exclusions d (x) F_i, angles about the vertex, dihedrals about j)."""
    tables = dict(tables or {})
    x = np.asarray(xabs, dtype=np.float64)
    n = len(x)
    dim = np.asarray(scn["dim"], dtype=np.float64)
    periodic = [b == "periodic" for b in scn["bc"]]
    f = np.zeros((n, 3))
    ep = 0.0
    W = np.zeros((3, 3))

    def vir(r, F):
        W[...] += np.einsum("na,nb->ab", np.atleast_2d(r), np.atleast_2d(F))

    def table(key, kind_params):
        if key not in tables:
            tables[key] = reference_table(*kind_params)
        return tables[key]

    t = np.asarray(scn["t"])
    if "ex_i" in scn and len(scn["ex_i"]):
        pots = {}
        for (kind, params, ti, tj) in scn["pots"]:
            pots[(ti, tj)] = pots[(tj, ti)] = (kind, params)
        cut2 = float(scn["cutoff"]) ** 2
        for i, j in zip(scn["ex_i"], scn["ex_j"]):
            kp = pots.get((int(t[i]), int(t[j])))
            if kp is None or kp[0] == "dpd":
                continue
            d = _min_image(x[i] - x[j], dim, periodic)
            r2 = float(d @ d)
            if r2 > cut2:
                continue
            info, coef = table(("pair",) + tuple(sorted((int(t[i]), int(t[j])))), kp)
            r = np.sqrt(r2)
            e, dv = _table_poly(coef, _table_index(info, r), r)
            f[i] += dv / r * d
            f[j] -= dv / r * d
            ep -= float(e)
            vir(d, dv / r * d)
    if "bi" in scn and len(scn["bi"]):
        info, coef = table("bond", scn["bond_pot"])
        bi, bj = np.asarray(scn["bi"]), np.asarray(scn["bj"])
        act = np.ones(len(bi), bool) if bond_flags is None else (np.asarray(bond_flags) & 1).astype(bool)
        bi, bj = bi[act], bj[act]
        d = _min_image(x[bi] - x[bj], dim, periodic)
        r = np.sqrt(np.clip((d * d).sum(1), info["a"] ** 2, info["b"] ** 2))
        e, dv = _table_poly(coef, _table_index(info, r), r)
        fi = -(dv / r)[:, None] * d
        np.add.at(f, bi, fi)
        np.add.at(f, bj, -fi)
        ep += float(e.sum())
        vir(d, fi)
    if "ai" in scn and len(scn["ai"]):
        info, coef = table("angle", scn["angle_pot"])
        ai, aj, ak = (np.asarray(scn[k]) for k in ("ai", "aj", "ak"))
        rji = _min_image(x[ai] - x[aj], dim, periodic)
        rjk = _min_image(x[ak] - x[aj], dim, periodic)
        c, gi, gk = _cos_grad(rji, rjk)
        cc = np.clip(np.clip(c, -1.0, 1.0), info["a"], info["b"])
        e, dv = _table_poly(coef, _table_index(info, cc), cc)
        wi, wk = dv[:, None] * gi, dv[:, None] * gk
        np.add.at(f, ai, -wi)
        np.add.at(f, ak, -wk)
        np.add.at(f, aj, wi + wk)
        ep += float(e.sum())
        vir(rji, -wi)
        vir(rjk, -wk)
    if "di" in scn and len(scn["di"]):
        info, coef = table("dihedral", scn["dihedral_pot"])
        di, dj, dk, dl = (np.asarray(scn[k]) for k in ("di", "dj", "dk", "dl"))
        b1 = _min_image(x[di] - x[dj], dim, periodic)
        b2 = _min_image(x[dk] - x[dj], dim, periodic)
        b3 = _min_image(x[dl] - x[dk], dim, periodic)
        A, B = np.cross(b1, b2), np.cross(b2, b3)
        c, gA, gB = _cos_grad(A, B)
        c, gA, gB = -c, -gA, -gB
        g1 = np.cross(b2, gA)                        # dc/db1 through A = b1 x b2
        g2 = np.cross(gA, b1) + np.cross(b3, gB)     # dc/db2 through A and B = b2 x b3
        g3 = np.cross(gB, b2)                        # dc/db3 through B
        cc = np.clip(np.clip(c, -1.0, 1.0), info["a"], info["b"])
        e, dv = _table_poly(coef, _table_index(info, cc), cc)
        wi, wj, wl = dv[:, None] * g1, dv[:, None] * (-g1 - g2), dv[:, None] * g3
        np.add.at(f, di, -wi)
        np.add.at(f, dj, -wj)
        np.add.at(f, dl, -wl)
        np.add.at(f, dk, wi + wj + wl)
        ep += float(e.sum())
        vir(b1, -wi)
        vir(b2, wi + wj + wl)
        vir(b2 + b3, -wl)
    if virial:
        return f, ep, W
    return f, ep
