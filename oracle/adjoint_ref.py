"""FP64 CPU reference of the adjoint workload.

TEST INFRASTRUCTURE ONLY: tests/ use it to check the engine's adjoint gradients;
the product never imports it.

A small-N restatement of the forward model the adjoint differentiates, in FP64:
pair forces by brute force over minimum-image pairs within the cutoff, with
  - table potentials evaluated on the engine's table coefficients with the
    reference's potential_eval_ex semantics (potential_eval.hpp:106-161:
    radius shift, a-clamp, quadratic interval map, Horner in x), and
  - the DPD force of dpd_eval.hpp:21-69 with the random term times a Philox
    draw xi keyed on (step, lower id, higher id), the stream the engine's
    Philox mode uses (Philox4x32-10, Salmon et al., SC'11),
as a sum of two terms per type pair; bonds with bond_eval's table semantics
(bond.cpp:99-312: length clamp, break test on f = V'(r)/r); forward Euler with
the speed clamp of engine_advance.cpp:164-173 or its overdamped form with the
step clamp (:174-182); and the Gaussian-smoothed A-B radial distribution loss.
Central finite differences of this model, with tables re-fitted on their frozen
nodes at theta +- h, are the reference gradient.
"""
import numpy as np

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
KEY_XI = (0x44504431, 0x58495F31)
MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 on arrays of uint64 holding 32-bit words."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint64) & MASK32 for c in (c0, c1, c2, c3))
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0 = np.uint64(M0) * c0
        p1 = np.uint64(M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK32, lo1, (hi0 ^ c3 ^ k1) & MASK32, lo0
        k0 = (k0 + np.uint64(W0)) & MASK32
        k1 = (k1 + np.uint64(W1)) & MASK32
    return c0, c1, c2, c3


def pair_xi(step, lo, hi):
    """Zero-mean unit-variance DPD random number of the pairs (lo, hi) at a step,
    in the engine's float32 arithmetic."""
    step = int(step)
    r0, _, _, _ = philox4x32(lo, hi, np.full_like(np.asarray(lo, dtype=np.uint64), step & 0xFFFFFFFF),
                             np.full_like(np.asarray(lo, dtype=np.uint64), step >> 32), *KEY_XI)
    u = ((r0 >> np.uint64(8)).astype(np.float32) + np.float32(0.5)) * np.float32(1.0 / 16777216.0)
    return (np.float32(1.7320508075688772) * (np.float32(2.0) * u - np.float32(1.0))).astype(np.float64)


class Table:
    """A table potential: coefficients (n+1)*8 floats, alpha[3], a, b, flags, r0_plusone."""

    def __init__(self, coef, alpha, a, b, n, flags, r0_plusone):
        # r0_plusone may be given in FP64 (construction r0 + 1) rather than the
        # engine's float, so that differences in r0 are not rounded away
        self.c = np.asarray(coef, dtype=np.float64).reshape(-1, 8)
        self.alpha = [float(v) for v in alpha[:3]]
        self.a, self.b, self.n = float(a), float(b), int(n)
        self.flags, self.r0p1 = int(flags), float(r0_plusone)

    def force_over_r(self, r, ri, rj):
        """f(r) with F_i = -f (x_i - x_j); 0 where the table has no value."""
        ro = np.maximum(r, np.finfo(np.float32).eps)
        rr = np.maximum(r, self.a)
        if self.flags & (1 << 11):
            s = rr / (ri + rj)
        elif self.flags & (1 << 12):
            s = rr - (ri + rj) + self.r0p1
        else:
            s = rr
        t = self.alpha[0] + s * (self.alpha[1] + s * self.alpha[2])
        ind = np.maximum(0.0, t).astype(np.int64)
        ok = (s <= self.b) & (ind <= self.n)
        ind = np.minimum(ind, self.n)
        c = self.c[ind]
        x = (s - c[:, 0]) * c[:, 1]
        ee = c[:, 2] * x + c[:, 3]
        eff = c[:, 2].copy()
        for k in range(4, 8):
            eff = eff * x + ee
            ee = ee * x + c[:, k]
        return np.where(ok, eff * c[:, 1] / ro, 0.0)

    def bond_force_over_r(self, r):
        """potential_eval semantics of a bond (bond.cpp:174-178, potential_eval.hpp:67-104):
        the length clamped to [a, b], no radius shift, the interval index clamped to n;
        returns f with F_i = -f (x_i - x_j)."""
        rc = np.clip(r, self.a, self.b)
        t = self.alpha[0] + rc * (self.alpha[1] + rc * self.alpha[2])
        ind = np.minimum(np.maximum(0.0, t).astype(np.int64), self.n)
        c = self.c[ind]
        x = (rc - c[:, 0]) * c[:, 1]
        ee = c[:, 2] * x + c[:, 3]
        eff = c[:, 2].copy()
        for k in range(4, 8):
            eff = eff * x + ee
            ee = ee * x + c[:, k]
        return eff * c[:, 1] / rc


class Bonds:
    """Harmonic/table bonds (i[k], j[k]) with one table, per-bond dissociation energies
    and active flags; a bond whose f = V'(r)/r reaches its dissociation energy is
    destroyed before it acts (bond.cpp:227-242), and stays destroyed."""

    def __init__(self, i, j, table, dissociation, active=None):
        self.i, self.j = np.asarray(i, dtype=np.int64), np.asarray(j, dtype=np.int64)
        self.table = table
        self.dissociation = np.broadcast_to(np.asarray(dissociation, dtype=np.float64), self.i.shape)
        self.active = np.ones(len(self.i), dtype=bool) if active is None else np.asarray(active, dtype=bool).copy()

    def forces(self, x, box):
        d = x[self.i] - x[self.j]
        d -= box * np.rint(d / box)
        r = np.sqrt((d * d).sum(1))
        f = self.table.bond_force_over_r(r)
        self.active &= ~(f >= self.dissociation)
        fi = np.where(self.active[:, None], -f[:, None] * d, 0.0)
        out = np.zeros_like(x)
        np.add.at(out, self.i, fi)
        np.add.at(out, self.j, -fi)
        return out


class Dpd:
    def __init__(self, alpha, gamma, sigma, cutoff, delta):
        self.alpha, self.gamma, self.sigma, self.cutoff, self.delta = map(float, (alpha, gamma, sigma, cutoff, delta))


def forces(x, v, types, ids, box, radius, terms, cutoff, step, philox=True):
    """Pair forces (N, 3) in FP64. terms[(ti, tj)] = list of Table / Dpd (ti <= tj)."""
    n = len(x)
    ii, jj = np.triu_indices(n, 1)
    d = x[ii] - x[jj]
    d -= box * np.rint(d / box)
    r2 = (d * d).sum(1)
    keep = r2 <= np.float32(cutoff) ** 2
    ii, jj, d, r2 = ii[keep], jj[keep], d[keep], r2[keep]
    r = np.sqrt(r2)
    f = np.zeros((n, 3))
    ti, tj = types[ii], types[jj]
    for (a, b), lst in terms.items():
        sel = ((ti == a) & (tj == b)) | ((ti == b) & (tj == a))
        if not sel.any():
            continue
        i, j, dd, rr = ii[sel], jj[sel], d[sel], r[sel]
        ri, rj = radius[types[i]], radius[types[j]]
        for term in lst:
            if isinstance(term, Table):
                fo = term.force_over_r(rr, ri, rj)
                fi = -fo[:, None] * dd
            else:
                inside = rr <= term.cutoff
                e = dd / rr[:, None]
                vij = v[i] - v[j]
                sv = (e * vij).sum(1)
                om = 1.0 - rr / term.cutoff
                lo, hi = np.minimum(ids[i], ids[j]), np.maximum(ids[i], ids[j])
                xi = pair_xi(step, lo.astype(np.uint64), hi.astype(np.uint64)) if philox else 1.0
                h = term.alpha * om - term.gamma * om * om * sv + term.sigma * om * xi * term.delta
                fi = np.where(inside[:, None], h[:, None] * e, 0.0)
            np.add.at(f, i, fi)
            np.add.at(f, j, -fi)
    return f


def run(x0, v0, types, ids, box, mass, radius, terms, cutoff, dt, nsteps, step0, maxv, philox=True, body=None,
        bonds=None, overdamped=False, maxx=None):
    """FP64 forward Euler (engine_advance.cpp:164-182); returns the final positions
    (unwrapped: minimum image is applied inside the force pass). bonds: a Bonds set
    (its flags change as bonds break). overdamped: x += clamp(dt f imass, maxx)."""
    x = np.array(x0, dtype=np.float64)
    v = np.array(v0, dtype=np.float64)
    imass = 1.0 / mass[types]
    for s in range(nsteps):
        f = forces(x, v, types, ids, box, radius, terms, cutoff, step0 + s, philox)
        if body is not None:
            f = f + body[types]
        if bonds is not None:
            f = f + bonds.forces(x, box)
        if overdamped:
            x = x + np.clip(dt * f * imass[:, None], -maxx, maxx)
            continue
        v = v + dt * f * imass[:, None]
        v = np.clip(v, -maxv, maxv)
        x = x + dt * v
    return x


def run_velocities(x0, v0, types, ids, box, mass, radius, terms, cutoff, dt, nsteps, step0, maxv, every=1,
                   philox=True):
    """As run(), returning the velocities every `every` steps (including step 0)."""
    x = np.array(x0, dtype=np.float64)
    v = np.array(v0, dtype=np.float64)
    imass = 1.0 / mass[types]
    out = [v.copy()]
    for s in range(nsteps):
        f = forces(x, v, types, ids, box, radius, terms, cutoff, step0 + s, philox)
        v = np.clip(v + dt * f * imass[:, None], -maxv, maxv)
        x = x + dt * v
        if (s + 1) % every == 0:
            out.append(v.copy())
    return np.array(out)


def rdf(x, types, box, ta, tb, nbins, rmax, sigma):
    """The smoothed A-B radial distribution of the engine's mxg_rdf, in FP64
    (Gaussian minus its value at the 4 sigma cut)."""
    A = np.where(types == ta)[0]
    B = np.where(types == tb)[0]
    dr = rmax / nbins
    c = (np.arange(nbins) + 0.5) * dr
    d = x[A][:, None, :] - x[B][None, :, :]
    d -= box * np.rint(d / box)
    r = np.sqrt((d * d).sum(-1)).ravel()
    r = r[(r > 0) & (r < nbins * dr + 4 * sigma)]
    t = r[:, None] - c[None, :]
    k = (np.exp(-0.5 * (t / sigma) ** 2) - np.exp(-8.0)) * (0.3989422804014327 / sigma)
    k = np.where(np.abs(t) <= 4 * sigma, k, 0.0)
    H = k.sum(0)
    V = float(np.prod(box))
    return H * V / (len(A) * len(B)) / (4 * np.pi * c ** 2)


def rdf_loss(x, types, box, ta, tb, target, nbins=64, rmax=2.5, sigma=None):
    sigma = rmax / nbins if sigma is None else sigma
    g = rdf(x, types, box, ta, tb, nbins, rmax, sigma)
    return float(((g - target) ** 2).sum())
