"""Adjoint gradients through harmonic bonds (bond_eval's VJP) against FP64 central
finite differences of the same tabulated model (oracle/adjoint_ref.py).

Workload: a 6x6x6 simple-cubic block (spacing 0.51, jittered: the bonds start
under tension) in the middle of a periodic box of 6, one overdamped type with a
weak form of the lattice's Morse nonbonded term (d = 0.05, a = 6, r0 = 0.5,
radius 0.5, table up to r = 0.95), harmonic bonds to the six nearest neighbours
(k = 20, r0 = 0.5, never breaking), plus a second group of bonds with the same
potential that break in the first step (second neighbours, about twice r0; the
dissociation energy 2 is compared with f = V'(r)/r, as bond.cpp:230 does) and a
third group switched off before the run. dt = 0.002, 10 steps, a snapshot every
4. Loss: a seeded linear functional of the final positions. (The lattice
workload's k = 200 with dt = 0.005 is beyond the stability limit of overdamped
Euler, dt 8 (2k + V''_Morse) < 2, while its bonds hold; there every bond breaks
in the first steps.)

Parameters: harmonic k and r0 (shared by all bond groups), Morse d and a. Every
pair distance and bond length stays away from the table edges over the run
(checked on the FP64 trajectory), so the loss is smooth in theta and x0 at the
finite-difference step."""
import ctypes

import numpy as np
import pytest
import torch

import mechanica_b200 as m
from mechanica_b200 import adjoint as A
from mechanica_b200._native import lib
from oracle import adjoint_ref as R

pytestmark = pytest.mark.gpu

NX, SP, L, CUT, DT, T, K = 6, 0.51, 6.0, 1.0, 0.002, 10, 4
MORSE = (0.05, 6.0, 0.5, 1e-4, 1.45, 1e-3)  # s = r - 2 radius + r0 + 1 = r + 0.5 <= 1.45: r <= 0.95
HARM = (20.0, 0.5, 0.1, 1.2, 0.009)
GRAD_TOL = 1e-3


def _system(seed=17):
    rng = np.random.default_rng(seed)
    g = (np.arange(NX) - (NX - 1) / 2) * SP + L / 2
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = (x + rng.normal(0, 0.005, size=x.shape)).astype(np.float32).astype(np.float64)
    n = len(x)
    idx = np.arange(n).reshape(NX, NX, NX)
    bi, bj = [], []
    for ax in range(3):
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[ax], b[ax] = slice(0, NX - 1), slice(1, NX)
        bi.append(idx[tuple(a)].ravel())
        bj.append(idx[tuple(b)].ravel())
    bi, bj = np.concatenate(bi), np.concatenate(bj)
    # bonds that break in the first step: second neighbours along x, length ~1.0
    # (f = 2k (r - r0) / r ~ 200 >= 2)
    ci, cj = idx[0:NX - 2, ::2, ::2].ravel(), idx[2:NX, ::2, ::2].ravel()
    # bonds switched off before the run: face diagonals in the bottom layer (length ~0.71)
    oi, oj = idx[0:NX - 1, 0:NX - 1, 0].ravel(), idx[1:NX, 1:NX, 0].ravel()
    c = rng.normal(size=(n, 3))
    return x, (bi, bj), (ci, cj), (oi, oj), c


def _build(x, groups, theta):
    m.init(dim=[L, L, L], cells=[6, 6, 6], cutoff=CUT, dt=DT, bc={"x": "periodic", "y": "periodic", "z": "periodic"},
           stream=torch.cuda.current_stream().cuda_stream)
    Tp = type("Bead", (m.Particle,), {"mass": 1.0, "radius": 0.5, "dynamics": m.Overdamped})
    u = m.universe
    mp = m.Potential.morse(*MORSE)
    m.bind(mp, Tp, Tp)
    hp = m.Potential.harmonic(*HARM)
    u._add_particles(x, np.zeros_like(x, dtype=np.float32), np.zeros(len(x), dtype=np.int32))
    (bi, bj), (ci, cj), (oi, oj) = groups
    u._add_bonds(hp, bi, bj, 1e30)
    u._add_bonds(hp, ci, cj, 2.0)
    u._add_bonds(hp, oi, oj, 1e30)
    P = A.Parameters(u, [[(hp, 0)], [(hp, 1)], [(mp, 0)], [(mp, 1)]])
    P.apply(theta)
    nb = len(bi) + len(ci) + len(oi)
    flags = np.ones(nb, dtype=np.uint32)
    flags[len(bi) + len(ci):] = 0
    u.set_bond_flags(flags)
    return u, P


def _tables(theta):
    """FP64 tables at theta, re-fitted on the frozen nodes of the construction fits."""
    out = []
    for q0, (k0, k1) in ((HARM, (0, 1)), (MORSE, (2, 3))):
        p = (m.Potential.harmonic if q0 is HARM else m.Potential.morse)(*q0)
        q = list(q0)
        q[0], q[1] = theta[k0], theta[k1]
        p.refit(q)
        info = p._info()
        coef = np.zeros((info["n"] + 1) * 8, dtype=np.float64)
        lib().mxg_potential_coeffs64(p._h, coef.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(coef))
        r0p1 = q[2] + 1.0 if q0 is MORSE else 0.0
        out.append(R.Table(coef, info["alpha"], info["a"], info["b"], info["n"], info["flags"], r0p1))
    return out


def _reference(x0, groups, theta, record=None):
    harm, morse = _tables(theta)
    (bi, bj), (ci, cj), (oi, oj) = groups
    i = np.concatenate([bi, ci, oi])
    j = np.concatenate([bj, cj, oj])
    diss = np.concatenate([np.full(len(bi), 1e30), np.full(len(ci), 2.0), np.full(len(oi), 1e30)])
    active = np.concatenate([np.ones(len(bi) + len(ci), bool), np.zeros(len(oi), bool)])
    bonds = R.Bonds(i, j, harm, diss, active)
    n = len(x0)
    box = np.array([L, L, L])
    maxx = float(np.float32(np.float32(L / 6) * np.float32(0.05)))
    xs = [np.array(x0)]
    x = np.array(x0, dtype=np.float64)
    for s in range(T):
        x = R.run(x, np.zeros((n, 3)), np.zeros(n, np.int64), np.arange(n), box, np.array([1.0]), np.array([0.5]),
                  {(0, 0): [morse]}, CUT, DT, 1, s, 1e30, philox=False, bonds=bonds, overdamped=True, maxx=maxx)
        xs.append(x)
    if record is not None:
        record.extend([xs, bonds])
    return x


def _loss_ref(x0, groups, theta, c):
    return float((_reference(x0, groups, theta) * c).sum())


def test_bond_adjoint_matches_fp64_finite_differences():
    x0, bonds, broken, off, c = _system()
    groups = (bonds, broken, off)
    theta0 = np.array([HARM[0], HARM[1], MORSE[0], MORSE[1]], dtype=np.float64)
    # preconditions on the FP64 trajectory: every pair distance and bond length away from
    # the table edges, the breaking group broken in the first step, no other bond broken
    rec = []
    _reference(x0, groups, theta0, rec)
    xs, bset = rec
    nb, nc = len(bonds[0]), len(broken[0])
    assert bset.active[:nb].all() and not bset.active[nb:].any()
    for x in xs:
        d = x[:, None, :] - x[None, :, :]
        r = np.sqrt((d * d).sum(-1))[np.triu_indices(len(x), 1)]
        assert np.abs(r - 0.95).min() > 5e-3
        bl = np.linalg.norm(x[bonds[0]] - x[bonds[1]], axis=1)
        assert bl.min() > 0.1 + 5e-3 and bl.max() < 1.2 - 5e-3
    u, P = _build(x0, groups, theta0)
    sim = A.Simulation(u, P, nsteps=T, checkpoint_every=K, step0=0)
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    xt = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    vt = torch.zeros_like(xt, requires_grad=True)
    x4 = A.trajectory(theta, xt, vt, sim)
    flags = u.bond_flags()
    assert flags[:nb].all() and not flags[nb:].any()
    C = torch.tensor(c, dtype=torch.float64, device="cuda")
    loss = (x4[:, :3].double() * C).sum()
    loss.backward()
    ref = _loss_ref(x0, groups, theta0, c)
    assert abs(loss.item() - ref) <= 1e-5 * abs(ref) + 1e-4, (loss.item(), ref)
    h = 1e-5
    fd = np.zeros(4)
    for k in range(4):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h * max(1.0, abs(theta0[k]))
        tm[k] -= h * max(1.0, abs(theta0[k]))
        fd[k] = (_loss_ref(x0, groups, tp, c) - _loss_ref(x0, groups, tm, c)) / (tp[k] - tm[k])
    adj = theta.grad.numpy()
    assert np.all(np.abs(adj - fd) <= GRAD_TOL * np.abs(fd) + 1e-6 * np.abs(fd).max()), (adj, fd)
    gx = xt.grad.numpy()
    for (i, kk) in [(0, 0), (37, 1), (108, 2), (215, 0), (150, 1)]:
        xp, xm = x0.copy(), x0.copy()
        xp[i, kk] += h
        xm[i, kk] -= h
        fdx = (_loss_ref(xp, groups, theta0, c) - _loss_ref(xm, groups, theta0, c)) / (2 * h)
        assert abs(gx[i, kk] - fdx) <= GRAD_TOL * abs(fdx) + 1e-3 * np.abs(gx).max(), (i, kk, gx[i, kk], fdx)
    u.close()


def test_bond_adjoint_without_bonds_acting_is_the_pair_adjoint():
    """All bonds switched off: the VJP equals the one of the same system without bonds."""
    x0, bonds, broken, off, c = _system(seed=23)
    theta0 = np.array([HARM[0], HARM[1], MORSE[0], MORSE[1]], dtype=np.float64)
    grads = []
    for with_bonds in (True, False):
        groups = (bonds, broken, off) if with_bonds else ((bonds[0][:0], bonds[1][:0]),) * 3
        u, P = _build(x0, groups, theta0)
        if with_bonds:
            u.set_bond_flags(np.zeros(len(u.bond_flags()), dtype=np.uint32))
        sim = A.Simulation(u, P, nsteps=4, checkpoint_every=2, step0=0)
        theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
        xt = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
        x4 = A.trajectory(theta, xt, torch.zeros_like(xt), sim)
        (x4[:, :3].double() * torch.tensor(c, dtype=torch.float64, device="cuda")).sum().backward()
        grads.append((theta.grad.numpy().copy(), xt.grad.numpy().copy()))
        u.close()
    assert np.array_equal(grads[0][1], grads[1][1])
    assert grads[0][0][0] == 0.0 and grads[0][0][1] == 0.0
    assert np.array_equal(grads[0][0][2:], grads[1][0][2:])
