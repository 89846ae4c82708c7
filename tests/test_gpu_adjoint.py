"""Adjoint gradients of a trajectory loss against FP64 central finite
differences of the same tabulated model (oracle/adjoint_ref.py), plus the
pieces they rest on: the summed Morse + DPD pair force against the FP64
restatement, bitwise replay from a state snapshot, and the loss gradient.

Workload: the two-type Morse mixture with a DPD thermostat summed on every type
pair (Philox random term), Newtonian, periodic; 512 particles, 12 steps with a
snapshot every 4. Parameters: Morse (d, a, r0) of AA, AB, BB and the shared
DPD gamma; the loss is the squared distance of the smoothed A-B radial
distribution (64 bins on [0, 2.5]) from a seeded target.

A finite difference of this model is only meaningful where the loss is smooth
in theta over the step. The tabulated Morse force does not vanish at the
cutoff, so a pair crossing it makes the force jump; the test uses a steeper
well (a = 8: the force at the cutoff is ~1e-4 d) over 12 steps, where central
differences with h = 1e-4 and 1e-5 agree to better than 1e-3 on every
component, and compares against h = 1e-5."""
import ctypes

import numpy as np
import pytest
import torch

import mechanica_b200 as m
from mechanica_b200 import adjoint as A
from mechanica_b200 import workloads as W
from mechanica_b200._native import lib
from oracle import adjoint_ref as R

pytestmark = pytest.mark.gpu

N, T, K = 512, 12, 4
GRAD_TOL = 1e-3


def _spec():
    return W.adjoint_spec(n=N, seed=3, a=8.0)


def _table(q):
    p = m.Potential.morse(*q)
    info = p._info()
    coef = np.zeros((info["n"] + 1) * 8, dtype=np.float32)
    lib().mxg_potential_coeffs(p._h, coef.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(coef))
    return p, info, coef


def _terms(spec, theta):
    """FP64 reference terms at theta: tables re-fitted on their frozen nodes."""
    terms = {}
    dt = spec["dt"]
    delta = float(np.float32(1.0 / np.sqrt(dt)))
    for k, (pair, q) in enumerate(spec["morse"].items()):
        p, info, _ = _table(q)
        qq = list(q)
        qq[0], qq[1], qq[2] = theta[3 * k], theta[3 * k + 1], theta[3 * k + 2]
        p.refit(qq)
        info = p._info()
        # the FP64 coefficients of the frozen-node fit, so the differences carry no float rounding
        coef = np.zeros((info["n"] + 1) * 8, dtype=np.float64)
        lib().mxg_potential_coeffs64(p._h, coef.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(coef))
        tab = R.Table(coef, info["alpha"], info["a"], info["b"], info["n"], info["flags"], theta[3 * k + 2] + 1.0)
        a, _, s, cut, _ = spec["dpd"]
        terms[pair] = [tab, R.Dpd(a, theta[9], s, cut, delta)]
    return terms


def _reference_loss(spec, theta, x0=None, target=None):
    box = np.asarray(spec["dim"])
    h = box[0] / spec["cells"][0]
    maxv = float(np.float32(np.float32(h) * np.float32(0.05)) / np.float32(spec["dt"]))
    x = R.run(spec["x"] if x0 is None else x0, spec["v"].astype(np.float64), spec["t"], np.arange(N), box,
              np.array([1.0, 1.0]), np.array([1.0, 1.0]), _terms(spec, theta), spec["cutoff"], spec["dt"], T, 0,
              maxv)
    return R.rdf_loss(x, spec["t"], box, 0, 1, target), x


def _gpu(spec):
    u, P = W.build_adjoint(spec, stream=torch.cuda.current_stream().cuda_stream)
    return u, P, A.Simulation(u, P, nsteps=T, checkpoint_every=K, step0=0)


def test_summed_pair_force_matches_fp64_restatement():
    spec = _spec()
    u, P, sim = _gpu(spec)
    u.force()
    x, v, f, c, xr = u.state()
    theta = P.theta()
    box = np.asarray(spec["dim"])
    fr = R.forces(spec["x"], spec["v"].astype(np.float64), spec["t"], np.arange(N), box, np.array([1.0, 1.0]),
                  _terms(spec, theta), spec["cutoff"], 0)
    rel = np.sqrt(((f - fr) ** 2).sum() / (fr ** 2).sum())
    assert rel <= 1e-5, rel


def test_snapshot_replays_bitwise():
    spec = _spec()
    u, P, sim = _gpu(spec)
    P.register()
    sim.load(spec["x"], spec["v"])
    sim.step(3)
    buf = sim.snapshot_buffer()
    sim.save(buf)
    sim.step(7)
    a = sim.positions().cpu().numpy()
    sim.restore(buf)
    sim.step(7)
    b = sim.positions().cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_vjp_step_with_saved_forces_matches_recomputed_forces():
    """The VJP of a step taken with the forces that the step itself produced
    (mxg_engine_save_forces, then mxg_engine_vjp_step_forces) gives the same adjoints and
    parameter terms, bit for bit, as the VJP that repeats the step's force pass."""
    spec = _spec()
    u, P, sim = _gpu(spec)
    P.register()
    sim.load(spec["x"], spec["v"])
    sim.step(2)
    e = sim._engine()
    buf = sim.snapshot_buffer()
    sim.save(buf)
    sim.step(1)
    fbuf = torch.empty((N, 4), dtype=torch.float32, device="cuda")
    assert lib().mxg_engine_save_forces(e, ctypes.c_void_p(fbuf.data_ptr())) == 0
    rng = np.random.default_rng(11)
    lam0 = torch.tensor(rng.normal(size=(N, 4)), dtype=torch.float32, device="cuda")
    outs = []
    for forces in (None, fbuf):
        sim.restore(buf)
        lx, lv = lam0.clone(), (0.5 * lam0).clone()
        g = torch.zeros(16, dtype=torch.float64, device="cuda")
        gp = ctypes.cast(g.data_ptr(), ctypes.POINTER(ctypes.c_double))
        if forces is None:
            rc = lib().mxg_engine_vjp_step(e, ctypes.c_void_p(lx.data_ptr()), ctypes.c_void_p(lv.data_ptr()), gp)
        else:
            rc = lib().mxg_engine_vjp_step_forces(e, ctypes.c_void_p(lx.data_ptr()), ctypes.c_void_p(lv.data_ptr()),
                                                  gp, ctypes.c_void_p(forces.data_ptr()))
        assert rc == 0
        torch.cuda.synchronize()
        outs.append((lx.cpu().numpy(), lv.cpu().numpy(), g.cpu().numpy()))
    (x0, v0, g0), (x1, v1, g1) = outs
    assert np.array_equal(x0.view(np.uint32), x1.view(np.uint32))
    assert np.array_equal(v0.view(np.uint32), v1.view(np.uint32))
    assert np.array_equal(g0.view(np.uint64), g1.view(np.uint64))
    assert np.abs(g0[:len(P.slots)]).sum() > 0


def test_adjoint_gradients_match_fp64_finite_differences():
    spec = _spec()
    target = W.rdf_target()
    u, P, sim = _gpu(spec)
    theta0 = P.theta()
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor(spec["x"], dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(spec["v"], dtype=torch.float64, requires_grad=True)
    x4 = A.trajectory(theta, x0, v0, sim)
    tgt = torch.tensor(target, dtype=torch.float64, device="cuda")
    loss, g = A.rdf_loss(x4, tgt, spec["dim"], 0, 1)
    loss.backward()
    ref_loss, _ = _reference_loss(spec, theta0, target=target)
    assert abs(loss.item() - ref_loss) <= 1e-4 * abs(ref_loss)
    # parameters: central differences, h = 1e-5
    h = 1e-5
    fd = np.zeros(10)
    for k in range(10):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        fd[k] = (_reference_loss(spec, tp, target=target)[0] - _reference_loss(spec, tm, target=target)[0]) / (2 * h)
    adj = theta.grad.numpy()
    err = np.linalg.norm(adj - fd) / np.linalg.norm(fd)
    assert err <= GRAD_TOL, (err, adj, fd)
    big = np.abs(fd) > 0.05 * np.abs(fd).max()
    assert np.all(np.abs(adj[big] - fd[big]) <= GRAD_TOL * np.abs(fd[big]) + 1e-3 * np.abs(fd).max())
    # positions: a few components
    gx = x0.grad.numpy()
    for (i, kk) in [(0, 0), (7, 1), (100, 2), (301, 0)]:
        xp, xm = spec["x"].copy(), spec["x"].copy()
        xp[i, kk] += h
        xm[i, kk] -= h
        fdx = (_reference_loss(spec, theta0, x0=xp, target=target)[0] -
               _reference_loss(spec, theta0, x0=xm, target=target)[0]) / (2 * h)
        assert abs(gx[i, kk] - fdx) <= 1e-2 * abs(fdx) + 1e-3 * np.abs(gx).max(), (i, kk, gx[i, kk], fdx)


def test_rdf_loss_gradient_matches_finite_differences():
    spec = _spec()
    target = torch.tensor(W.rdf_target(), dtype=torch.float64, device="cuda")
    x = torch.tensor(np.c_[spec["x"], np.zeros(N)], dtype=torch.float32)
    x[:, 3] = torch.from_numpy(spec["t"].astype(np.int32)).view(torch.float32)
    x4 = x.cuda().requires_grad_(True)
    loss, g = A.rdf_loss(x4, target, spec["dim"], 0, 1)
    loss.backward()
    ref = R.rdf_loss(spec["x"], spec["t"], np.asarray(spec["dim"]), 0, 1, W.rdf_target())
    assert abs(loss.item() - ref) <= 1e-5 * abs(ref)
    gx = x4.grad.cpu().numpy()
    h = 1e-4
    for (i, kk) in [(3, 0), (50, 1), (222, 2)]:
        xp, xm = spec["x"].copy(), spec["x"].copy()
        xp[i, kk] += h
        xm[i, kk] -= h
        box = np.asarray(spec["dim"])
        fd = (R.rdf_loss(xp, spec["t"], box, 0, 1, W.rdf_target()) -
              R.rdf_loss(xm, spec["t"], box, 0, 1, W.rdf_target())) / (2 * h)
        assert abs(gx[i, kk] - fd) <= 1e-3 * abs(fd) + 1e-4 * np.abs(gx).max(), (i, kk, gx[i, kk], fd)


def test_adjoint_at_the_workload_parameters():
    """The same check at the adjoint workload's own Morse steepness (a = 5; 512 particles, 4
    steps, a snapshot every 2) with the workload's finite-difference step h = 1e-4. The Morse
    d and a and the DPD gamma gradients agree with FP64 central differences within 1e-3.
    r0 moves the table's range edge (s = r - 2 radius + r0 + 1 <= cutoff) across the pairs
    that sit at the cutoff, so its finite difference carries O(jump / h) terms: its spread
    over h = 1e-4, 1e-5, 1e-6 is measured here, and the adjoint must agree with the h = 1e-4
    difference within that spread (or 1e-3, whichever is larger)."""
    global T
    saved = T
    T = 4
    try:
        spec = W.adjoint_spec(n=N, seed=3, a=5.0)
        target = W.rdf_target()
        u, P = W.build_adjoint(spec, stream=torch.cuda.current_stream().cuda_stream)
        sim = A.Simulation(u, P, nsteps=T, checkpoint_every=2, step0=0)
        theta0 = P.theta()
        theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
        x0 = torch.tensor(spec["x"], dtype=torch.float64)
        v0 = torch.tensor(spec["v"], dtype=torch.float64)
        x4 = A.trajectory(theta, x0, v0, sim)
        loss, _ = A.rdf_loss(x4, torch.tensor(target, dtype=torch.float64, device="cuda"), spec["dim"], 0, 1)
        loss.backward()
        adj = theta.grad.numpy()

        def fd(k, h):
            tp, tm = theta0.copy(), theta0.copy()
            tp[k] += h
            tm[k] -= h
            return (_reference_loss(spec, tp, target=target)[0] - _reference_loss(spec, tm, target=target)[0]) / (2 * h)

        for k in range(10):
            f4 = fd(k, 1e-4)
            if k in (2, 5, 8):  # Morse r0
                spread = max(abs(f4 - fd(k, 1e-5)), abs(f4 - fd(k, 1e-6)))
                assert abs(adj[k] - f4) <= max(GRAD_TOL * abs(f4), 2 * spread), (k, adj[k], f4, spread)
            else:
                assert abs(adj[k] - f4) <= GRAD_TOL * abs(f4) + 1e-6, (k, adj[k], f4)
        u.close()
    finally:
        T = saved
