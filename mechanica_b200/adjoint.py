"""Reverse-mode gradients of trajectories through the engine's adjoint kernels.

``Trajectory`` is a ``torch.autograd.Function`` mapping (theta, x0, v0) to the
final state of an n-step run (absolute positions by particle id, float4 with
the type in w). Its forward pass steps the engine and keeps a snapshot of the
whole device state every K steps; its backward pass recomputes each segment
from its snapshot, keeping the segment's per-step states, and walks back
through them with ``mxg_engine_vjp_step`` (the adjoint of the force pass, the
bonds and the integrator), which also accumulates d loss / d theta. The DPD random term
is replayed exactly: its Philox stream is keyed on the step counter, which the
snapshots carry.

theta maps onto potential construction parameters through ``Parameters``:
slot k holds one value shared by a list of (potential, parameter index)
entries, e.g. one DPD gamma for all type pairs. Tables are re-fitted on their
frozen nodes when theta changes, so the gradients are those of the tabulated
model the engine integrates (see ``Potential.refit``).

``rdf_loss`` is the workload's loss: the squared distance between a
Gaussian-smoothed A-B radial distribution and a target, with its own
hand-written gradient kernel (``mxg_rdf``).

The reference has no counterpart (mdcore has no adjoint).
"""
import ctypes

import numpy as np
import torch

from . import _native
from ._native import check, lib

RDF_FIXED = float(2 ** 32)


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Parameters:
    """theta[slot] is the value of every (potential, parameter index) entry of slot."""

    def __init__(self, universe, slots):
        self.u = universe
        self.slots = [list(entries) for entries in slots]

    @staticmethod
    def construction(pot):
        n = lib().mxg_potential_params(pot._h, None, 0)
        out = np.zeros(n)
        lib().mxg_potential_params(pot._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        return out

    def theta(self):
        return np.array([self.construction(e[0][0])[e[0][1]] for e in self.slots])

    def apply(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        for k, entries in enumerate(self.slots):
            for pot, j in entries:
                q = self.construction(pot)
                q[j] = theta[k]
                self.u.set_potential_params(pot, q)

    def register(self):
        """Tells the engine which (engine potential, parameter) feeds which slot: every
        copy of the potential bound to a type pair or used by bonds."""
        pots, params, slots = [], [], []
        for k, entries in enumerate(self.slots):
            for pot, j in entries:
                idxs = [self.u.potential_index(a, b, rep, which) for (p, a, b, rep, which) in self.u._pots
                        if p is pot]
                for idx in idxs + self.u.bond_potential_indices(pot):
                    pots.append(idx)
                    params.append(j)
                    slots.append(k)
        n = len(pots)
        arr = lambda v: (ctypes.c_int * max(1, n))(*v)
        check(lib().mxg_engine_adjoint_params(self.u.handle, n, arr(pots), arr(params), arr(slots)), "adjoint_params")


class Simulation:
    """What a Trajectory runs: the universe, its parameters, the step count, the
    checkpoint interval K and the Philox step counter at the start."""

    def __init__(self, universe, parameters, nsteps, checkpoint_every=20, step0=0):
        self.u = universe
        self.params = parameters
        self.nsteps = int(nsteps)
        self.K = int(checkpoint_every)
        self.step0 = int(step0)
        self._bytes = None
        # the bonds' active flags at the start: every run from (x0, v0) starts from them
        self.bond_flags0 = universe.bond_flags() if universe._bonds else None

    def _engine(self):
        return self.u.handle

    def snapshot_buffer(self):
        if self._bytes is None:
            b = ctypes.c_size_t()
            check(lib().mxg_engine_snapshot_bytes(self._engine(), ctypes.byref(b)), "snapshot_bytes")
            self._bytes = b.value
        return torch.empty(self._bytes, dtype=torch.uint8, device="cuda")

    def save(self, buf):
        check(lib().mxg_engine_snapshot(self._engine(), _dptr(buf), 1), "snapshot save")

    def restore(self, buf):
        check(lib().mxg_engine_snapshot(self._engine(), _dptr(buf), 0), "snapshot load")

    def load(self, x0, v0):
        x = np.ascontiguousarray(x0, dtype=np.float64)
        v = np.ascontiguousarray(v0, dtype=np.float32)
        e = self._engine()
        check(lib().mxg_engine_load(e, len(x), x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "load")
        check(lib().mxg_engine_set_step_counter(e, self.step0), "set_step_counter")
        if self.bond_flags0 is not None:
            self.u.set_bond_flags(self.bond_flags0)

    def positions(self):
        """Absolute positions by id, (N, 4) float32 with the type in w; waits for the
        engine's stream, so the tensor is ready on any torch stream."""
        n = lib().mxg_engine_nr_parts(self._engine())
        x4 = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        check(lib().mxg_engine_positions(self._engine(), _dptr(x4), None), "positions")
        check(lib().mxg_engine_status(self._engine()), "positions")
        return x4

    def step(self, n=1):
        check(lib().mxg_engine_step(self._engine(), n), "step")


class Trajectory(torch.autograd.Function):
    """(theta, x0, v0) -> final positions (N, 4) float32 on the device, by id."""

    @staticmethod
    def forward(ctx, theta, x0, v0, sim):
        torch.cuda.synchronize()
        sim.params.apply(theta.detach().cpu().numpy())
        sim.u.handle  # (re)builds the engine if parameters or particles changed
        sim.params.register()
        sim.load(x0.detach().cpu().numpy(), v0.detach().cpu().numpy())
        snaps = []
        for s in range(sim.nsteps):
            if s % sim.K == 0:
                buf = sim.snapshot_buffer()
                sim.save(buf)
                snaps.append(buf)
            sim.step(1)
        x4 = sim.positions()
        check(lib().mxg_engine_status(sim._engine()), "trajectory")
        ctx.sim = sim
        ctx.snaps = snaps
        ctx.nslots = len(sim.params.slots)
        ctx.dtypes = (theta.dtype, x0.dtype, v0.dtype)
        return x4

    @staticmethod
    def backward(ctx, gx4):
        sim = ctx.sim
        torch.cuda.synchronize()
        n = gx4.shape[0]
        lam_x = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        lam_x[:, :3] = gx4[:, :3].to(torch.float32)
        lam_v = torch.zeros_like(lam_x)
        grad = torch.zeros(max(1, ctx.nslots), dtype=torch.float64, device="cuda")
        e = sim._engine()
        for seg in reversed(range(len(ctx.snaps))):
            s0 = seg * sim.K
            s1 = min(sim.nsteps, s0 + sim.K)
            sim.restore(ctx.snaps[seg])
            states = []
            for s in range(s0, s1):  # recompute the segment, keeping every state and its forces
                buf = sim.snapshot_buffer()
                sim.save(buf)
                sim.step(1)
                fbuf = torch.empty((n, 4), dtype=torch.float32, device="cuda")
                check(lib().mxg_engine_save_forces(e, _dptr(fbuf)), "save_forces")
                states.append((buf, fbuf))
            for buf, fbuf in reversed(states):
                sim.restore(buf)
                check(lib().mxg_engine_vjp_step_forces(e, _dptr(lam_x), _dptr(lam_v),
                                                       ctypes.cast(grad.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                                       _dptr(fbuf)), "vjp_step")
        torch.cuda.synchronize()
        check(lib().mxg_engine_status(e), "adjoint")
        tdt, xdt, vdt = ctx.dtypes
        g_theta = grad[: ctx.nslots].cpu().to(tdt)
        return g_theta, lam_x[:, :3].cpu().to(xdt), lam_v[:, :3].cpu().to(vdt), None


def trajectory(theta, x0, v0, sim):
    return Trajectory.apply(theta, x0, v0, sim)


class _RdfLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x4, target, cfg):
        box, ta, tb, nbins, dr, sigma, norm = cfg
        hist = torch.zeros(nbins, dtype=torch.int64, device="cuda")
        boxa = (ctypes.c_double * 3)(*box)
        torch.cuda.synchronize()
        check(lib().mxg_rdf(_dptr(x4), x4.shape[0], boxa, ta, tb, nbins, dr, sigma, _dptr(hist), None, None,
                            None), "rdf")
        torch.cuda.synchronize()
        H = hist.to(torch.float64) / RDF_FIXED
        g = H * norm
        ctx.save_for_backward(x4, g, target)
        ctx.cfg = cfg
        return ((g - target) ** 2).sum(), g

    @staticmethod
    def backward(ctx, gl, gg):
        x4, g, target = ctx.saved_tensors
        box, ta, tb, nbins, dr, sigma, norm = ctx.cfg
        coef = (2.0 * (g - target) * gl + (gg if gg is not None else 0.0)) * norm
        coef = coef.contiguous()
        grad4 = torch.zeros_like(x4)
        boxa = (ctypes.c_double * 3)(*box)
        torch.cuda.synchronize()
        check(lib().mxg_rdf(_dptr(x4), x4.shape[0], boxa, ta, tb, nbins, dr, sigma, None,
                            ctypes.cast(coef.data_ptr(), ctypes.POINTER(ctypes.c_double)), _dptr(grad4), None),
              "rdf_grad")
        torch.cuda.synchronize()
        return grad4, None, None


def rdf_loss(x4, target, box, type_a, type_b, nbins=64, rmax=2.5, sigma=None, counts=None):
    """(loss, g): g(r_b) = V / (N_a N_b) sum_pairs K(r - r_b) / (4 pi r_b^2) on nbins bins of
    [0, rmax] with a Gaussian K of width sigma (default one bin), loss = sum_b (g - target)^2.
    counts = (N_a, N_b) if known (else counted from x4's types)."""
    dr = rmax / nbins
    sigma = dr if sigma is None else sigma
    if counts is None:
        t = x4[:, 3].contiguous().view(torch.int32)
        counts = (int((t == type_a).sum()), int((t == type_b).sum()))
    V = float(np.prod(box))
    c = (torch.arange(nbins, dtype=torch.float64, device="cuda") + 0.5) * dr
    norm = V / (counts[0] * counts[1]) / (4 * np.pi * c ** 2)
    cfg = (tuple(float(b) for b in box), int(type_a), int(type_b), int(nbins), float(dr), float(sigma), norm)
    return _RdfLoss.apply(x4, target, cfg)
