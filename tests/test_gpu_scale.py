"""Size-independent properties at two million particles, where a comparison with the
reference engine pair by pair would take too long: a DPD fluid periodic on every axis with no
body force, in the reference's random mode.

- Every pair force is evaluated once and applied to its two particles as exact negations, so
  the forces of a pass sum to zero up to the rounding of the per-particle FP32 sums.
- After five steps every particle id is in exactly one slot, every cell lists its particles in
  ascending id, and the cell occupancies add up to the particle count.
- Two engines built from the same input give the same bits after five steps (fixed-order sums,
  no atomics in any force sum, the work-item schedule changes no result).
"""
import numpy as np
import pytest
import torch

from mechanica_b200 import workloads as W

pytestmark = pytest.mark.gpu

N = 2_000_000


def _scenario():
    scn = W.dpd(n=N, dims=(100.0, 50.0, 40.0), seed=9, body=0.0)
    scn["bc"] = ("periodic", "periodic", "periodic")
    scn["forces"] = []
    return scn


def test_forces_sum_to_zero_at_two_million_particles():
    u = W.build_gpu(_scenario())
    u.force()
    x, v, f, c, xr = u.state()
    f = np.asarray(f, dtype=np.float64)
    total = np.abs(f.sum(axis=0))
    scale = np.abs(f).sum(axis=0)
    assert np.all(total <= 1e-6 * scale), (total, scale)
    u.close()


def test_steps_keep_every_particle_and_repeat_bit_for_bit():
    scn = _scenario()
    out = []
    for _ in range(2):
        u = W.build_gpu(scn)
        u.steps(5)
        x, v, f, c, xr = u.state()
        out.append((np.asarray(c), np.asarray(xr, np.float32), np.asarray(v, np.float32), np.asarray(f, np.float32)))
        ids_per_cell = np.bincount(np.asarray(c), minlength=100 * 50 * 40)
        assert ids_per_cell.sum() == N
        # the slot order: cells ascending, ids ascending inside a cell, every id once
        d = u.device_state()
        cell = d["cell"].cpu().numpy()
        ids = d["vel"][:, 3].contiguous().view(torch.int32).cpu().numpy()
        assert np.all(np.diff(cell) >= 0)
        same = np.diff(cell) == 0
        assert np.all(np.diff(ids)[same] > 0)
        assert np.array_equal(np.sort(ids), np.arange(N))
        u.close()
    (c0, x0, v0, f0), (c1, x1, v1, f1) = out
    assert len(c0) == N
    assert np.array_equal(c0, c1)
    for a, b in ((x0, x1), (v0, v1), (f0, f1)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
