"""Checkpoint and resume: a saved state restored into the same universe
continues the trajectory bit for bit (positions, velocities, cells, bond
flags, species), including the counter that keys the Philox DPD stream."""
import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import load

pytestmark = pytest.mark.gpu


def _state(u):
    x, v, f, c, xr = u.state()
    return x, v, c, xr


@pytest.mark.parametrize("name", ["dpd_small", "lattice_small", "species_fluxes"])
def test_restore_resumes_bit_for_bit(name, tmp_path):
    z, scn = load(name)
    u = S.build_gpu(scn, rng_mode="philox" if name == "dpd_small" else "reference")
    u.steps(3)
    path = str(tmp_path / "ckpt.npz")
    u.checkpoint(path)
    u.steps(4)
    a = _state(u)
    fa = u.bond_flags() if "bi" in scn else None
    sa = u.species_values()
    u.restore(path)
    u.steps(4)
    b = _state(u)
    for p, q in zip(a, b):
        assert np.array_equal(p, q)
    if fa is not None:
        assert np.array_equal(fa, u.bond_flags())
    assert np.array_equal(sa, u.species_values())


def test_restore_rejects_another_universe(tmp_path):
    z, scn = load("dpd_small")
    u = S.build_gpu(scn)
    ck = u.checkpoint()
    z2, scn2 = load("argon_small")
    u2 = S.build_gpu(scn2)
    with pytest.raises(ValueError):
        u2.restore(ck)


def test_device_state_views_match_state():
    """The zero-copy device views hold the same state as the host copies."""
    import torch
    z, scn = load("argon_small")
    u = S.build_gpu(scn)
    u.steps(2)
    d = u.device_state()
    torch.cuda.synchronize()
    x, v, f, c, xr = u.state()
    ids = d["vel"].view(torch.int32)[:, 3].cpu().numpy()
    assert sorted(ids.tolist()) == list(range(len(x)))
    assert np.array_equal(d["pos"][:, :3].cpu().numpy(), xr[ids].astype(np.float32))
    assert np.array_equal(d["vel"][:, :3].cpu().numpy(), v[ids])
    assert np.array_equal(d["cell"].cpu().numpy(), c[ids])
