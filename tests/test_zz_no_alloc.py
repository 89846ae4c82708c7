"""The allocation-free kinetic-energy entry point against the engine's own
kinetic energy.

mxg_kinetic_energy_noalloc serves callers that cannot call cudaMalloc (device
memory reserved by another allocator, or loops that must not take an
allocation's implicit device synchronisation). Its scratch is a file-scope
device array; this test calls it twice in a row through the C ABI on the
engine's resident state and compares both results with mxg_engine_kinetic_energy
and with a host recomputation per type. It lives in a file that pytest collects
last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import scenarios as S
from golden_util import load

pytestmark = pytest.mark.gpu


def _per_type_host(v, types, masses):
    out = []
    for t, m in enumerate(masses):
        vv = v[types == t].astype(np.float32)
        v2 = (vv[:, 0] * vv[:, 0] + vv[:, 1] * vv[:, 1]) + vv[:, 2] * vv[:, 2]
        e = (0.5 * m * v2.astype(np.float64)).astype(np.float32)
        out.append(float(e.astype(np.float64).sum()))
    return np.array(out)


@pytest.mark.parametrize("name", ["argon_small", "morse2_small", "dpd_small"])
def test_noalloc_kinetic_energy_matches_engine(name):
    import torch
    from mechanica_b200._native import lib

    L = lib()
    z, scn = load(name)
    if name == "morse2_small":
        # give the overdamped mixture velocities so the energies are non-trivial
        scn = dict(scn, v=np.random.default_rng(3).normal(0, 1, size=scn["x"].shape))
        scn["types"] = [(m, r, 0) for (m, r, d) in scn["types"]]
    u = S.build_gpu(scn)
    u.steps(3)
    assert L.mxg_engine_status(u._e) == 0  # also waits for the engine's stream
    pos, vel = ctypes.c_void_p(), ctypes.c_void_p()
    assert L.mxg_engine_device_state(u._e, ctypes.byref(pos), ctypes.byref(vel), None, None) == 0
    n = L.mxg_engine_nr_parts(u._e)
    masses = [float(t[0]) for t in scn["types"]]
    dev = torch.device("cuda", 0)
    type_mass = torch.tensor(masses, dtype=torch.float64, device=dev)
    ek_engine = L.mxg_engine_kinetic_energy(u._e)
    x, v, f, c, xr = u.state()
    per_type = _per_type_host(v, np.asarray(scn["t"]), masses)
    for call in range(2):
        out = torch.full((1 + len(masses),), -1.0, dtype=torch.float64, device=dev)
        rc = L.mxg_kinetic_energy_noalloc(vel, pos, n, ctypes.c_void_p(type_mass.data_ptr()),
                                          len(masses), ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0
        torch.cuda.synchronize(dev)
        res = out.cpu().numpy()
        assert abs(res[0] - ek_engine) <= 1e-12 * abs(ek_engine) + 1e-12, (call, res[0], ek_engine)
        assert np.allclose(res[1:], per_type, rtol=1e-12, atol=1e-12), (call, res[1:], per_type)
    u.close()


def test_noalloc_rejects_too_many_types():
    import torch
    from mechanica_b200._native import lib

    dev = torch.device("cuda", 0)
    buf = torch.zeros(4 * 8, dtype=torch.float32, device=dev)
    mass = torch.ones(65, dtype=torch.float64, device=dev)
    out = torch.zeros(66, dtype=torch.float64, device=dev)
    p = ctypes.c_void_p(buf.data_ptr())
    rc = lib().mxg_kinetic_energy_noalloc(p, p, 8, ctypes.c_void_p(mass.data_ptr()), 65,
                                          ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -6  # MXG_ERR_RANGE: more types than the scratch array holds


def test_noalloc_on_a_stream_and_with_unlisted_types():
    """On a caller's stream (not the default one), and with ntypes smaller than the largest
    type id present: particles whose type is outside [0, ntypes) add nothing, so the total
    is the sum over the types that remain."""
    import torch
    from mechanica_b200._native import lib

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    n = 5000
    types = rng.integers(0, 4, size=n).astype(np.int32)
    v = rng.normal(size=(n, 3)).astype(np.float32)
    pos = np.zeros((n, 4), dtype=np.float32)
    pos[:, 3] = types.view(np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    vel[:, :3] = v
    masses = [1.0, 2.5, 0.5, 4.0]
    pd, vd = torch.from_numpy(pos).to(dev), torch.from_numpy(vel).to(dev)
    st = torch.cuda.Stream(device=dev)
    for ntypes in (4, 2):
        tm = torch.tensor(masses[:ntypes], dtype=torch.float64, device=dev)
        out = torch.full((1 + ntypes,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        rc = lib().mxg_kinetic_energy_noalloc(ctypes.c_void_p(vd.data_ptr()), ctypes.c_void_p(pd.data_ptr()), n,
                                              ctypes.c_void_p(tm.data_ptr()), ntypes,
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream))
        assert rc == 0
        st.synchronize()
        res = out.cpu().numpy()
        want = _per_type_host(v, types, masses[:ntypes])
        assert np.allclose(res[1:], want, rtol=1e-12, atol=1e-12)
        assert abs(res[0] - want.sum()) <= 1e-12 * abs(want.sum())
