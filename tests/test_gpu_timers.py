"""Per-phase step timers (the reference's engine timers, engine.h:113-135):
timed steps run the same kernels as graph-launched steps, so the state after
them is identical, and every phase reports a positive time that adds up to at
most the whole step."""
import numpy as np
import pytest

import scenarios as S
from golden_util import load

pytestmark = pytest.mark.gpu


def test_timed_steps_match_plain_steps():
    z, scn = load("lattice_small")
    u = S.build_gpu(scn)
    t = u.timers(5)
    x1, v1, _, c1, _ = u.state()
    u2 = S.build_gpu(scn)
    u2.steps(5)
    x2, v2, _, c2, _ = u2.state()
    assert np.array_equal(c1, c2)
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    for k in ("step", "nonbond", "bonded", "advance", "shuffle"):
        assert t[k] > 0.0, (k, t)
    parts = t["prepare"] + t["nonbond"] + t["bonded"] + t["advance"] + t["shuffle"]
    assert parts <= t["step"] * 1.0001 + 1e-6


def test_force_launch_timing_leaves_the_forces_of_a_force_pass():
    """mxg_engine_time_force_launches times launches of the force kernel alone and then
    recomputes the forces in full: the state's forces are bit-identical to those of a
    plain force pass, and every launch reports a positive duration."""
    import ctypes
    from mechanica_b200._native import check, lib
    z, scn = load("dpd_small")
    u = S.build_gpu(scn)
    u.force()
    f0 = np.ascontiguousarray(u.state()[2], dtype=np.float32).copy()
    ms = np.zeros(3)
    check(lib().mxg_engine_time_force_launches(u._e, 3, None, 0, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
          "time_force_launches")
    assert np.all(ms > 0.0), ms
    f1 = np.ascontiguousarray(u.state()[2], dtype=np.float32)
    assert np.array_equal(f0.view(np.uint32), f1.view(np.uint32))
