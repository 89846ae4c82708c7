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
