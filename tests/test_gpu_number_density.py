"""Number density f[3] (MxParticle::number_density) and the computed volume, against the
reference engine (oracle tier A, its f[3] after engine_force) and an FP64 restatement.

The reference forms each pair's r with qsqrt, a 12-bit reciprocal square-root estimate
(_mm_rsqrt_ss, smoothing_kernel.hpp:19-24: relative error up to 1.5 x 2^-12), so a pair
term near the cutoff differs by up to ~1e-3 relative; a particle's sum, dominated by the
exact self term W(0, rc), stays within 2e-3 of the reference (the stated tolerance). On
cubic grids, where no pair inside the cutoff is pruned, the sums also match an FP64
restatement (W0 + sum of W(r) over pairs within the cutoff, exact square root) to 1e-5."""
import numpy as np
import pytest

import scenarios as S
from golden_util import load
from oracle import refengine

pytestmark = pytest.mark.gpu

ND_TOL_REFERENCE = 2e-3


def _w(r, h):
    x = r / h
    y = np.where(x < 1, 1 - 1.5 * x * x + 0.75 * x ** 3, np.where(x < 2, 0.25 * (2 - x) ** 3, 0.0))
    return y / (np.pi * h ** 3)


@pytest.mark.skipif(not refengine.available(), reason="reference library not built")
@pytest.mark.parametrize("name", ["argon_small", "dpd_small", "morse2_small", "lattice_noisy", "chains_morse"])
def test_number_density_matches_reference(name):
    z, scn = load(name)
    u = S.build_gpu(scn)
    nd, vol = u.number_density()
    ref = refengine.run(dict(scn, action="force", runners=2))
    nr = ref["number_density"].astype(np.float64)
    rel = np.abs(nd - nr) / nr
    assert rel.max() <= ND_TOL_REFERENCE, rel.max()
    assert abs(vol - (1.0 / nr).sum()) <= ND_TOL_REFERENCE * (1.0 / nr).sum()
    u.close()


@pytest.mark.parametrize("name", ["argon_small", "dpd_small"])
def test_number_density_matches_fp64_restatement(name):
    z, scn = load(name)
    u = S.build_gpu(scn)
    nd, vol = u.number_density()
    x = u.state()[0]
    L = np.asarray(scn["dim"], dtype=np.float64)
    periodic = np.array([b == "periodic" for b in scn["bc"]])
    h = float(scn["cutoff"])
    want = np.full(len(x), _w(0.0, h))
    for i in range(len(x)):
        d = x - x[i]
        d[:, periodic] -= L[periodic] * np.round(d[:, periodic] / L[periodic])
        r2 = (d * d).sum(1)
        sel = (r2 <= np.float32(h) ** 2)
        sel[i] = False
        want[i] += _w(np.sqrt(r2[sel]), h).sum()
    assert np.abs(nd - want).max() <= 1e-5 * want.max()
    u.close()
