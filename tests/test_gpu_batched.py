"""Batched replicas: every replica in one engine steps exactly as it does alone
(the kernels process each cell independently, so results are bit-identical),
and the ensemble matches the reference per replica."""
import numpy as np
import pytest

from mechanica_b200 import workloads as W
from oracle import refengine

from golden_util import rel_rms

pytestmark = pytest.mark.gpu


def _small_specs():
    return W.cell_sorting_specs(nrep=4, seed=9, nmin=300, nmax=1500)


def test_batched_equals_separate_runs():
    specs = _small_specs()
    u = W.build_gpu_batch(specs)
    u.steps(5)
    xb, vb, fb, cb, xrb = u.state()
    ep_b, ek_b = u.energies()
    off = 0
    for sc in specs:
        n = len(sc["t"])
        us = W.build_gpu(sc)
        us.steps(5)
        xs, vs, fs, cs, xrs = us.state()
        assert np.array_equal(xrb[off:off + n].view(np.uint32), xrs.view(np.uint32))
        assert np.array_equal(fb[off:off + n].view(np.uint32), fs.view(np.uint32))
        off += n
    assert off == len(xb)


@pytest.mark.skipif(not refengine.available(), reason="reference library not built")
def test_batched_force_pass_matches_reference_per_replica():
    specs = _small_specs()
    u = W.build_gpu_batch(specs)
    u.force()
    x, v, f, c, xr = u.state()
    off = 0
    for sc in specs:
        n = len(sc["t"])
        ref = refengine.run(dict(sc, action="force", runners=2))
        assert rel_rms(f[off:off + n], ref["f"]) <= 1e-5
        assert np.array_equal(xr[off:off + n].view(np.uint32), ref["xrel"].view(np.uint32))
        off += n


def test_autotune_keeps_results():
    specs = _small_specs()
    u = W.build_gpu_batch(specs)
    u.force()
    f0 = u.state()[2]
    per_sm = u.autotune()
    assert per_sm > 0
    u.force()
    assert np.array_equal(u.state()[2], f0)
