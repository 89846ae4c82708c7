"""The pairwise bond constructor (Universe.bind_pairwise; make_pairlist,
src/mdcore/src/bond.cpp:892-942) on the device against the reference's own
constructor run on identical inputs (tests/golden/pairwise.npz): the same
pairs in the same order, bit for bit, with and without a type-pair filter and
with a cutoff beyond the engine's cell size."""
import os

import numpy as np
import pytest

import mechanica_b200 as m
import scenarios as S
from golden_util import GOLDEN

pytestmark = pytest.mark.gpu

PW = np.load(os.path.join(GOLDEN, "pairwise.npz"))
CASES = {
    "pw_morse_short": lambda: S.morse2(n=2000, seed=31),
    "pw_morse_long_ab": lambda: S.morse2(n=2000, seed=32),
    "pw_lattice": lambda: S.lattice(nx=6, seed=33, noise=2e-2),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_pairwise_matches_reference(name):
    scn = CASES[name]()
    u = S.build_gpu(scn)
    ids = PW[f"{name}__ids"]
    pairs = [tuple(p) for p in PW[f"{name}__pairs"]] or None
    nb0 = sum(len(b[1]) for b in u._bonds)
    pot = m.Potential.harmonic(k=1.0, r0=0.5, min=0.1, max=1.0, tol=0.009)
    bonds = u.bind_pairwise(pot, ids, float(PW[f"{name}__cutoff"]), pairs=pairs)
    _, bi, bj, _ = u._bonds[-1]
    assert np.array_equal(bi, PW[f"{name}__i"])
    assert np.array_equal(bj, PW[f"{name}__j"])
    assert [b.id for b in bonds] == list(range(nb0, nb0 + len(bi)))
    # the new bonds take part in the next force pass
    u.force()
    assert np.all(u.bond_flags()[nb0:] & 1)


def test_pairwise_respects_list_and_distance():
    """Properties on a fresh random gas: every returned pair is within the
    cutoff in global coordinates, each unordered pair appears once with the
    later list entry first, and nothing within the cutoff is missed."""
    rng = np.random.default_rng(9)
    m.init(dim=[12.0, 12.0, 12.0], cells=[6, 6, 6], cutoff=2.0, dt=0.01)

    class A(m.Particle):
        mass = 1.0
        radius = 0.2

    x = rng.uniform(0, 12, size=(3000, 3))
    ids = A.factory(positions=x)
    u = m.universe
    order = rng.permutation(len(ids)).astype(np.int32)
    pot = m.Potential.harmonic(k=1.0, r0=1.0, min=0.1, max=3.0, tol=0.01)
    cut = 0.9
    u.bind_pairwise(pot, order, cut)
    _, bi, bj, _ = u._bonds[-1]
    pos = u.state()[0].astype(np.float32).astype(np.float64)
    d = np.linalg.norm(pos[bi] - pos[bj], axis=1)
    assert np.all(d <= cut * (1 + 1e-6))
    rank = np.empty(len(order), dtype=np.int64)
    rank[order] = np.arange(len(order))
    assert np.all(rank[bi] > rank[bj])
    key = rank[bi] * len(order) + rank[bj]
    assert np.all(np.diff(key) > 0)
    from scipy.spatial import cKDTree
    ref = cKDTree(pos).query_pairs(cut * (1 - 1e-5))
    got = {(min(a, b), max(a, b)) for a, b in zip(bi.tolist(), bj.tolist())}
    assert ref <= got
