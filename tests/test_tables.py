"""Potential tables: the engine's host table builder against the reference's
own builder (bit-exact FP32 coefficients, interval maps and counts), both the
committed golden tables and, when the reference is built here, live ones."""
import numpy as np
import pytest

import mechanica_b200 as m
from oracle import refengine

import scenarios as S

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "tables.npz"))
NAMES = sorted({k.split("__")[0] for k in GOLD.files})


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_table_matches_golden(name):
    kind = str(GOLD[f"{name}__kind"])
    params = tuple(GOLD[f"{name}__params"])
    p = S.make_potential(kind, params)
    info = p._info()
    n, flags = GOLD[f"{name}__info"]
    assert info["n"] == n
    assert info["flags"] == flags
    assert np.array_equal(_bits(info["alpha"][:3]), _bits(GOLD[f"{name}__alpha"][:3]))
    a, b, r0 = GOLD[f"{name}__ab"]
    assert np.float32(info["a"]) == a and np.float32(info["b"]) == b and np.float32(info["r0_plusone"]) == r0
    assert np.array_equal(_bits(p.coefficients), _bits(GOLD[f"{name}__coef"]))


@pytest.mark.parametrize("name", NAMES)
def test_eval_matches_golden(name):
    """potential_eval_ex at radii 0.5+0.5 across the domain, bit for bit."""
    import ctypes
    from mechanica_b200._native import lib
    kind = str(GOLD[f"{name}__kind"])
    p = S.make_potential(kind, tuple(GOLD[f"{name}__params"]))
    r = GOLD[f"{name}__r"]
    for q, rr in enumerate(r):
        e, f = ctypes.c_float(), ctypes.c_float()
        ok = lib().mxg_potential_eval(p._h, 0.5, 0.5, float(np.float32(rr) * np.float32(rr)), ctypes.byref(e),
                                      ctypes.byref(f))
        assert ok == GOLD[f"{name}__ok"][q]
        if ok:
            assert _bits(e.value) == _bits(GOLD[f"{name}__e"][q])
            assert _bits(f.value) == _bits(GOLD[f"{name}__f"][q])


def test_dpd_potential_fields():
    p = m.Potential.dpd(25.0, 4.5, 3.0, 1.0)
    info = p._info()
    assert info["kind"] == 1
    assert np.float32(info["a"]) == np.sqrt(np.float32(np.finfo(np.float32).eps))
    assert info["b"] == 1.0
    sh = m.Potential.dpd(1, 1, 1, 1, shifted=True)
    assert sh.flags & (1 << 12)


def test_invalid_arguments_raise():
    with pytest.raises(m.EngineError):
        m.Potential.lennard_jones_12_6(1.0, 0.5, 1.0, 1.0, 1e-3)
    with pytest.raises(m.EngineError):
        m.Potential.morse(1, 6, 0, 2.0, 1.0, 1e-3)


@pytest.mark.skipif(not refengine.available(), reason="reference not built here")
def test_tables_random_parameters_live():
    """Seeded parameter sweep against the reference builder compiled in place."""
    from oracle.restatement import reference_table
    rng = np.random.default_rng(7)
    cases = []
    for _ in range(6):
        cases.append(("morse", (float(rng.uniform(0.05, 1.0)), float(rng.uniform(3, 7)), float(rng.uniform(0, 1.5)),
                                1e-4, float(rng.uniform(1.0, 3.0)), 1e-3)))
        A, B = float(rng.uniform(1e-6, 1e-4)), float(rng.uniform(1e-3, 1e-2))
        lo = float(rng.uniform(0.2, 0.4))
        cases.append(("lj126", (lo, float(rng.uniform(1.0, 3.0)), A, B, 1e-3)))
        k, r0 = float(rng.uniform(1, 300)), float(rng.uniform(0.3, 1.5))
        cases.append(("harmonic", (k, r0, 0.2 * r0, 2 * r0, 0.018 * r0)))
        lo, hi = float(rng.uniform(0.0, 1.2)), float(rng.uniform(2.0, 3.4))
        cases.append(("harmonic_angle", (float(rng.uniform(0.5, 50)), float(rng.uniform(lo, hi)), lo, hi,
                                         0.005 * (hi - lo))))
        cases.append(("harmonic_dihedral", (float(rng.uniform(0.5, 5)), int(rng.integers(1, 5)),
                                            float(rng.choice([0.0, np.pi])), 0.001)))
        cases.append(("harmonic_dihedral", (float(rng.uniform(0.5, 5)), int(rng.integers(1, 4)),
                                            float(rng.uniform(0.1, 3.0)), 0.01)))
    for kind, params in cases:
        info, coef = reference_table(kind, params)
        if info is None:  # the reference's fit fails: so must this one
            with pytest.raises(m.EngineError):
                S.make_potential(kind, params)
            continue
        p = S.make_potential(kind, params)
        mine = p._info()
        assert mine["n"] == info["n"], (kind, params)
        assert mine["flags"] == info["flags"], (kind, params)
        assert np.float32(mine["a"]) == np.float32(info["a"]) and np.float32(mine["b"]) == np.float32(info["b"])
        assert np.array_equal(_bits(mine["alpha"][:3]), _bits(info["alpha"])), (kind, params)
        assert np.array_equal(_bits(p.coefficients), _bits(coef)), (kind, params)
