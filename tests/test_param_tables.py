"""Frozen-node re-fits and parameter-derivative tables (host side, no GPU).

The adjoint differentiates the tabulated model: with the interval count, map
and nodes frozen, a table's coefficients are a linear function of the sampled
potential, so dV/dtheta has a table on the same nodes. Checks: a re-fit at the
construction parameters reproduces the coefficients bit for bit, and the
derivative tables agree with central differences of frozen re-fits."""
import ctypes

import numpy as np
import pytest

import mechanica_b200 as m
from mechanica_b200._native import lib


def _coeffs(p):
    n = p._info()["n"]
    out = np.zeros((n + 1) * 8, dtype=np.float32)
    lib().mxg_potential_coeffs(p._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(out))
    return out


def _eval(p, r, ri=1.0, rj=1.0):
    e, f = ctypes.c_float(), ctypes.c_float()
    vals = []
    for x in r:
        ok = lib().mxg_potential_eval(p._h, ctypes.c_float(ri), ctypes.c_float(rj), ctypes.c_float(x * x),
                                      ctypes.byref(e), ctypes.byref(f))
        vals.append((e.value, f.value) if ok == 1 else (np.nan, np.nan))
    return np.array(vals, dtype=np.float64)


CASES = {
    "morse": (lambda q: m.Potential.morse(d=q[0], a=q[1], r0=q[2], min=q[3], max=q[4], tol=q[5]),
              [0.6, 5.0, 1.0, 1e-4, 2.5, 1e-3], [0, 1], np.linspace(0.8, 2.4, 57)),
    "lj126": (lambda q: m.Potential.lennard_jones_12_6(q[0], q[1], q[2], q[3], q[4]),
              [0.275, 1.0, 9.5075e-06, 6.1545e-03, 1e-3], [2, 3], np.linspace(0.3, 0.99, 57)),
    "harmonic": (lambda q: m.Potential.harmonic(k=q[0], r0=q[1], min=q[2], max=q[3], tol=q[4]),
                 [200.0, 0.5, 0.1, 1.0, 1e-3], [0, 1], np.linspace(0.15, 0.95, 57)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_refit_at_construction_parameters_is_bit_exact(name):
    make, q, _, _ = CASES[name]
    p = make(q)
    c0 = _coeffs(p)
    p.refit(q)
    assert np.array_equal(c0.view(np.uint32), _coeffs(p).view(np.uint32))


@pytest.mark.parametrize("name", list(CASES))
def test_param_tables_match_central_differences(name):
    make, q, ks, r = CASES[name]
    p = make(q)
    # the Morse table's argument is shifted by r0: evaluate with unit radii so s = r - 2 + r0 + 1
    for k in ks:
        dt = p.param_table(k)
        got = _eval(dt, r)[:, 0]
        h = 1e-3 * abs(q[k])
        lo, hi = list(q), list(q)
        lo[k] -= h
        hi[k] += h
        pl, ph = make(q), make(q)
        pl.refit(lo)
        ph.refit(hi)
        fd = (_eval(ph, r)[:, 0] - _eval(pl, r)[:, 0]) / (2 * h)
        ok = np.isfinite(fd) & np.isfinite(got)
        assert ok.mean() > 0.9
        scale = np.abs(fd[ok]).max()
        assert np.abs(got[ok] - fd[ok]).max() <= 2e-3 * scale, (k, np.abs(got[ok] - fd[ok]).max(), scale)


def test_refit_keeps_interval_count():
    make, q, _, _ = CASES["morse"]
    p = make(q)
    n0 = p._info()["n"]
    q2 = list(q)
    q2[1] = 7.0  # a steeper well would need more intervals in a fresh fit
    p.refit(q2)
    assert p._info()["n"] == n0
    fresh = make(q2)
    assert fresh._info()["n"] >= n0


def test_dpd_refit_changes_coefficients_only():
    p = m.Potential.dpd(alpha=0.0, gamma=1.0, sigma=1.0, cutoff=2.5)
    p.refit([0.0, 2.0, 1.0, 2.5, 0.0])
    a, g, s = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    lib().mxg_potential_dpd_params(p._h, ctypes.byref(a), ctypes.byref(g), ctypes.byref(s))
    assert (a.value, g.value, s.value) == (0.0, 2.0, 1.0)
    with pytest.raises(Exception):
        p.refit([0.0, 2.0, 1.0, 3.0, 0.0])  # the cutoff is part of the frozen structure
