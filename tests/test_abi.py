"""The C-ABI library loads without a GPU and exports every entry point that
include/mxg.h declares; host-only entry points work on the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from mechanica_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "mxg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mxg_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(_native.exported_symbols())


def test_engine_without_device_fails_loudly():
    import mechanica_b200 as m
    if _has_gpu():
        pytest.skip("a GPU is present")
    m.init(dim=[4, 4, 4], cells=[4, 4, 4])
    T = type("T", (m.Particle,), {"mass": 1.0, "radius": 0.1})
    T.factory(positions=np.array([[1.0, 1.0, 1.0]]))
    with pytest.raises(m.EngineError) as exc:
        m.universe.force()
    assert exc.value.code == -22  # no CUDA device; there is no CPU fallback


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_argument_errors():
    lib = _native.lib()
    h = ctypes.c_void_p()
    o = np.zeros(3)
    d = np.array([10.0, 10.0, 10.0])
    c = np.array([0, 4, 4], dtype=np.int32)
    rc = lib.mxg_engine_init(_native.ptr(o, ctypes.c_double), _native.ptr(d, ctypes.c_double),
                             _native.ptr(c, ctypes.c_int), 1.0, None, None, None, 8, 0, ctypes.byref(h))
    assert rc == -104
    c = np.array([4, 4, 4], dtype=np.int32)
    rc = lib.mxg_engine_init(_native.ptr(o, ctypes.c_double), _native.ptr(d, ctypes.c_double),
                             _native.ptr(c, ctypes.c_int), 1.0, None, None, None, 8, 0, ctypes.byref(h))
    assert rc == 0
    # a particle outside the domain is a space error, as space_addpart's range check
    x = np.array([[11.0, 1.0, 1.0]])
    t = np.zeros(1, dtype=np.int32)
    assert lib.mxg_engine_addtype(h, 1.0, 0.1, 0, 0) == 0
    rc = lib.mxg_engine_addparts(h, 1, _native.ptr(x, ctypes.c_double), None, _native.ptr(t, ctypes.c_int), None)
    assert rc == -3
    t = np.array([5], dtype=np.int32)
    x = np.array([[1.0, 1.0, 1.0]])
    rc = lib.mxg_engine_addparts(h, 1, _native.ptr(x, ctypes.c_double), None, _native.ptr(t, ctypes.c_int), None)
    assert rc == -6
    lib.mxg_engine_finalize(h)
