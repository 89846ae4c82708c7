"""ctypes binding of libmxg.so, the engine's C ABI (include/mxg.h).

The shared library is built in-tree by mechanica_b200/build.py. Loading fails
loudly if it is missing: there is no CPU fallback for the engine.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmxg.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_uint_p = ctypes.POINTER(ctypes.c_uint)
_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_vpp = ctypes.POINTER(ctypes.c_void_p)

# status codes (include/mxg.h)
MXG_OK = 0
ERRORS = {
    -1: "null pointer",
    -2: "device allocation failed",
    -3: "space error (particle outside the domain or bad geometry)",
    -6: "value out of range",
    -7: "cell error",
    -11: "bond error",
    -17: "potential error",
    -21: "CUDA error",
    -22: "no CUDA device",
    -29: "particle moving too fast (moved more than one cell in a step)",
    -101: "cell bucket overflow (no longer raised)",
    -102: "non-finite position or velocity",
    -103: "call made in the wrong engine state",
    -104: "invalid argument",
}


class EngineError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, 'error')} (code {code})")


def check(rc, where=""):
    if rc < 0:
        raise EngineError(rc, where)
    return rc


_SIGS = {
    "mxg_potential_create_lj126": ([ctypes.c_double] * 5 + [_vpp], ctypes.c_int),
    "mxg_potential_create_morse": ([ctypes.c_double] * 6 + [_vpp], ctypes.c_int),
    "mxg_potential_create_harmonic": ([ctypes.c_double] * 5 + [_vpp], ctypes.c_int),
    "mxg_potential_create_power": ([ctypes.c_double] * 6 + [_vpp], ctypes.c_int),
    "mxg_potential_create_harmonic_angle": ([ctypes.c_double] * 5 + [_vpp], ctypes.c_int),
    "mxg_potential_create_harmonic_dihedral": ([ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, _vpp],
                                               ctypes.c_int),
    "mxg_potential_create_dpd": ([ctypes.c_double] * 4 + [ctypes.c_int, _vpp], ctypes.c_int),
    "mxg_potential_info": ([_vp, _c_int_p, _c_uint_p, _c_int_p, _c_float_p, _c_float_p, _c_float_p, _c_float_p],
                           ctypes.c_int),
    "mxg_potential_coeffs": ([_vp, _c_float_p, ctypes.c_int], ctypes.c_int),
    "mxg_potential_dpd_params": ([_vp, _c_float_p, _c_float_p, _c_float_p], ctypes.c_int),
    "mxg_potential_eval": ([_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, _c_float_p, _c_float_p],
                           ctypes.c_int),
    "mxg_potential_free": ([_vp], None),
    "mxg_engine_init": ([_c_double_p, _c_double_p, _c_int_p, ctypes.c_double, _c_int_p, _c_float_p, _c_float_p,
                         ctypes.c_int, ctypes.c_uint, _vpp], ctypes.c_int),
    "mxg_engine_set_dt": ([_vp, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "mxg_engine_set_rng_mode": ([_vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_set_pair_pruning": ([_vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_addtype": ([_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_uint], ctypes.c_int),
    "mxg_engine_addpot": ([_vp, _vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "mxg_engine_add_singlebody_force": ([_vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float],
                                        ctypes.c_int),
    "mxg_engine_addparts": ([_vp, ctypes.c_int, _c_double_p, _c_float_p, _c_int_p, _c_int_p], ctypes.c_int),
    "mxg_engine_addparts_cellrel": ([_vp, ctypes.c_int, ctypes.c_int, _c_int_p, _c_float_p, _c_float_p, _c_int_p,
                                     _c_int_p], ctypes.c_int),
    "mxg_engine_set_occupancy_hint": ([_vp, ctypes.c_longlong], ctypes.c_int),
    "mxg_engine_addbonds": ([_vp, ctypes.c_int, _c_int_p, _c_int_p, _vp, ctypes.c_double, _c_int_p], ctypes.c_int),
    "mxg_engine_addangles": ([_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, _vp, _c_int_p], ctypes.c_int),
    "mxg_engine_set_boundary_potential": ([_vp, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
    "mxg_engine_add_cuboid": ([_vp, ctypes.c_int, _c_float_p, _c_float_p, _c_float_p, _c_int_p], ctypes.c_int),
    "mxg_engine_set_cuboid_potential": ([_vp, ctypes.c_int, _vp], ctypes.c_int),
    "mxg_engine_cuboid_info": ([_vp, ctypes.c_int, _c_float_p], ctypes.c_int),
    "mxg_engine_set_type_species": ([_vp, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
    "mxg_engine_add_flux": ([_vp] + [ctypes.c_int] * 5 + [ctypes.c_float] * 3, ctypes.c_int),
    "mxg_engine_set_species": ([_vp, ctypes.c_int, ctypes.c_int, _c_float_p], ctypes.c_int),
    "mxg_engine_get_species": ([_vp, ctypes.c_int, ctypes.c_int, _c_float_p], ctypes.c_int),
    "mxg_engine_pairs_within": ([_vp, ctypes.c_int, _c_int_p, ctypes.c_float, _vp, ctypes.c_int, _c_int_p, _c_int_p,
                                 ctypes.c_int, _c_int_p], ctypes.c_int),
    "mxg_engine_group_metrics": ([_vp, ctypes.c_int, _c_int_p, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "mxg_engine_step_timed": ([_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int], ctypes.c_int),
    "mxg_engine_add_exclusions": ([_vp, ctypes.c_int, _c_int_p, _c_int_p], ctypes.c_int),
    "mxg_engine_exclusion_shrink": ([_vp], ctypes.c_int),
    "mxg_engine_adddihedrals": ([_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _vp, _c_int_p],
                                ctypes.c_int),
    "mxg_engine_start": ([_vp, _vp], ctypes.c_int),
    "mxg_engine_step": ([_vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_force": ([_vp], ctypes.c_int),
    "mxg_engine_status": ([_vp], ctypes.c_int),
    "mxg_engine_clear_status": ([_vp], ctypes.c_int),
    "mxg_engine_nr_parts": ([_vp], ctypes.c_int),
    "mxg_engine_nr_cells": ([_vp], ctypes.c_int),
    "mxg_engine_unload": ([_vp, ctypes.c_int, _c_double_p, _c_float_p, _c_float_p, _c_int_p, _c_float_p],
                          ctypes.c_int),
    "mxg_engine_load": ([_vp, ctypes.c_int, _c_double_p, _c_float_p], ctypes.c_int),
    "mxg_engine_energy": ([_vp, _c_double_p, _c_double_p, _c_double_p], ctypes.c_int),
    "mxg_engine_kinetic_energy": ([_vp], ctypes.c_double),
    "mxg_engine_tasks": ([_vp, _c_int_p, ctypes.c_int], ctypes.c_int),
    "mxg_engine_bond_flags": ([_vp, _c_uint_p, ctypes.c_int], ctypes.c_int),
    "mxg_engine_set_bond_flags": ([_vp, _c_uint_p, ctypes.c_int], ctypes.c_int),
    "mxg_engine_number_density": ([_vp, ctypes.c_int, _c_float_p, _c_double_p], ctypes.c_int),
    "mxg_engine_bond_pot_index": ([_vp, ctypes.c_int, _c_int_p], ctypes.c_int),
    "mxg_engine_space_info": ([_vp, _c_int_p, _c_double_p, _c_int_p, _c_uint_p], ctypes.c_int),
    "mxg_engine_device_state": ([_vp, _vpp, _vpp, _vpp, _vpp], ctypes.c_int),
    "mxg_engine_copy_state": ([_vp, _vp, _vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_energy_async": ([_vp, _c_double_p], ctypes.c_int),
    "mxg_engine_finalize": ([_vp], ctypes.c_int),
    "mxg_engine_time_force": ([_vp, ctypes.c_int, _c_double_p], ctypes.c_int),
    "mxg_engine_time_force_launches": ([_vp, ctypes.c_int, _vp, ctypes.c_size_t, _c_double_p], ctypes.c_int),
    "mxg_engine_pair_counts": ([_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
                               ctypes.c_int),
    "mxg_engine_add_replica": ([_vp, _c_double_p, _c_double_p, _c_int_p, _c_int_p, _c_float_p, _c_float_p],
                               ctypes.c_int),
    "mxg_engine_nr_replicas": ([_vp], ctypes.c_int),
    "mxg_engine_addpot_replica": ([_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "mxg_engine_set_integrator": ([_vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_add_singlebody_force_kind": ([_vp, ctypes.c_int, ctypes.c_int, _c_float_p], ctypes.c_int),
    "mxg_engine_set_target_temperature": ([_vp, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "mxg_engine_addpot_second": ([_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "mxg_engine_pot_index": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_int_p],
                             ctypes.c_int),
    "mxg_engine_set_pot_params": ([_vp, ctypes.c_int, _c_double_p, ctypes.c_int], ctypes.c_int),
    "mxg_engine_snapshot_bytes": ([_vp, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "mxg_engine_snapshot": ([_vp, _vp, ctypes.c_int], ctypes.c_int),
    "mxg_engine_adjoint_params": ([_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p], ctypes.c_int),
    "mxg_engine_vjp_step": ([_vp, _vp, _vp, _vp], ctypes.c_int),
    "mxg_engine_vjp_step_forces": ([_vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "mxg_engine_save_forces": ([_vp, _vp], ctypes.c_int),
    "mxg_engine_positions": ([_vp, _vp, _vp], ctypes.c_int),
    "mxg_engine_set_step_counter": ([_vp, ctypes.c_ulonglong], ctypes.c_int),
    "mxg_rdf": ([_vp, ctypes.c_int, _c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                 ctypes.c_double, _vp, _vp, _vp, _vp], ctypes.c_int),
    "mxg_potential_params": ([_vp, _c_double_p, ctypes.c_int], ctypes.c_int),
    "mxg_potential_coeffs64": ([_vp, _c_double_p, ctypes.c_int], ctypes.c_int),
    "mxg_potential_refit": ([_vp, _c_double_p, ctypes.c_int], ctypes.c_int),
    "mxg_potential_param_table": ([_vp, ctypes.c_int, _vpp], ctypes.c_int),
    "mxg_engine_addparts_replica": ([_vp, ctypes.c_int, ctypes.c_int, _c_double_p, _c_float_p, _c_int_p, _c_int_p],
                                    ctypes.c_int),
    "mxg_engine_autotune": ([_vp], ctypes.c_int),
    "mxg_engine_force_config": ([_vp, _c_int_p, _c_int_p, ctypes.c_int], ctypes.c_int),
    "mxg_kinetic_energy_noalloc": ([_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp], ctypes.c_int),
}

_lib = None


def lib():
    """Loads libmxg.so (building it first if the sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            try:
                from . import build as _build
                _build.build()
            except Exception as exc:  # pragma: no cover - build failures surface here
                raise RuntimeError(f"mechanica_b200: libmxg.so is missing and could not be built: {exc}")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def ptr(a, ctype):
    """ctypes pointer into a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
