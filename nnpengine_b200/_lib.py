"""ctypes binding of libnnpe.so (the C ABI declared in include/nnpe.h).

The library is loaded from the package's ``lib/`` directory; there is no fallback: if it is
missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnnpe.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class Thermo(C.Structure):
    _fields_ = [("step", C.c_int), ("nbuild", C.c_int), ("erg", C.c_double), ("virial", C.c_double),
                ("ekin", C.c_double), ("temperature", C.c_double), ("pressure", C.c_double),
                ("erg_nnp", C.c_double), ("erg_exp", C.c_double)]


_SIGS = {
    "nnpe_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "nnpe_destroy": (None, [_vp]),
    "nnpe_last_error": (C.c_char_p, [_vp]),
    "nnpe_device_errors": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "nnpe_stream": (_vp, [_vp]),
    "nnpe_device_bytes": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "nnpe_set_system": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, _i32p, _f32p, _f32p, _f32p, _i32p, _i32p, _i32p,
                                  C.c_int, C.c_int, _i32p]),
    "nnpe_load_system_file": (C.c_int, [_vp, C.c_char_p]),
    "nnpe_natom": (C.c_int, [_vp]),
    "nnpe_npair": (C.c_int, [_vp]),
    "nnpe_set_positions": (C.c_int, [_vp, _f32p]),
    "nnpe_set_velocities": (C.c_int, [_vp, _f32p]),
    "nnpe_setup": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_int]),
    "nnpe_set_box": (C.c_int, [_vp, C.c_double]),
    "nnpe_pair_set_table": (C.c_int, [_vp, C.c_int, _f32p, _f32p]),
    "nnpe_pair_load_table": (C.c_int, [_vp, C.c_int, C.c_char_p]),
    "nnpe_pair_get_table": (C.c_int, [_vp, _f32p, _f32p]),
    "nnpe_pair_enable": (C.c_int, [_vp, C.c_int]),
    "nnpe_pair_exact": (C.c_int, [_vp, C.c_int]),
    "nnpe_bond_coef": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, _f32p]),
    "nnpe_angle_coef": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, _f32p]),
    "nnpe_dihedral_coef": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, _f32p]),
    "nnpe_bonded_set": (C.c_int, [_vp, C.c_int, _i32p, C.c_int, _f32p, C.c_int, _i32p, C.c_int, _f32p, C.c_int, _i32p,
                                  C.c_int, _f32p]),
    "nnpe_verlet_setup": (C.c_int, [_vp, C.c_double, C.c_int]),
    "nnpe_set_total_steps": (C.c_int, [_vp, C.c_int]),
    "nnpe_thermostat": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_uint64]),
    "nnpe_list_build": (C.c_int, [_vp]),
    "nnpe_list_isvalid": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "nnpe_ghost_update": (C.c_int, [_vp]),
    "nnpe_list_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nnpe_set_prune": (C.c_int, [_vp, C.c_double]),
    "nnpe_prune_info": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "nnpe_list_get": (C.c_int, [_vp, C.c_int64, _i32p, C.POINTER(C.c_int64)]),
    "nnpe_verify_grid": (C.c_int, [_vp]),
    "nnpe_verify_grid_arrays": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _i32p, _i32p, _i32p, _i32p,
                                          _i32p, _f32p, C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "nnpe_compute_forces": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nnpe_get_forces": (C.c_int, [_vp, C.c_int, _f32p]),
    "nnpe_force_step": (C.c_int, [_vp, _vp, _vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nnpe_force_step_noalloc": (C.c_int, [_vp, _vp, _vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nnpe_get_positions": (C.c_int, [_vp, _f32p]),
    "nnpe_get_positions_f64": (C.c_int, [_vp, _f64p]),
    "nnpe_get_velocities": (C.c_int, [_vp, _f32p]),
    "nnpe_get_velocities_f64": (C.c_int, [_vp, _f64p]),
    "nnpe_get_atom_energy": (C.c_int, [_vp, _f64p]),
    "nnpe_verlet_update_x": (C.c_int, [_vp, C.c_double]),
    "nnpe_verlet_update_v": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "nnpe_init_velocities": (C.c_int, [_vp, C.c_double, C.c_double, C.c_uint64]),
    "nnpe_run": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(Thermo), C.c_int, C.POINTER(C.c_int)]),
    "nnpe_run_graph": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(Thermo), C.c_int, C.POINTER(C.c_int)]),
    "nnpe_nnp_set": (C.c_int, [_vp, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                               _vp, _vp, _vp, _vp, _vp, _vp]),
    "nnpe_nnp_load": (C.c_int, [_vp, C.c_double, C.c_int, C.c_char_p, C.c_char_p]),
    "nnpe_nnp_precision": (C.c_int, [_vp, C.c_int]),
    "nnpe_nnp_enable": (C.c_int, [_vp, C.c_int]),
    "nnpe_nnp_get": (C.c_int, [_vp, _vp, _vp, _vp]),
    "nnpe_nnp_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nnpe_nnp_pairs": (C.c_int64, [_vp]),
    "nnpe_sqd_setup": (C.c_int, [_vp, C.c_int, C.c_double, C.POINTER(C.c_int)]),
    "nnpe_sqd_compute": (C.c_int, [_vp]),
    "nnpe_sqd_get": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nnpe_sqd_dump": (C.c_int, [_vp, C.c_char_p, C.c_int]),
    "nnpe_nnp_autotune": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nnpe_nnp_grids": (C.c_int, [_vp, C.c_int, C.c_int]),
    "nnpe_nnp_get_grids": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nnpe_bonded_autogen": (C.c_int, [_vp, C.c_int, _f32p, C.c_int, _f32p, C.c_int, _f32p]),
    "nnpe_profile_enqueue": (C.c_int, [_vp, C.c_int]),
    "nnpe_tc_selftest": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p]),
    "nnpe_launches_per_step": (C.c_int, [_vp]),
    "nnpe_gr_setup": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]),
    "nnpe_gr_tally": (C.c_int, [_vp, C.c_int]),
    "nnpe_gr_nbin": (C.c_int, [_vp, C.c_int]),
    "nnpe_gr_get": (C.c_int, [_vp, C.c_int, _u64p, _f64p]),
    "nnpe_sq_compute": (C.c_int, [_vp, C.c_int, _f64p, _f64p]),
    "nnpe_rmdf_set": (C.c_int, [_vp, C.c_int, _f64p, _f64p, _f64p, C.c_double, C.c_double]),
    "nnpe_rmdf_load": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_char_p), C.c_double, C.c_double]),
    "nnpe_rmdf_load_delta": (C.c_int, [_vp, C.c_char_p]),
    "nnpe_rmdf_step": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double)]),
    "nnpe_rmdf_get": (C.c_int, [_vp, _vp, _vp, _vp]),
    "nnpe_rmdf_dump_sq": (C.c_int, [_vp, C.c_char_p, C.c_int]),
}

_lib = None


def load() -> C.CDLL:
    """Load libnnpe.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libnnpe.so not built ({LIB_PATH}); run __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        if not hasattr(lib, name):
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols():
    """Function names declared in include/*.h (for the export check)."""
    import re
    inc = os.path.join(HERE, "..", "include")
    names = []
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(inc, fn)) as f:
            txt = f.read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(nnpe_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))
