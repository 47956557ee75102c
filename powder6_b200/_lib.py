"""ctypes binding of libp6cuda.so (declared in include/p6cuda.h).

The library is loaded from this package directory.  There is no fallback: if
the shared library is missing or cannot be loaded, every product entry point
raises P6Error.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / 'libp6cuda.so'

P6_OK = 0
P6_ERR_CAPACITY = 2
STATUS_NAMES = {0: 'OK', 1: 'INVALID_ARG', 2: 'CAPACITY', 3: 'DEVICE_LOST', 4: 'TIMEOUT', 5: 'NOT_CONVERGED',
                6: 'VALIDATION', 7: 'CUDA'}


class P6Error(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = code
        self.status = STATUS_NAMES.get(code, str(code))
        super().__init__(f'p6 {self.status}: {message}')


class P6WyParticleState(C.Structure):
    _fields_ = [('fit', C.c_float), ('cc', C.c_float), ('pen', C.c_float), ('step_size', C.c_float),
                ('temp', C.c_float), ('seed', C.c_uint32), ('accepted', C.c_uint32), ('pad', C.c_uint32),
                ('best_fit', C.c_float), ('best_cc', C.c_float), ('best_pen', C.c_float), ('best_pad', C.c_float)]


class P6WyProblem(C.Structure):
    _fields_ = [('num_particles', C.c_int),
                ('gen_pack', C.POINTER(C.c_uint32)), ('n_assign', C.c_int), ('n_tot', C.c_int),
                ('sym_packed', C.POINTER(C.c_float)), ('n_ops', C.c_int),
                ('site_proj', C.POINTER(C.c_float)), ('max_sites', C.c_int),
                ('refl_pack', C.POINTER(C.c_uint32)), ('n_refl', C.c_int),
                ('group_meta', C.POINTER(C.c_float)), ('n_groups', C.c_int), ('group_stride', C.c_int),
                ('f_tab', C.POINTER(C.c_float)), ('n_elem', C.c_int),
                ('restraint_tables', C.POINTER(C.c_float)), ('n_restraint_floats', C.c_int),
                ('r_min_off', C.c_int), ('rule_off', C.c_int), ('n_rules', C.c_int),
                ('max_coord_slots', C.c_int), ('geom_slots', C.c_int),
                ('orth', C.c_double * 9), ('xform', C.c_double * 9), ('inv_orth', C.c_double * 9),
                ('min_image_shell', C.c_int), ('count_shell', C.c_int), ('centro', C.c_int),
                ('pen_clash', C.c_float), ('pen_bond', C.c_float), ('pen_coord', C.c_float),
                ('pen_geom', C.c_float), ('poly_prob', C.c_float),
                ('step_up', C.c_float), ('step_down', C.c_float), ('step_min', C.c_float), ('step_max', C.c_float),
                ('cos_mode', C.c_int), ('run_key', C.c_uint32), ('incremental', C.c_int)]


class P6PtProblem(C.Structure):
    _fields_ = [('n_refl', C.c_int), ('hkl', C.c_void_p), ('mult', C.c_void_p),
                ('n_reps', C.c_int), ('rep_rot', C.c_void_p), ('rep_trans', C.c_void_p),
                ('n_atoms', C.c_int), ('atom_pos', C.c_void_p), ('atom_wmult', C.c_void_p), ('atom_occ', C.c_void_p),
                ('ff_a', C.c_void_p), ('ff_b', C.c_void_p), ('ff_c', C.c_void_p),
                ('n_points', C.c_int), ('tth', C.c_void_p), ('y', C.c_void_p), ('w', C.c_void_p),
                ('lambda1', C.c_double), ('lambda2', C.c_double), ('ratio', C.c_double), ('pol_k', C.c_double),
                ('min_fwhm', C.c_double), ('dmin', C.c_double), ('n_bkg', C.c_int),
                ('n_full', C.c_int), ('full_values', C.c_void_p),
                ('nv', C.c_int), ('index', C.c_void_p), ('lo', C.c_void_p), ('hi', C.c_void_p), ('scales', C.c_void_p),
                ('cubic', C.c_int), ('chains', C.c_int), ('max_temp', C.c_double), ('seed', C.c_uint32),
                ('has_po', C.c_int), ('eq_start', C.c_void_p), ('eq_hkl', C.c_void_p), ('po_dir', C.c_double * 3),
                ('has_asym', C.c_int), ('method', C.c_int), ('has_shift', C.c_int)]


_P = C.c_void_p
class P6CtProblem(C.Structure):
    _fields_ = [('n_refl', C.c_int), ('n_points', C.c_int), ('max_replicas', C.c_int),
                ('profile_t', C.c_void_p), ('yobs', C.c_void_p), ('w', C.c_void_p)]


_SIGS = {
    'p6_last_error': (C.c_char_p, []),
    'p6_abi_version': (C.c_int, []),
    'p6_debug_inject_failure': (None, [C.c_int, C.c_int]),
    'p6_philox_device': (C.c_int, [_P, _P, _P]),
    'p6_wy_create': (C.c_int, [C.POINTER(P6WyProblem), C.c_int, C.POINTER(C.c_void_p)]),
    'p6_wy_destroy': (C.c_int, [_P]),
    'p6_wy_set_assign': (C.c_int, [_P, _P]),
    'p6_wy_set_params': (C.c_int, [_P, C.c_int, C.c_float]),
    'p6_wy_sync_state': (C.c_int, [_P, _P, _P]),
    'p6_wy_read_state': (C.c_int, [_P, _P, _P, _P]),
    'p6_wy_dispatch': (C.c_int, [_P, _P, C.c_int]),
    'p6_wy_evaluate_sync': (C.c_int, [_P, _P, C.c_int, _P]),
    'p6_wy_set_ladders': (C.c_int, [_P, _P, C.c_int, C.c_int]),
    'p6_wy_set_schedule': (C.c_int, [_P, _P, _P, C.c_int]),
    'p6_wy_set_quench': (C.c_int, [_P, _P, C.c_int]),
    'p6_wy_run': (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    'p6_wy_run_host': (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P]),
    'p6_wy_synchronize': (C.c_int, [_P, C.c_double]),
    'p6_wy_write_positions_fixed': (C.c_int, [_P, _P]),
    'p6_wy_read_positions_fixed': (C.c_int, [_P, _P, _P]),
    'p6_wy_write_state_fixed': (C.c_int, [_P, _P, _P, _P]),
    'p6_wy_set_ladder_split': (C.c_int, [_P, C.c_int]),
    'p6_wy_refine': (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P]),
    'p6_wy_set_trace': (C.c_int, [_P, C.c_int]),
    'p6_wy_read_trace': (C.c_int, [_P, _P, _P]),
    'p6_wy_read_trace_ic': (C.c_int, [_P, _P]),
    'p6_wy_read_trace_sums': (C.c_int, [_P, _P]),
    'p6_wy_set_fragment': (C.c_int, [_P, _P]),
    'p6_wy_write_fragment_state': (C.c_int, [_P, _P]),
    'p6_wy_read_fragment_state': (C.c_int, [_P, _P, _P]),
    'p6_wy_debug_fragment': (C.c_int, [_P, _P, C.c_int, _P]),
    'p6_wy_debug_expand': (C.c_int, [_P, C.c_int, _P]),
    'p6_wy_last_kernel_ms': (C.c_int, [_P, C.POINTER(C.c_float)]),
    'p6_wy_launch_count': (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    'p6_wy_query': (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    'p6_pt_create': (C.c_int, [C.POINTER(P6PtProblem), C.c_int, C.POINTER(C.c_void_p)]),
    'p6_pt_destroy': (C.c_int, [_P]),
    'p6_pt_costs': (C.c_int, [_P, _P, C.c_int, _P, _P]),
    'p6_pt_initial': (C.c_int, [_P, _P, C.c_int]),
    'p6_pt_batch': (C.c_int, [_P, C.c_int, C.c_int]),
    'p6_pt_read_state': (C.c_int, [_P, _P, _P, _P, _P, _P]),
    'p6_pt_synchronize': (C.c_int, [_P, C.c_double]),
    'p6_pt_last_batch_ms': (C.c_int, [_P, C.POINTER(C.c_float)]),
    'p6_pt_launch_count': (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    'p6_pt_set_trace': (C.c_int, [_P, C.c_int]),
    'p6_pt_read_trace': (C.c_int, [_P, _P]),
    'p6_pt_set_split': (C.c_int, [_P, C.c_int]),
    'p6_pt_get_split': (C.c_int, [_P, C.POINTER(C.c_int)]),
    'p6_pt_costs_static': (C.c_int, [_P, _P, C.c_int, _P, _P]),
    'p6_pt_vector_capacity': (C.c_int, [_P, C.POINTER(C.c_int)]),
    'p6_pt_model_costs': (C.c_int, [_P, _P, C.c_int, _P]),
    'p6_pt_normal': (C.c_int, [_P, _P, _P, _P, C.POINTER(C.c_double)]),
    'p6_pt_linear_start': (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    'p6_pt_lm': (C.c_int, [_P, _P, C.c_int, C.c_double, _P]),
    'p6_wy_batch_create': (C.c_int, [_P, C.c_int, C.POINTER(C.c_void_p)]),
    'p6_wy_batch_destroy': (C.c_int, [_P]),
    'p6_wy_batch_set_launch': (C.c_int, [_P, C.c_int, C.c_int]),
    'p6_wy_batch_query': (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_longlong)]),
    'p6_wy_batch_run': (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int]),
    'p6_wy_batch_synchronize': (C.c_int, [_P, C.c_double]),
    'p6_wy_batch_last_ms': (C.c_int, [_P, C.POINTER(C.c_float)]),
    'p6_mlp_create': (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]),
    'p6_mlp_destroy': (C.c_int, [_P]),
    'p6_mlp_params': (C.c_int, [_P, _P, _P, C.POINTER(C.c_longlong)]),
    'p6_mlp_gradients': (C.c_int, [_P, _P, _P, _P, C.c_int, _P, C.POINTER(C.c_float)]),
    'p6_mlp_train': (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint32, _P]),
    'p6_mlp_predict': (C.c_int, [_P, _P, C.c_int, _P]),
    'p6_wy_learned_step': (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P]),
    'p6_wy_time_mark': (C.c_int, [_P, C.c_int]),
    'p6_ct_create': (C.c_int, [C.POINTER(P6CtProblem), C.c_int, C.POINTER(C.c_void_p)]),
    'p6_ct_destroy': (C.c_int, [_P]),
    'p6_ct_set_intensities': (C.c_int, [_P, _P, C.c_int]),
    'p6_ct_evaluate': (C.c_int, [_P, C.c_int, C.c_int]),
    'p6_ct_read': (C.c_int, [_P, _P, _P]),
    'p6_ct_run_host': (C.c_int, [_P, _P, C.c_int, C.c_int, _P]),
    'p6_ct_synchronize': (C.c_int, [_P]),
    'p6_ct_last_ms': (C.c_int, [_P, C.POINTER(C.c_float)]),
    'p6_ct_query': (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                              C.POINTER(C.c_longlong)]),
    'p6_ct_set_fitted': (C.c_int, [_P, C.c_int]),
    'p6_ct_read_scale': (C.c_int, [_P, _P]),
    'p6_wy_profile_run': (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    'p6_wy_set_profile': (C.c_int, [_P, _P, _P, C.c_int, C.c_double]),
    'p6_cf_create': (C.c_int, [_P, C.c_int, _P, C.c_int, C.POINTER(C.c_void_p)]),
    'p6_cf_destroy': (C.c_int, [_P]),
    'p6_cf_set_grid': (C.c_int, [_P, C.c_int, _P]),
    'p6_cf_run': (C.c_int, [_P, C.c_int, _P]),
    'p6_cf_best_r': (C.c_int, [_P, _P]),
    'p6_cf_read': (C.c_int, [_P, C.c_int, C.c_int, _P]),
    'p6_cf_last_ms': (C.c_int, [_P, C.POINTER(C.c_float)]),
    'p6_cf_launch_count': (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    'p6_cf_time_kernels': (C.c_int, [_P, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
}

_lib = None


def load(build_if_missing: bool = True):
    """Load libp6cuda.so; builds it in-tree when missing and nvcc is present."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() and build_if_missing:
        from . import build as _build
        try:
            _build.build()
        except Exception as e:  # no toolchain on this machine
            raise P6Error(7, f'libp6cuda.so is missing and could not be built: {e}') from e
    if not LIB_PATH.exists():
        raise P6Error(7, f'libp6cuda.so not found at {LIB_PATH}')
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols():
    return list(_SIGS)


def check(status: int):
    if status != P6_OK:
        msg = load().p6_last_error()
        raise P6Error(status, msg.decode() if msg else '')


def ptr(a):
    """numpy array -> void* (None passes NULL)."""
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)
