"""ctypes binding of ``libmpsw.so`` (C ABI declared in include/mpsw.h).

There is no fallback: if the library is missing or a call fails, a RuntimeError says why.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the library built in place by build.py; MPSW_LIB names another build of it
LIB_PATH = os.environ.get('MPSW_LIB') or os.path.join(PKG_DIR, 'libmpsw.so')

_c_int, _c_double, _vp, _cp, _ll = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                    ctypes.c_char_p, ctypes.c_longlong)

# name -> (restype, argtypes)
SIGNATURES = {
    'mpsw_create': (_c_int, [ctypes.POINTER(_vp)]),
    'mpsw_destroy': (None, [_vp]),
    'mpsw_last_error': (_cp, [_vp]),
    'mpsw_version': (_cp, []),
    'mpsw_set_scalar': (_c_int, [_vp, _cp, _c_double]),
    'mpsw_get_scalar': (_c_int, [_vp, _cp, ctypes.POINTER(_c_double)]),
    'mpsw_var_count': (_c_int, []),
    'mpsw_var_name': (_cp, [_c_int]),
    'mpsw_var_info': (_c_int, [_vp, _cp, ctypes.POINTER(_c_int), ctypes.POINTER(_ll),
                               ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)]),
    'mpsw_set_var': (_c_int, [_vp, _cp, _vp, _ll]),
    'mpsw_get_var': (_c_int, [_vp, _cp, _vp, _ll]),
    'mpsw_var_allocation': (_c_int, [_vp]),
    'mpsw_var_allocation_tlm': (_c_int, [_vp]),
    'mpsw_var_allocation_adj': (_c_int, [_vp]),
    'mpsw_sw_mpas_init_block': (_c_int, [_vp]),
    'mpsw_sw_rk4': (_c_int, [_vp, _c_int]),
    'mpsw_sw_rk4_tlm': (_c_int, [_vp, _c_int]),
    'mpsw_sw_rk4_adj': (_c_int, [_vp]),
    'mpsw_solve_diagnostics': (_c_int, [_vp]),
    'mpsw_compute_tend': (_c_int, [_vp]),
    'mpsw_reconstruct_2d': (_c_int, [_vp]),
    'mpsw_solve_diagnostics_tlm': (_c_int, [_vp]),
    'mpsw_compute_tend_tlm': (_c_int, [_vp]),
    'mpsw_reconstruct_2d_tlm': (_c_int, [_vp]),
    'mpsw_adjoint_at_state': (_c_int, [_vp]),
    'mpsw_to_internal': (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    'mpsw_to_reference': (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    'mpsw_forward': (_c_int, [_vp, _c_int, _c_int]),
    'mpsw_grid_to_points': (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp, _ll, _vp, _vp, _vp, _vp]),
    'mpsw_get_stream': (_c_int, [_vp, ctypes.POINTER(_vp)]),
    'mpsw_window_init': (_c_int, [_vp, _c_int, _c_int, _vp]),
    'mpsw_window_storage': (_c_int, [_vp, _c_int, ctypes.c_double]),
    'mpsw_window_tuning': (_c_int, [_vp, _c_int, _c_int, ctypes.POINTER(_c_int)]),
    'mpsw_sw_test_case': (_c_int, [_vp, _c_int]),
    'mpsw_window_snapshots': (_c_int, [_vp, _c_int]),
    'mpsw_window_forward_steps': (_c_int, [_vp, ctypes.POINTER(_ll)]),
    'mpsw_window_fused': (_c_int, [_vp, _c_int, _c_int, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)]),
    'mpsw_window_tl': (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    'mpsw_window_ad': (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    'mpsw_window_final_state': (_c_int, [_vp, _vp, _vp, _vp]),
    'mpsw_state_from_device': (_c_int, [_vp, _vp, _vp, _vp]),
    'mpsw_state_to_device': (_c_int, [_vp, _vp, _vp, _vp]),
    'mpsw_launch_count': (_ll, []),
    'mpsw_compute_tend_noalloc': (_c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    'mpsw_time_kernel': (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_c_double)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libmpsw.so (built by build.py) and declare every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'{LIB_PATH} is missing: build it with `python build.py` '
                           f'(or __graft_entry__.build()); there is no CPU fallback')
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class Handle:
    """Owner of one ``mpsw_handle`` (one module instance)."""

    def __init__(self):
        L = load()
        h = ctypes.c_void_p()
        rc = L.mpsw_create(ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f'mpsw_create failed ({rc}): {L.mpsw_last_error(None).decode()}')
        self.lib = L
        self.ptr = h

    def close(self):
        if self.ptr:
            self.lib.mpsw_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc, what):
        if rc != 0:
            msg = self.lib.mpsw_last_error(self.ptr).decode()
            raise RuntimeError(f'{what} failed ({rc}): {msg}')

    def call(self, name, *args):
        self.check(getattr(self.lib, name)(self.ptr, *args), name)
