"""The C-ABI library loads on a machine without a GPU, exports every entry point that
include/mpsw.h declares, and its host-side logic (scalars, variable table, allocation shapes,
error reporting) works without touching the device."""
import ctypes
import os
import re

import numpy as np

from mpsw import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include', 'mpsw.h')


def declared():
    src = open(HEADER).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(mpsw_[a-z0-9_]+)\s*\(', src)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SIGNATURES)


def test_handle_host_logic_without_device():
    h = _lib.Handle()
    L = h.lib
    v = ctypes.c_double()
    h.check(L.mpsw_get_scalar(h.ptr, b'config_apvm_upwinding', ctypes.byref(v)), 'get')
    assert v.value == 0.5                      # src/mpas_sw_module.f90:41
    h.check(L.mpsw_get_scalar(h.ptr, b'A', ctypes.byref(v)), 'get')
    assert v.value == 6371229.0                # case-insensitive, src/mpas_sw_module.f90:9
    assert L.mpsw_set_scalar(h.ptr, b'gravity', 1.0) != 0     # parameters are read-only
    assert b'parameter' in L.mpsw_last_error(h.ptr)
    assert L.mpsw_get_scalar(h.ptr, b'no_such_thing', ctypes.byref(v)) != 0
    assert L.mpsw_var_allocation(h.ptr) != 0   # dimensions not set yet
    for k, n in (('ncells', 42), ('nedges', 120), ('nvertices', 80), ('maxedges', 6),
                 ('maxedges2', 12), ('vertexdegree', 3), ('ntracers', 1)):
        h.check(L.mpsw_set_scalar(h.ptr, k.encode(), n), k)
    h.check(L.mpsw_var_allocation(h.ptr), 'alloc')
    rank, alloc, is_int = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dims = (ctypes.c_longlong * 4)()
    h.check(L.mpsw_var_info(h.ptr, b'u', ctypes.byref(rank), dims, ctypes.byref(is_int), ctypes.byref(alloc)), 'info')
    assert (rank.value, dims[0], dims[1], dims[2], is_int.value, alloc.value) == (3, 2, 1, 120, 0, 1)
    h.check(L.mpsw_var_info(h.ptr, b'edgesOnEdge', ctypes.byref(rank), dims, ctypes.byref(is_int), ctypes.byref(alloc)), 'info')
    assert (rank.value, dims[0], dims[1], is_int.value) == (2, 12, 120, 1)
    h.check(L.mpsw_var_info(h.ptr, b'u_tl', ctypes.byref(rank), dims, ctypes.byref(is_int), ctypes.byref(alloc)), 'info')
    assert alloc.value == 0                    # var_allocation_tlm not called
    x = np.arange(240, dtype=np.float64)
    h.check(L.mpsw_set_var(h.ptr, b'u', x.ctypes.data_as(ctypes.c_void_p), 240), 'set')
    y = np.zeros(240)
    h.check(L.mpsw_get_var(h.ptr, b'u', y.ctypes.data_as(ctypes.c_void_p), 240), 'get')
    assert np.array_equal(x, y)
    assert L.mpsw_set_var(h.ptr, b'u', x.ctypes.data_as(ctypes.c_void_p), 239) != 0
    assert b'count' in L.mpsw_last_error(h.ptr)
    # routines that need the mesh fail with a status, never abort
    assert L.mpsw_sw_rk4(h.ptr, 1) != 0
    assert L.mpsw_window_tl(h.ptr, 0, 1, None, None, None) != 0
    h.close()


def test_variable_table_matches_reference_module():
    L = _lib.load()
    names = {L.mpsw_var_name(i).decode() for i in range(L.mpsw_var_count())}
    for n in ('u', 'h', 'tracers', 'coeffs_reconstruct', 'uReconstructZonal_ad', 'gradPVt_tl',
              'tend_u_ad', 'kiteAreasOnVertex', 'deriv_two', 'boundaryEdge'):
        assert n in names, n
    assert L.mpsw_var_name(-1) is None


def _load_small_mesh(h, level=2):
    """A valid level-2 mesh loaded through the C ABI (host only)."""
    from helpers import mesh
    m = mesh(level)
    L = h.lib
    for k, n in (('ncells', m['nCells']), ('nedges', m['nEdges']), ('nvertices', m['nVertices']),
                 ('maxedges', m['maxEdges']), ('maxedges2', m['maxEdges2']), ('vertexdegree', 3), ('ntracers', 1)):
        h.check(L.mpsw_set_scalar(h.ptr, k.encode(), n), k)
    h.check(L.mpsw_var_allocation(h.ptr), 'alloc')
    arrays = {}
    for name in ('cellsOnEdge', 'verticesOnEdge', 'edgesOnEdge', 'nEdgesOnEdge', 'edgesOnCell', 'nEdgesOnCell',
                 'cellsOnVertex', 'edgesOnVertex', 'cellsOnCell', 'verticesOnCell', 'weightsOnEdge', 'dcEdge',
                 'dvEdge', 'areaCell', 'areaTriangle', 'kiteAreasOnVertex', 'xCell', 'yCell', 'zCell', 'xEdge',
                 'yEdge', 'zEdge', 'xVertex', 'yVertex', 'zVertex', 'latCell', 'lonCell', 'latEdge', 'lonEdge',
                 'latVertex', 'lonVertex', 'angleEdge', 'meshDensity'):
        a = np.ascontiguousarray(m[name], dtype=np.int32 if name[0] in 'cvne' and 'On' in name else np.float64)
        arrays[name] = a
        h.check(L.mpsw_set_var(h.ptr, name.encode(), a.ctypes.data_as(ctypes.c_void_p), a.size), name)
    return m, arrays


def test_corrupt_mesh_is_refused_with_mesh_status():
    """sw_mpas_init_block validates the mesh on the host before anything reaches a device: an
    out-of-range index or an inconsistent count returns MPSW_ERR_MESH (3) with a message naming
    the problem, instead of the reference's unchecked reads."""
    MPSW_ERR_MESH = 3
    h = _lib.Handle()
    _load_small_mesh(h)
    rc = h.lib.mpsw_sw_mpas_init_block(h.ptr)  # the intact mesh passes validation (then needs a GPU)
    assert rc != MPSW_ERR_MESH, h.lib.mpsw_last_error(h.ptr)
    h.close()
    for name, corrupt in (('cellsOnEdge', lambda a, m: a.__setitem__((5, 0), m['nCells'] + 7)),
                          ('edgesOnEdge', lambda a, m: a.__setitem__((3, 2), 0)),
                          ('nEdgesOnCell', lambda a, m: a.__setitem__(4, 9))):
        h = _lib.Handle()
        m, arrays = _load_small_mesh(h)
        a = arrays[name].copy()
        corrupt(a, m)
        h.check(h.lib.mpsw_set_var(h.ptr, name.encode(), a.ctypes.data_as(ctypes.c_void_p), a.size), name)
        rc = h.lib.mpsw_sw_mpas_init_block(h.ptr)
        assert rc == MPSW_ERR_MESH, (name, rc, h.lib.mpsw_last_error(h.ptr))
        assert h.lib.mpsw_last_error(h.ptr)
        h.close()
