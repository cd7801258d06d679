"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

``OracleModule`` mimics the attribute surface of the reference's f2py object
``module_sw_mpas.mpas_sw_module``: lower-case attribute names, Fortran-ordered numpy arrays
with the shapes ``var_allocation*`` gives them (``src/mpas_sw_module.f90:211-493``), 1-based
index arrays, whole-array assignment that (re)allocates, and argument-less subroutines.  The
numerics run in ``_build/liboracle.so`` (``sw_oracle.c``), a line-by-line FP64 restatement of
the reference Fortran.  Only tests, the smoke check and the benchmark's CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, '_build', 'liboracle.so')

# module constants, src/mpas_sw_module.f90:8-18
CONSTANTS = {'pii': 3.141592653589793, 'a': 6371229.0, 'omega': 7.29212e-5, 'gravity': 9.80616,
             'rgas': 287.0, 'rv': 461.6}


def build():
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(['make', '-s', '-C', _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_name.restype = ctypes.c_char_p
        L.orc_name.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_count.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _names(kind):
    L = lib()
    return [L.orc_name(kind, i).decode() for i in range(L.orc_count(kind))]


class _OrcMod(ctypes.Structure):
    pass


def _struct_type():
    nr, ni, nis, nrs = (len(_names(k)) for k in range(4))
    if not getattr(_OrcMod, '_fields_', None):
        _OrcMod._fields_ = [('r', ctypes.c_void_p * nr), ('i', ctypes.c_void_p * ni),
                            ('is_', ctypes.c_int * nis), ('rs', ctypes.c_double * nrs)]
    return _OrcMod


def _shapes(d):
    """Allocation shapes of var_allocation / _tlm / _adj (src/mpas_sw_module.f90:211-493)."""
    nC, nE, nV = d['ncells'], d['nedges'], d['nvertices']
    nL, nT, mE, mE2, vd, R3 = (d['nvertlevels'], d['ntracers'], d['maxedges'], d['maxedges2'],
                               d['vertexdegree'], d['r3'])
    base = {
        'u': (2, nL, nE), 'h': (2, nL, nC), 'tracers': (2, nT, nL, nC),
        'u_src': (nL, nE), 'h_s': (nC,), 'fCell': (nC,), 'fVertex': (nV,), 'fEdge': (nE,),
        'areaTriangle': (nV,), 'areaCell': (nC,), 'dvEdge': (nE,), 'dcEdge': (nE,),
        'weightsOnEdge': (mE2, nE), 'kiteAreasOnVertex': (vd, nV), 'meshDensity': (nC,),
        'boundaryCell': (nL, nC), 'boundaryEdge': (nL, nE), 'advCells': (21, nC),
        'cellsOnCell': (mE, nC), 'cellsOnEdge': (2, nE), 'cellsOnVertex': (vd, nV),
        'edgesOnCell': (mE, nC), 'edgesOnEdge': (mE2, nE), 'edgesOnVertex': (vd, nV),
        'verticesOnCell': (mE, nC), 'verticesOnEdge': (2, nE), 'nEdgesOnCell': (nC,),
        'nEdgesOnEdge': (nE,), 'latCell': (nC,), 'lonCell': (nC,), 'xCell': (nC,),
        'yCell': (nC,), 'zCell': (nC,), 'meshScalingDel2': (nE,), 'meshScalingDel4': (nE,),
        'deriv_two': (15, 2, nE), 'latEdge': (nE,), 'lonEdge': (nE,), 'xEdge': (nE,),
        'yEdge': (nE,), 'zEdge': (nE,), 'angleEdge': (nE,), 'latVertex': (nV,),
        'lonVertex': (nV,), 'xVertex': (nV,), 'yVertex': (nV,), 'zVertex': (nV,),
        'defc_a': (mE, nC), 'defc_b': (mE, nC), 'localVerticalUnitVectors': (R3, nC),
        'edgeNormalVectors': (R3, nE), 'cellTangentPlane': (R3, 2, nC),
        'coeffs_reconstruct': (R3, mE, nC),
        'tend_u': (nL, nE), 'tend_h': (nL, nC), 'tend_tracer': (nT, nL, nC),
    }
    diag = {'uReconstructX': nC, 'uReconstructY': nC, 'uReconstructZ': nC,
            'uReconstructZonal': nC, 'uReconstructMeridional': nC, 'v': nE, 'h_edge': nE,
            'h_vertex': nV, 'pv_edge': nE, 'pv_vertex': nV, 'pv_cell': nC, 'circulation': nV,
            'vorticity': nV, 'divergence': nC, 'ke': nC, 'vh': nE, 'vorticity_cell': nC,
            'gradPVn': nE, 'gradPVt': nE}
    for k, n in diag.items():
        base[k] = (nL, n)
    tl = {'u_tl': (2, nL, nE), 'h_tl': (2, nL, nC), 'tracers_tl': (2, nT, nL, nC),
          'tend_u_tl': (nL, nE), 'tend_h_tl': (nL, nC), 'tend_tracer_tl': (nT, nL, nC)}
    ad = {'u_ad': (2, nL, nE), 'h_ad': (2, nL, nC), 'tracers_ad': (2, nT, nL, nC),
          'tend_u_ad': (nL, nE), 'tend_h_ad': (nL, nC), 'tend_tracer_ad': (nT, nL, nC)}
    for k, n in diag.items():
        tl[k + '_tl'] = (nL, n)
        ad[k + '_ad'] = (nL, n)
    return base, tl, ad


_INT_ARRAYS = {'boundaryCell', 'boundaryEdge', 'advCells', 'cellsOnCell', 'cellsOnEdge',
               'cellsOnVertex', 'edgesOnCell', 'edgesOnEdge', 'edgesOnVertex', 'verticesOnCell',
               'verticesOnEdge', 'nEdgesOnCell', 'nEdgesOnEdge'}

_SCALAR_DEFAULTS = {  # src/mpas_sw_module.f90:23-55
    'config_advect_tracers': 0,  # tracer transport switch (off: tracers carried, as the reference)
    'config_test_case': 5, 'config_dt': 150.0, 'config_stats_interval': 100,
    'config_h_ScaleWithMesh': False, 'config_h_mom_eddy_visc2': 0.0,
    'config_h_mom_eddy_visc4': 0.0, 'config_h_tracer_eddy_diff2': 0.0,
    'config_h_tracer_eddy_diff4': 0.0, 'config_thickness_adv_order': 2,
    'config_tracer_adv_order': 2, 'config_positive_definite': False, 'config_monotonic': False,
    'config_wind_stress': False, 'config_bottom_drag': False, 'config_apvm_upwinding': 0.5,
    'config_num_halos': 2, 'nVertLevels': 1, 'nCells': 0, 'nEdges': 0, 'nVertices': 0,
    'nTracers': 0, 'cellStart': 0, 'cellEnd': 0, 'vertexStart': 0, 'vertexEnd': 0,
    'edgeStart': 0, 'edgeEnd': 0, 'vertexDegree': 0, 'nCellsSolve': 0, 'nEdgesSolve': 0,
    'maxEdges': 0, 'maxEdges2': 0, 'cellSolveStart': 0, 'cellSolveEnd': 0,
    'edgeSolveStart': 0, 'edgeSolveEnd': 0, 'R3': 0, 'on_a_sphere': False,
    'is_periodic': False, 'x_period': 0.0, 'y_period': 0.0, 'sphere_radius': 0.0,
    'rk_step': 0, 'LHS': 0.0, 'RHS': 0.0, 'pt': 0.0,
}


class OracleModule:
    """Stand-in for ``mpas_sw_module`` backed by the C oracle."""

    def __init__(self):
        object.__setattr__(self, '_arr', {})
        object.__setattr__(self, '_sc', {k.lower(): v for k, v in _SCALAR_DEFAULTS.items()})
        object.__setattr__(self, '_canon', {})
        for k in _SCALAR_DEFAULTS:
            self._canon[k.lower()] = k
        for k in _names(0) + _names(1):
            self._canon[k.lower()] = k

    # ---- attribute surface -------------------------------------------------------------
    def __getattr__(self, name):
        key = name.lower()
        if key in CONSTANTS:
            return np.float64(CONSTANTS[key])
        arr = self.__dict__['_arr']
        if key in arr:
            return arr[key]
        sc = self.__dict__['_sc']
        if key in sc:
            return sc[key]
        if key in self.__dict__['_canon']:
            return None  # unallocated allocatable
        raise AttributeError(name)

    def __setattr__(self, name, value):
        key = name.lower()
        if key in CONSTANTS:
            raise AttributeError(f'{name} is a parameter')
        canon = self._canon.get(key)
        if canon is None:
            self._canon[key] = name
            canon = name
        if canon in _SCALAR_DEFAULTS or (np.ndim(value) == 0 and key not in self._arr):
            self._sc[key] = value.item() if hasattr(value, 'item') else value
            return
        dtype = np.int32 if canon in _INT_ARRAYS else np.float64
        self._arr[key] = np.array(value, dtype=dtype, order='F', copy=True)

    def _alloc(self, table):
        d = {k: int(self._sc[k]) for k in ('ncells', 'nedges', 'nvertices', 'nvertlevels',
                                           'ntracers', 'maxedges', 'maxedges2', 'vertexdegree',
                                           'r3')}
        for name, shape in table(d).items():
            dtype = np.int32 if name in _INT_ARRAYS else np.float64
            self._arr[name.lower()] = np.zeros(shape, dtype=dtype, order='F')

    def var_allocation(self):
        self._alloc(lambda d: _shapes(d)[0])

    def var_allocation_tlm(self):
        self._alloc(lambda d: _shapes(d)[1])

    def var_allocation_adj(self):
        self._alloc(lambda d: _shapes(d)[2])

    # ---- calls into C --------------------------------------------------------------------
    def _struct(self):
        S = _struct_type()
        s = S()
        keep = []
        for i, n in enumerate(_names(0)):
            a = self._arr.get(n.lower())
            if a is not None:
                if not (a.flags.f_contiguous and a.dtype == np.float64):
                    a = np.asfortranarray(a, dtype=np.float64)
                    self._arr[n.lower()] = a
                s.r[i] = a.ctypes.data
                keep.append(a)
        for i, n in enumerate(_names(1)):
            a = self._arr.get(n.lower())
            if a is not None:
                if not (a.flags.f_contiguous and a.dtype == np.int32):
                    a = np.asfortranarray(a, dtype=np.int32)
                    self._arr[n.lower()] = a
                s.i[i] = a.ctypes.data
                keep.append(a)
        for i, n in enumerate(_names(2)):
            s.is_[i] = int(bool(self._sc[n.lower()])) if isinstance(self._sc[n.lower()], bool) \
                else int(self._sc[n.lower()])
        for i, n in enumerate(_names(3)):
            s.rs[i] = float(self._sc[n.lower()])
        return s, keep

    def _call(self, fn, *extra):
        s, keep = self._struct()
        rc = getattr(lib(), fn)(ctypes.byref(s), *extra)
        if rc != 0:
            raise RuntimeError(f'oracle {fn} failed ({rc})')
        for i, n in enumerate(_names(2)):
            self._sc[n.lower()] = s.is_[i]
        for i, n in enumerate(_names(3)):
            self._sc[n.lower()] = s.rs[i]
        del keep

    def sw_mpas_init_block(self):
        self._call('orc_sw_mpas_init_block')

    def sw_rk4(self):
        self._call('orc_sw_rk4')

    def sw_rk4_tlm(self):
        self._call('orc_sw_rk4_tlm')

    def sw_rk4_adj(self):
        self._call('orc_sw_rk4_adj')

    def link_tlm_adj(self, verbose=False):
        """Reference's one-stage dot-product test; returns (LHS, RHS) instead of STOPping."""
        self._call('orc_link_tlm_adj', ctypes.c_int(1 if verbose else 0))
        return self._sc['lhs'], self._sc['rhs']

    def sw_test_case_1(self):
        self._call('orc_sw_test_case_1')

    def sw_test_case_2(self):
        self._call('orc_sw_test_case_2')

    def sw_test_case_5(self):
        self._call('orc_sw_test_case_5')

    def sw_test_case_6(self):
        self._call('orc_sw_test_case_6')

    # single-routine calls (level-1 state)
    def solve_diagnostics(self):
        self._call('orc_solve_diagnostics')

    def compute_tend(self):
        self._call('orc_compute_tend')

    def solve_diagnostics_tlm(self):
        self._call('orc_solve_diagnostics_tlm')

    def compute_scalar_tend(self):
        self._call('orc_compute_scalar_tend')

    def compute_tend_tlm(self):
        self._call('orc_compute_tend_tlm')

    def solve_diagnostics_adj(self):
        self._call('orc_solve_diagnostics_adj')

    def compute_tend_adj(self):
        self._call('orc_compute_tend_adj')

    def reconstruct_2d(self):
        self._call('orc_reconstruct_2d')


def load_mesh(mod, mesh: dict, ntracers: int = 1):
    """Do what ``read_dims`` + ``read_vars`` do (``src/mpas_sw_driver.py:33-119``) with a mesh
    dict laid out like the grid file (see ``mpsw.mesh``)."""
    mod.nvertlevels = 1
    mod.ncells = mesh['nCells']
    mod.nedges = mesh['nEdges']
    mod.nvertices = mesh['nVertices']
    mod.maxedges = mesh['maxEdges']
    mod.maxedges2 = mesh['maxEdges2']
    mod.vertexdegree = mesh['vertexDegree']
    mod.r3 = 3
    mod.ntracers = ntracers
    for k in ('ncellssolve', 'cellend', 'cellsolveend'):
        setattr(mod, k, mesh['nCells'])
    for k in ('nedgessolve', 'edgeend', 'edgesolveend'):
        setattr(mod, k, mesh['nEdges'])
    mod.var_allocation()
    mod.on_a_sphere = True
    mod.is_periodic = False
    mod.sphere_radius = 1.0
    for k in ('latCell', 'lonCell', 'xCell', 'yCell', 'zCell', 'latEdge', 'lonEdge', 'xEdge',
              'yEdge', 'zEdge', 'latVertex', 'lonVertex', 'xVertex', 'yVertex', 'zVertex',
              'cellsOnEdge', 'nEdgesOnCell', 'nEdgesOnEdge', 'edgesOnCell', 'edgesOnEdge',
              'weightsOnEdge', 'dvEdge', 'dcEdge', 'angleEdge', 'areaCell', 'areaTriangle',
              'cellsOnCell', 'verticesOnCell', 'verticesOnEdge', 'edgesOnVertex', 'cellsOnVertex',
              'kiteAreasOnVertex', 'meshDensity'):
        setattr(mod, k.lower(), np.asarray(mesh[k]).T)


def grid_to_points(lat1d, lon1d, grid, lat, lon):
    """Restatement of grid2mpas (src/grid2mpas.f90:21-70) for points whose longitudes are already
    in the axis range: for each point the first index of the minimum |axis - x| in latitude and
    in longitude (minloc, :53-63), the section of up to 3 x 3 values around them clamped at the
    axis ends, summed in Fortran element order (latitude fastest, :65-66) and divided by its
    size.  Loops over points in Python: small cases only."""
    lat1d, lon1d = np.asarray(lat1d, dtype=np.float64), np.asarray(lon1d, dtype=np.float64)
    grid = np.asarray(grid, dtype=np.float64)
    nlat, nlon = lat1d.size, lon1d.size
    out = np.empty(len(lat))
    for k, (y, x) in enumerate(zip(np.asarray(lat, dtype=np.float64), np.asarray(lon, dtype=np.float64))):
        i0 = int(np.argmin(np.abs(y - lat1d)))
        j0 = int(np.argmin(np.abs(x - lon1d)))
        i1, i2 = max(i0 - 1, 0), min(i0 + 1, nlat - 1)
        j1, j2 = max(j0 - 1, 0), min(j0 + 1, nlon - 1)
        s = 0.0
        for j in range(j1, j2 + 1):
            for i in range(i1, i2 + 1):
                s = s + float(grid[i, j])
        out[k] = s / float((i2 - i1 + 1) * (j2 - j1 + 1))
    return out
