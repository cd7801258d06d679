"""Drop-in replacement for the reference's f2py extension ``module_sw_mpas``.

The reference drivers do ``from module_sw_mpas import mpas_sw_module as mpsw``
(src/mpas_sw_driver.py:8, demo/run-*.py) and then

* set scalars and whole arrays as attributes (``mpsw.ncells = ...``,
  ``mpsw.cellsonedge = infile['cellsOnEdge'][()].T``),
* mutate arrays in place through attribute access (``mpsw.u[0, 0] = ...``,
  ``mpsw.xcell[()] *= mpsw.a``),
* call argument-less subroutines (``mpsw.sw_rk4()``), and
* read results back (``mpsw.h[0, 0].copy()``, ``mpsw.ureconstructzonal[0]``).

``mpas_sw_module`` below offers that surface over the B200 engine (libmpsw.so, C ABI in
include/mpsw.h).  Attribute names are case-insensitive like f2py's; arrays are Fortran-ordered
numpy arrays with the reference's shapes and 1-based index values.  The numerics run on the
GPU; there is no CPU fallback.

Synchronisation with the device follows the f2py view semantics as far as a host mirror can:

* before a subroutine runs, every state / adjoint-seed array it reads is sent if it changed
  since it was last exchanged (in-place edits included); mesh arrays are sent at
  ``sw_mpas_init_block`` and whenever an attribute is reassigned;
* after it runs, the prognostic arrays it wrote (u, h and their _tl/_ad) are copied back into
  the same numpy objects, so references held across the call see the new values; diagnostics,
  reconstructions and tendencies are refreshed when next accessed as attributes.

Differences from the reference, by design: ``link_tlm_adj`` returns ``(LHS, RHS)`` after
printing instead of STOPping the interpreter; misuse raises RuntimeError/ValueError with the
engine's message instead of crashing; only global (closed-sphere) meshes with nVertLevels = 1
and thickness_adv_order 2 are accepted (orders 3/4 are accepted while ``deriv_two`` is zero,
where they coincide with order 2, as in the reference whose deriv_two is never filled).

Extension: with ``config_advect_tracers = 1`` (default 0, the reference's behaviour of only
carrying the tracers) ``sw_rk4`` and ``sw_rk4_steps(n, 0)`` also transport ``tracers`` (MPAS's
order-2 scalar tendency with its mass-weighted RK4) and set ``tend_tracer``.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
if _HERE not in sys.path:
    sys.path.insert(0, _HERE)

from mpsw import testcases as _tc  # noqa: E402
from mpsw._lib import Handle as _Handle  # noqa: E402

_DIAG = ('uReconstructX', 'uReconstructY', 'uReconstructZ', 'uReconstructZonal',
         'uReconstructMeridional', 'v', 'h_edge', 'h_vertex', 'pv_edge', 'pv_vertex', 'pv_cell',
         'circulation', 'vorticity', 'divergence', 'ke', 'vh', 'vorticity_cell', 'gradPVn',
         'gradPVt')
_RECON = _DIAG[:5]
_STATE = ('u', 'h')

_ROUTINES = {'var_allocation', 'var_allocation_tlm', 'var_allocation_adj', 'sw_mpas_init_block',
             'sw_rk4', 'sw_rk4_tlm', 'sw_rk4_adj', 'link_tlm_adj', 'sw_test_case_1',
             'sw_test_case_2', 'sw_test_case_5', 'sw_test_case_6', 'solve_diagnostics',
             'compute_tend', 'reconstruct_2d', 'solve_diagnostics_tlm', 'compute_tend_tlm',
             'reconstruct_2d_tlm', 'adjoint_at_state'}


def _sfx(names, s):
    return tuple(n + s for n in names)


class MpasSwModule:
    """One shallow-water module instance (the f2py object ``mpas_sw_module``)."""

    def __init__(self):
        d = self.__dict__
        d['_h'] = _Handle()
        lib = d['_h'].lib
        names = [lib.mpsw_var_name(i).decode() for i in range(lib.mpsw_var_count())]
        d['_canon'] = {n.lower(): n for n in names}
        d['_arr'] = {}         # lower name -> ndarray (Fortran order)
        d['_synced'] = {}      # lower name -> copy of the content last exchanged with the engine
        d['_stale'] = set()    # lower names to refresh from the engine on next access
        d['_mesh_dirty'] = set()

    # ---- attribute surface ---------------------------------------------------------------
    def __getattr__(self, name):
        key = name.lower()
        d = self.__dict__
        if key in d['_canon']:
            if key in d['_stale']:
                self._pull(key)
            return d['_arr'].get(key)   # None while unallocated, as f2py
        v = ctypes.c_double()
        if d['_h'].lib.mpsw_get_scalar(d['_h'].ptr, key.encode(), ctypes.byref(v)) == 0:
            x = v.value
            return np.float64(x) if x != int(x) or key in _REAL_SCALARS else np.int64(int(x))
        raise AttributeError(name)

    def __setattr__(self, name, value):
        key = name.lower()
        d = self.__dict__
        if key in d['_canon']:
            arr = d['_arr'].get(key)
            if arr is None:
                raise ValueError(f'{name} is not allocated (call var_allocation first)')
            val = np.asarray(value)
            if val.size != arr.size:
                raise ValueError(f'{name}: shape {val.shape} does not match the allocated {arr.shape}')
            arr[...] = val.reshape(arr.shape, order='F') if val.shape != arr.shape else val
            d['_stale'].discard(key)
            if key not in d['_synced']:
                d['_mesh_dirty'].add(key)
            return
        if isinstance(value, (bool, np.bool_)):
            value = 1.0 if value else 0.0
        d['_h'].check(d['_h'].lib.mpsw_set_scalar(d['_h'].ptr, key.encode(), float(value)),
                      f'setting {name}')

    def __dir__(self):
        return sorted(set(self.__dict__['_canon']) | _ROUTINES)

    # ---- host <-> engine -------------------------------------------------------------------
    def _push(self, key, force=False):
        d = self.__dict__
        arr = d['_arr'][key]
        last = d['_synced'].get(key)
        if not force and last is not None and np.array_equal(last, arr):
            return
        ptr = arr.ctypes.data_as(ctypes.c_void_p)
        d['_h'].call('mpsw_set_var', d['_canon'][key].encode(), ptr, arr.size)
        if last is not None or key in _TRACKED:
            d['_synced'][key] = arr.copy(order='F')

    def _pull(self, key):
        d = self.__dict__
        arr = d['_arr'][key]
        d['_h'].call('mpsw_get_var', d['_canon'][key].encode(), arr.ctypes.data_as(ctypes.c_void_p),
                     arr.size)
        d['_stale'].discard(key)
        if key in d['_synced']:
            d['_synced'][key] = arr.copy(order='F')

    def _push_mesh(self, everything=False):
        d = self.__dict__
        keys = [k for k in d['_arr'] if k not in _TRACKED] if everything else list(d['_mesh_dirty'])
        for k in keys:
            if k in d['_arr'] and k not in d['_stale']:
                self._push(k, force=True)
        d['_mesh_dirty'].clear()

    def _run(self, routine, *args, reads=(), eager=(), lazy=()):
        d = self.__dict__
        self._push_mesh()
        for k in reads:
            k = k.lower()
            if k in d['_arr'] and k not in d['_stale']:
                self._push(k)
        try:
            d['_h'].call(routine, *args)
        except RuntimeError:
            # a routine that failed part-way may have written its outputs on the device: the
            # host copies of them are no longer current, so the next read fetches them
            for k in tuple(eager) + tuple(lazy):
                if k.lower() in d['_arr']:
                    d['_stale'].add(k.lower())
            raise
        for k in eager:
            k = k.lower()
            if k in d['_arr']:
                self._pull(k)
        for k in lazy:
            k = k.lower()
            if k in d['_arr']:
                d['_stale'].add(k)

    # ---- module subroutines ------------------------------------------------------------------
    def _allocate(self, routine, group):
        d = self.__dict__
        d['_h'].call(routine)
        lib = d['_h'].lib
        for lname, canon in d['_canon'].items():
            rank, alloc, is_int = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            dims = (ctypes.c_longlong * 4)()
            d['_h'].check(lib.mpsw_var_info(d['_h'].ptr, canon.encode(), ctypes.byref(rank), dims,
                                            ctypes.byref(is_int), ctypes.byref(alloc)), 'var_info')
            if not alloc.value or _group(canon) != group:
                continue
            shape = tuple(dims[i] for i in range(rank.value))
            d['_arr'][lname] = np.zeros(shape, dtype=np.int32 if is_int.value else np.float64, order='F')
            d['_stale'].discard(lname)
            if lname in _TRACKED:
                d['_synced'][lname] = d['_arr'][lname].copy(order='F')
            else:
                d['_mesh_dirty'].add(lname)

    def var_allocation(self):
        self._allocate('mpsw_var_allocation', 0)

    def var_allocation_tlm(self):
        self._allocate('mpsw_var_allocation_tlm', 1)

    def var_allocation_adj(self):
        self._allocate('mpsw_var_allocation_adj', 2)

    def sw_mpas_init_block(self):
        self._push_mesh(everything=True)
        self._run('mpsw_sw_mpas_init_block', reads=_STATE, lazy=_DIAG)
        for k in ('meshscalingdel2', 'meshscalingdel4', 'localverticalunitvectors',
                  'edgenormalvectors', 'celltangentplane', 'coeffs_reconstruct'):
            self._pull(k)

    def _tracers_advected(self):
        return bool(self.config_advect_tracers) and self.__dict__['_arr'].get('tracers') is not None

    def sw_rk4(self):
        adv = self._tracers_advected()
        tr = ('tracers',) if adv else ()
        self._run('mpsw_sw_rk4', 1, reads=_STATE + tr, eager=_STATE + tr,
                  lazy=_DIAG + ('tend_u', 'tend_h') + (('tend_tracer',) if adv else ()))
        arr = self.__dict__['_arr'].get('tracers')
        if arr is not None and not adv:
            arr[1] = arr[0]
        self.rk_step = 5

    def sw_rk4_steps(self, nsteps, precision=0):
        """``nsteps`` calls of sw_rk4 in one device call (no counterpart in the reference).
        precision 0 is bit-identical to repeated sw_rk4; precision 1 runs the stencils in FP32
        and keeps the state and its RK4 accumulation in FP64 (tend_u / tend_h are then left
        as they were)."""
        adv = self._tracers_advected()
        tr = ('tracers',) if adv else ()
        self._run('mpsw_forward', int(precision), int(nsteps), reads=_STATE + tr, eager=_STATE + tr,
                  lazy=_DIAG + (('tend_u', 'tend_h') + (('tend_tracer',) if adv else ())
                                if int(precision) == 0 else ()))
        arr = self.__dict__['_arr'].get('tracers')
        if arr is not None and nsteps > 0 and not adv:
            arr[1] = arr[0]
        if nsteps > 0:
            self.rk_step = 5

    def sw_rk4_tlm(self):
        self._run('mpsw_sw_rk4_tlm', 1, reads=_STATE + _sfx(_STATE, '_tl'),
                  eager=_STATE + _sfx(_STATE, '_tl'),
                  lazy=_DIAG + _sfx(_DIAG, '_tl') + ('tend_u', 'tend_h', 'tend_u_tl', 'tend_h_tl'))
        self.rk_step = 5

    def sw_rk4_adj(self):
        self._run('mpsw_sw_rk4_adj', reads=_STATE + _sfx(_STATE, '_ad') + _sfx(_DIAG, '_ad')
                  + ('tend_u_ad', 'tend_h_ad'),
                  eager=_STATE + _sfx(_STATE, '_ad'),
                  lazy=_DIAG + _sfx(_DIAG, '_ad') + ('tend_u_ad', 'tend_h_ad'))
        self.rk_step = 0

    def solve_diagnostics(self):
        self._run('mpsw_solve_diagnostics', reads=_STATE, lazy=_DIAG[5:])

    def compute_tend(self):
        self._run('mpsw_compute_tend', reads=_STATE, lazy=_DIAG[5:] + ('tend_u', 'tend_h'))

    def reconstruct_2d(self):
        self._run('mpsw_reconstruct_2d', reads=_STATE, lazy=_RECON)

    def solve_diagnostics_tlm(self):
        self._run('mpsw_solve_diagnostics_tlm', reads=_STATE + _sfx(_STATE, '_tl'),
                  lazy=_DIAG[5:] + _sfx(_DIAG[5:], '_tl'))

    def compute_tend_tlm(self):
        self._run('mpsw_compute_tend_tlm', reads=_STATE + _sfx(_STATE, '_tl'),
                  lazy=_DIAG[5:] + _sfx(_DIAG[5:], '_tl') + ('tend_u', 'tend_h', 'tend_u_tl', 'tend_h_tl'))

    def reconstruct_2d_tlm(self):
        self._run('mpsw_reconstruct_2d_tlm', reads=_STATE + _sfx(_STATE, '_tl'),
                  lazy=_RECON + _sfx(_RECON, '_tl'))

    def adjoint_at_state(self):
        self._run('mpsw_adjoint_at_state', reads=_STATE + _sfx(_STATE, '_ad') + _sfx(_DIAG, '_ad')
                  + ('tend_u_ad', 'tend_h_ad'),
                  eager=_sfx(_STATE, '_ad'), lazy=_sfx(_DIAG, '_ad') + ('tend_u_ad', 'tend_h_ad'))

    def link_tlm_adj(self, verbose=True):
        """One-stage dot-product test of src/mpas_sw_module.f90:1006-1218.

        The caller sets u_tl(1) = u(1)*pt and h_tl(1) = h(1)*pt with pt = 1e-3, as the reference
        expects.  Prints LHS, RHS and their relative differences and returns (LHS, RHS)
        instead of stopping the interpreter.
        """
        pt = 1.E-3
        self.pt = pt
        rks1 = float(self.config_dt) / 2.
        self.solve_diagnostics_tlm()
        self.reconstruct_2d_tlm()
        self.compute_tend_tlm()
        u, h, ut, ht = self.u, self.h, self.u_tl, self.h_tl
        uPt = ut[0, 0] + rks1 * self.tend_u_tl[0]
        hPt = ht[0, 0] + rks1 * self.tend_h_tl[0]
        ut[1] = ut[0]
        ht[1] = ht[0]
        u[1] = u[0]
        h[1] = h[0]
        terms = [uPt, hPt, self.tend_h_tl, self.tend_u_tl, ut[1], ht[1]]
        terms += [getattr(self, n.lower() + '_tl') for n in _DIAG[5:] if n != 'vh']
        terms += [getattr(self, n.lower() + '_tl') for n in _RECON]
        LHS = 0.0
        for t in terms:
            LHS = LHS + float(np.sum(np.asarray(t) ** 2))
        # adjoint seeds are the tangent-linear outputs (:1112-1135)
        self.tend_h_ad = self.tend_h_tl + rks1 * hPt
        self.tend_u_ad = self.tend_u_tl + rks1 * uPt
        ua, ha = self.u_ad, self.h_ad
        ua[1] = ut[1]
        ha[1] = ht[1]
        for n in _DIAG[5:] + _RECON:
            if n != 'vh':
                setattr(self, n.lower() + '_ad', getattr(self, n.lower() + '_tl'))
        ha[0, 0] += hPt
        ua[0, 0] += uPt
        self.adjoint_at_state()
        ua, ha = self.u_ad, self.h_ad
        ha[0] += ha[1]
        ha[1] = 0.
        ua[0] += ua[1]
        ua[1] = 0.
        RHS = float(np.sum(ua[0] * u[0] * pt)) + float(np.sum(ha[0] * h[0] * pt))
        self.lhs = LHS
        self.rhs = RHS
        if verbose:
            print(LHS)
            print(RHS)
            print((LHS - RHS) / LHS)
            print((LHS - RHS) / RHS)
        return LHS, RHS

    def sw_test_case_1(self):
        _tc.test_case_1(self)

    def sw_test_case_2(self):
        _tc.test_case_2(self)

    def sw_test_case_5(self):
        _tc.test_case_5(self)

    def sw_test_case_6(self):
        _tc.test_case_6(self)

    def sw_test_case_device(self, tc):
        """Williamson test case ``tc`` (1, 2, 5 or 6) set up by GPU kernels instead of on the host
        (no counterpart in the reference, whose sw_test_case_* this mirrors): the same fields as
        sw_test_case_<tc>, to the last bit or two of the device's sin / cos / pow."""
        scaled = ('xcell', 'ycell', 'zcell', 'xvertex', 'yvertex', 'zvertex', 'xedge', 'yedge', 'zedge',
                  'dvedge', 'dcedge', 'areacell', 'areatriangle', 'kiteareasonvertex')
        out = scaled + ('u', 'h', 'fedge', 'fvertex', 'h_s', 'loncell', 'tracers')
        self._run('mpsw_sw_test_case', int(tc), reads=('u', 'h', 'tracers'), eager=out)

    # ---- access to the engine for the device-resident API -----------------------------------
    @property
    def handle(self):
        """The underlying engine handle (mpsw._lib.Handle)."""
        return self.__dict__['_h']

    def sync(self):
        """Send every pending host change to the engine (mesh and state)."""
        self._push_mesh()
        for k in list(self.__dict__['_synced']):
            if k not in self.__dict__['_stale']:
                self._push(k)


_REAL_SCALARS = {'config_dt', 'config_h_mom_eddy_visc2', 'config_h_mom_eddy_visc4',
                 'config_h_tracer_eddy_diff2', 'config_h_tracer_eddy_diff4',
                 'config_apvm_upwinding', 'x_period', 'y_period', 'sphere_radius', 'lhs', 'rhs',
                 'pt', 'pii', 'a', 'omega', 'gravity', 'rgas', 'rv', 'rvord', 'cp', 'cv', 'cvpm',
                 'prandtl'}

# arrays exchanged with change detection: prognostic state, adjoint seeds and tendencies
_TRACKED = set(n.lower() for n in _STATE + _sfx(_STATE, '_tl') + _sfx(_STATE, '_ad')
               + _sfx(_DIAG, '_ad') + _DIAG + _sfx(_DIAG, '_tl')
               + ('tend_u', 'tend_h', 'tend_u_tl', 'tend_h_tl', 'tend_u_ad', 'tend_h_ad'))


def _group(canon):
    c = canon.lower()
    if c.endswith('_tl'):
        return 1
    if c.endswith('_ad'):
        return 2
    return 0


mpas_sw_module = MpasSwModule()
