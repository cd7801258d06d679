"""Shared set-up for the tests: the same mesh and initial state loaded into the oracle and into
the engine-backed module, through the reference driver's attribute protocol
(src/mpas_sw_driver.py:33-119)."""
import functools

import numpy as np

import oracle as O
from mpsw import ic
from mpsw.mesh import icosahedral_mesh


@functools.lru_cache(maxsize=None)
def mesh(level):
    return icosahedral_mesh(level)


def configure(m, dt=600.0, visc2=0.0, visc4=0.0, drag=False, wind=False, tc=5, apvm=0.5):
    m.config_dt = dt
    m.config_h_mom_eddy_visc2 = visc2
    m.config_h_mom_eddy_visc4 = visc4
    m.config_bottom_drag = drag
    m.config_wind_stress = wind
    m.config_test_case = tc
    m.config_apvm_upwinding = apvm


def setup(m, level, case='tc5', seed=0, tl=False, ad=False, ntracers=1, **cfg):
    """Load mesh + initial condition into module `m` (oracle or engine) and run init_block."""
    msh = mesh(level)
    O.load_mesh(m, msh, ntracers)
    configure(m, tc=5 if case == 'tc5' else (2 if case == 'tc2' else (1 if case == 'tc1' else 7)), **cfg)
    if case == 'tc5':
        m.sw_test_case_5()
    elif case == 'tc2':
        m.sw_test_case_2()
    elif case == 'tc1':
        m.sw_test_case_1()
    elif case == 'tc6':
        m.sw_test_case_6()
    else:  # seeded balanced flow, with mountains ('seeded') or over a flat bottom ('balanced')
        scaled = ic.scale_mesh(msh)
        for k in ('xCell', 'yCell', 'zCell', 'xVertex', 'yVertex', 'zVertex', 'xEdge', 'yEdge',
                  'zEdge', 'dvEdge', 'dcEdge', 'areaCell', 'areaTriangle', 'kiteAreasOnVertex'):
            setattr(m, k.lower(), np.asarray(scaled[k]).T)
        st = ic.balanced_flow(scaled, seed)
        b = ic.mountains(scaled, seed + 1000) if case == 'seeded' else np.zeros(msh['nCells'])
        m.fvertex = st['fVertex']
        m.fedge = st['fEdge']
        m.h_s = b
        m.u[0, 0] = st['u']
        m.h[0, 0] = st['h'] - b
    if cfg.get('wind'):
        rng = np.random.default_rng(seed + 7)
        m.u_src = rng.standard_normal((1, msh['nEdges'])) * 0.1
    if tl:
        m.var_allocation_tlm()
    if ad:
        m.var_allocation_adj()
    m.sw_mpas_init_block()
    return m


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def maxrel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    scale = np.abs(b).max()
    return np.abs(a - b).max() / scale if scale > 0 else np.abs(a - b).max()
