"""FP64 parity of the engine-backed module against the oracle (C restatement of the reference)
on identical inputs, through the drop-in module surface.

Tolerances (relative to the field's max magnitude): forward and tangent-linear steps are
computed with the reference's operation order and no FMA, so they are held to 1e-13 per step
(the bar for the FP64 path is 1e-12 after one step); the adjoint gathers sum in a different order
than the reference's reverse scatters, so it is held to 1e-11.
"""
import numpy as np
import pytest

import oracle as O
from helpers import maxrel, rel, setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-13
ADJ_TOL = 1e-11

PHYSICS = [
    dict(),
    dict(visc2=2.0e5, visc4=1.0e15),
    dict(drag=True, wind=True),
]
DIAG = ['v', 'h_edge', 'h_vertex', 'pv_edge', 'pv_vertex', 'pv_cell', 'circulation', 'vorticity',
        'divergence', 'ke', 'vorticity_cell', 'gradpvn', 'gradpvt']
RECON = ['ureconstructx', 'ureconstructy', 'ureconstructz', 'ureconstructzonal',
         'ureconstructmeridional']


def pair(level=3, case='tc5', **kw):
    """Oracle and engine module on bit-identical inputs: the oracle builds the case, the
    engine module receives its arrays through the attribute protocol."""
    o = setup(O.OracleModule(), level, case, **kw)
    g = clone(o, MpasSwModule(), **kw)
    return o, g


def clone(o, g, tl=False, ad=False, **cfg):
    for k in ('ncells', 'nedges', 'nvertices', 'nvertlevels', 'maxedges', 'maxedges2',
              'vertexdegree', 'r3', 'ntracers', 'config_dt', 'config_test_case',
              'config_h_mom_eddy_visc2', 'config_h_mom_eddy_visc4', 'config_bottom_drag',
              'config_wind_stress', 'config_apvm_upwinding', 'on_a_sphere'):
        setattr(g, k, getattr(o, k))
    g.var_allocation()
    if tl:
        g.var_allocation_tlm()
    if ad:
        g.var_allocation_adj()
    for k, arr in o._arr.items():
        if g.__dict__['_arr'].get(k) is not None and not k.endswith(('_tl', '_ad')):
            setattr(g, k, arr)
    g.sw_mpas_init_block()
    return g


@pytest.mark.parametrize('case', ['tc5', 'seeded', 'tc2', 'tc6'])
def test_init_block_diagnostics(case):
    o, g = pair(3, case)
    for n in DIAG + RECON:
        assert maxrel(getattr(g, n), getattr(o, n)) <= FWD_TOL, n
    for n in ('coeffs_reconstruct', 'meshscalingdel2', 'edgenormalvectors', 'celltangentplane'):
        assert maxrel(getattr(g, n), getattr(o, n)) <= FWD_TOL, n


@pytest.mark.parametrize('phys', PHYSICS)
def test_sw_rk4_steps(phys):
    o, g = pair(3, 'seeded', **phys)
    for step in range(6):
        o.sw_rk4()
        g.sw_rk4()
        assert maxrel(g.u, o.u) <= FWD_TOL * (step + 1), step
        assert maxrel(g.h, o.h) <= FWD_TOL * (step + 1), step
    for n in DIAG + RECON + ['tend_u', 'tend_h']:
        assert maxrel(getattr(g, n), getattr(o, n)) <= 1e-12, n


def test_sw_rk4_bit_identical_one_step():
    """Same operation order, no contraction: the first step reproduces the oracle exactly."""
    o, g = pair(3, 'tc5')
    o.sw_rk4()
    g.sw_rk4()
    assert np.array_equal(g.u, o.u)
    assert np.array_equal(g.h, o.h)


def test_test_case_1_frozen_wind():
    o, g = pair(2, 'tc1')
    u0 = g.u.copy()
    for _ in range(3):
        o.sw_rk4()
        g.sw_rk4()
    assert np.array_equal(g.u[0], u0[0])
    assert maxrel(g.h, o.h) <= 1e-12


@pytest.mark.parametrize('phys', PHYSICS)
def test_sw_rk4_tlm_steps(phys):
    o, g = pair(3, 'seeded', tl=True, **phys)
    rng = np.random.default_rng(3)
    du = rng.standard_normal(o.u.shape[2]) * 0.1
    dh = rng.standard_normal(o.h.shape[2])
    for m in (o, g):
        m.u_tl[0, 0] = du
        m.h_tl[0, 0] = dh
    for step in range(4):
        o.sw_rk4_tlm()
        g.sw_rk4_tlm()
        assert maxrel(g.u_tl, o.u_tl) <= FWD_TOL * (step + 1)
        assert maxrel(g.h_tl, o.h_tl) <= FWD_TOL * (step + 1)
        assert maxrel(g.u, o.u) <= FWD_TOL * (step + 1)
    for n in DIAG + RECON:
        assert maxrel(getattr(g, n + '_tl'), getattr(o, n + '_tl')) <= 1e-12, n


@pytest.mark.parametrize('phys', PHYSICS)
def test_sw_rk4_adj_steps(phys):
    o, g = pair(3, 'seeded', ad=True, **phys)
    rng = np.random.default_rng(4)
    au = rng.standard_normal(o.u.shape[2])
    ah = rng.standard_normal(o.h.shape[2])
    for m in (o, g):
        m.u_ad[0, 0] = au
        m.h_ad[0, 0] = ah
    for step in range(3):
        o.sw_rk4_adj()
        g.sw_rk4_adj()
        assert maxrel(g.u_ad, o.u_ad) <= ADJ_TOL, step
        assert maxrel(g.h_ad, o.h_ad) <= ADJ_TOL, step
        assert maxrel(g.u, o.u) <= FWD_TOL  # u(2) holds the forward result
        assert np.all(g.u_ad[1] == 0) and np.all(g.h_ad[1] == 0)


def test_sw_rk4_adj_with_diagnostic_seeds():
    """Seeds left in the module's diagnostic and reconstruction adjoints are consumed."""
    o, g = pair(3, 'seeded', ad=True)
    rng = np.random.default_rng(5)
    for n in ('pv_edge_ad', 'ke_ad', 'h_vertex_ad', 'ureconstructzonal_ad', 'tend_h_ad'):
        arr = rng.standard_normal(getattr(o, n).shape)
        setattr(o, n, arr)
        setattr(g, n, arr)
    o.sw_rk4_adj()
    g.sw_rk4_adj()
    assert maxrel(g.u_ad, o.u_ad) <= ADJ_TOL
    assert maxrel(g.h_ad, o.h_ad) <= ADJ_TOL
    for n in ('pv_edge_ad', 'ke_ad', 'ureconstructzonal_ad', 'tend_h_ad'):
        assert not np.any(getattr(g, n)), n


@pytest.mark.parametrize('phys', PHYSICS)
def test_link_tlm_adj(phys):
    o, g = pair(3, 'tc5', tl=True, ad=True, **phys)
    pt = 1e-3
    for m in (o, g):
        m.u_tl[0] = m.u[0] * pt
        m.h_tl[0] = m.h[0] * pt
    lo, ro = o.link_tlm_adj()
    lg, rg = g.link_tlm_adj(verbose=False)
    assert abs(lg - rg) / abs(lg) < 1e-12
    assert abs(lg - lo) / abs(lo) < 1e-12
    assert abs(rg - ro) / abs(ro) < 1e-11


def test_step_dot_product():
    """<M dx, y> = <dx, M^T y> for one full RK4 step of the engine, FP64."""
    g = setup(MpasSwModule(), 3, 'seeded', tl=True, ad=True, visc2=1e5, drag=True)
    rng = np.random.default_rng(6)
    ub, hb = g.u[0, 0].copy(), g.h[0, 0].copy()
    dx_u = rng.standard_normal(ub.size) * 0.1
    dx_h = rng.standard_normal(hb.size)
    g.u_tl[0, 0] = dx_u
    g.h_tl[0, 0] = dx_h
    g.sw_rk4_tlm()
    Mu, Mh = g.u_tl[0, 0].copy(), g.h_tl[0, 0].copy()
    yu = rng.standard_normal(ub.size)
    yh = rng.standard_normal(hb.size)
    g.u[0, 0] = ub
    g.h[0, 0] = hb
    g.u_ad[0, 0] = yu
    g.h_ad[0, 0] = yh
    g.sw_rk4_adj()
    lhs = float(Mu @ yu + Mh @ yh)
    rhs = float(dx_u @ g.u_ad[0, 0] + dx_h @ g.h_ad[0, 0])
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_stencil_routines():
    o, g = pair(3, 'seeded', tl=True, ad=True, visc2=1e5)
    rng = np.random.default_rng(8)
    for m in (o, g):
        m.u_tl[0, 0] = rng.standard_normal(m.u.shape[2]) if m is o else o.u_tl[0, 0]
        m.h_tl[0, 0] = rng.standard_normal(m.h.shape[2]) if m is o else o.h_tl[0, 0]
    o.compute_tend()
    g.compute_tend()
    for n in ('tend_u', 'tend_h'):
        assert maxrel(getattr(g, n), getattr(o, n)) <= FWD_TOL, n
    o.solve_diagnostics_tlm()
    o.compute_tend_tlm()
    g.compute_tend_tlm()
    for n in ('tend_u_tl', 'tend_h_tl'):
        assert maxrel(getattr(g, n), getattr(o, n)) <= FWD_TOL, n


def test_forward_steps_fp64_matches_sw_rk4():
    """mpsw_forward precision 0 (one call, graph-captured steps) equals repeated sw_rk4."""
    a = setup(MpasSwModule(), 3, 'seeded', visc2=1e5, drag=True)
    b = setup(MpasSwModule(), 3, 'seeded', visc2=1e5, drag=True)
    for _ in range(5):
        a.sw_rk4()
    b.sw_rk4_steps(5)
    assert np.array_equal(a.u[0, 0], b.u[0, 0]) and np.array_equal(a.h[0, 0], b.h[0, 0])
    assert np.array_equal(a.pv_edge, b.pv_edge)


@pytest.mark.parametrize('phys', [dict(), dict(visc2=1e5, visc4=5e14, drag=True)])
def test_forward_fp32_stencils_close_to_fp64(phys):
    """FP32 stencils with FP64 RK accumulation stay within 1e-5 relative L2 of the FP64 forward
    over 48 steps (8 h at dt = 600 s) on the level-4 mesh."""
    a = setup(MpasSwModule(), 4, 'seeded', dt=600.0, **phys)
    b = setup(MpasSwModule(), 4, 'seeded', dt=600.0, **phys)
    a.sw_rk4_steps(48, 0)
    b.sw_rk4_steps(48, 1)
    eu, eh = rel(b.u[0, 0], a.u[0, 0]), rel(b.h[0, 0], a.h[0, 0])
    assert eu < 1e-5 and eh < 1e-5, (eu, eh)
    assert not np.array_equal(a.h[0, 0], b.h[0, 0])  # the FP32 path did run


# ---- tracer transport (config_advect_tracers; the reference leaves it out) -----------------
def tracer_pair(level=3, ntr=2, seed=3, **kw):
    o = setup(O.OracleModule(), level, 'tc5', ntracers=ntr, **kw)
    rng = np.random.default_rng(seed)
    o.tracers[0] = 1.0 + 0.1 * rng.standard_normal(o.tracers[0].shape)
    o.tracers[1] = o.tracers[0]
    g = clone(o, MpasSwModule(), **kw)
    for m in (o, g):
        m.config_advect_tracers = 1
    return o, g


@pytest.mark.parametrize('phys', [dict(), dict(visc2=2.0e5, visc4=1.0e15)])
def test_tracer_transport_bit_identical(phys):
    """sw_rk4 with tracer transport: tracers and tend_tracer equal the oracle's bit for bit, and
    u, h are those of a run without transport."""
    o, g = tracer_pair(**phys)
    plain = clone(o, MpasSwModule(), **phys)
    plain.config_advect_tracers = 0
    for _ in range(3):
        o.sw_rk4()
        g.sw_rk4()
        plain.sw_rk4()
    assert o.tracers.shape[1] == 2
    assert np.array_equal(g.tracers, o.tracers)
    assert np.array_equal(g.tend_tracer, o.tend_tracer)
    assert not np.array_equal(g.tracers[0], plain.tracers[0])  # the tracers did move
    assert np.array_equal(g.u, plain.u) and np.array_equal(g.h, plain.h)


def test_tracer_transport_steps_and_conservation():
    """sw_rk4_steps(n) with transport equals n sw_rk4 calls; on level 5 the tracer mass
    sum(areaCell h tracer) is conserved to rounding and a constant tracer stays constant."""
    o, g = tracer_pair(level=3)
    g2 = clone(o, MpasSwModule())
    g2.config_advect_tracers = 1
    for _ in range(4):
        g.sw_rk4()
    g2.sw_rk4_steps(4)
    assert np.array_equal(g.tracers, g2.tracers)
    with pytest.raises(RuntimeError):
        g2.sw_rk4_steps(1, precision=1)

    m = setup(MpasSwModule(), 5, 'seeded', dt=300.0, ntracers=2)
    m.tracers[0, 0, 0] = 1.0
    x = np.asarray(m.xcell).ravel()
    m.tracers[0, 1, 0] = 1.0 + 0.5 * x / np.abs(x).max()
    m.config_advect_tracers = 1
    area = np.asarray(m.areacell).ravel()
    mass0 = (area * m.h[0, 0] * m.tracers[0, 1, 0]).sum()
    m.sw_rk4_steps(20)
    mass1 = (area * m.h[0, 0] * m.tracers[0, 1, 0]).sum()
    assert abs(mass1 - mass0) / abs(mass0) < 1e-12
    assert np.abs(m.tracers[0, 0, 0] - 1.0).max() < 1e-12
    assert np.abs(m.tracers[0, 1, 0] - m.tracers[0, 1, 0].mean()).max() > 1e-3
