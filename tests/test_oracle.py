"""Self-consistency of the oracle (the C restatement of the reference): the hand-written
tangent linear is the derivative of the forward model (finite differences), the adjoint is its
transpose (dot-product tests, as src/mpas_sw_module.f90:1006-1218 and the FD check of
src/mpas_sw_driver.py:335-377 do, here asserted), and Williamson TC2's steady state is kept
with an error that falls with resolution."""
import numpy as np
import pytest

import oracle as O
from helpers import setup

PHYS = [dict(), dict(visc2=2e5, visc4=1e15), dict(drag=True, wind=True)]


@pytest.mark.parametrize('phys', PHYS)
def test_link_tlm_adj_dot_product(phys):
    m = setup(O.OracleModule(), 3, 'tc5', tl=True, ad=True, **phys)
    m.u_tl[0] = m.u[0] * 1e-3
    m.h_tl[0] = m.h[0] * 1e-3
    lhs, rhs = m.link_tlm_adj()
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


@pytest.mark.parametrize('phys', PHYS)
def test_step_dot_product(phys):
    m = setup(O.OracleModule(), 3, 'seeded', tl=True, ad=True, **phys)
    rng = np.random.default_rng(1)
    ub, hb = m.u[0, 0].copy(), m.h[0, 0].copy()
    du, dh = rng.standard_normal(ub.size) * 0.1, rng.standard_normal(hb.size)
    m.u_tl[0, 0], m.h_tl[0, 0] = du, dh
    m.sw_rk4_tlm()
    Mu, Mh = m.u_tl[0, 0].copy(), m.h_tl[0, 0].copy()
    yu, yh = rng.standard_normal(ub.size), rng.standard_normal(hb.size)
    m.u[0, 0], m.h[0, 0] = ub, hb
    m.u_ad[0, 0], m.h_ad[0, 0] = yu, yh
    m.sw_rk4_adj()
    lhs = Mu @ yu + Mh @ yh
    rhs = du @ m.u_ad[0, 0] + dh @ m.h_ad[0, 0]
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_tangent_linear_vs_finite_differences():
    m = setup(O.OracleModule(), 3, 'seeded', tl=True, visc2=1e5, drag=True)
    ub, hb = m.u[0, 0].copy(), m.h[0, 0].copy()
    rng = np.random.default_rng(2)
    du, dh = rng.standard_normal(ub.size) * 0.1, rng.standard_normal(hb.size)
    m.u_tl[0, 0], m.h_tl[0, 0] = du, dh
    for _ in range(3):
        m.sw_rk4_tlm()
    tlu = m.u_tl[0, 0].copy()
    errs = []
    for eps in (1e-2, 1e-4, 1e-6):
        out = []
        for s in (1, -1):
            m.u[0, 0], m.h[0, 0] = ub + s * eps * du, hb + s * eps * dh
            for _ in range(3):
                m.sw_rk4()
            out.append(m.u[0, 0].copy())
        fd = (out[0] - out[1]) / (2 * eps)
        errs.append(np.linalg.norm(fd - tlu) / np.linalg.norm(tlu))
    assert errs[0] < 1e-8 and errs[1] < 1e-7 and errs[2] < 1e-5


def test_tc2_steady_state_converges():
    """TC2's initial state is an exact steady solution: the 6-hour drift shrinks with resolution."""
    drift = []
    for level, dt in ((3, 600.0), (4, 300.0)):
        m = setup(O.OracleModule(), level, 'tc2', dt=dt)
        h0 = m.h[0, 0].copy()
        for _ in range(int(6 * 3600 / dt)):
            m.sw_rk4()
        drift.append(np.abs(m.h[0, 0] - h0).max() / np.abs(h0).max())
    assert drift[1] < drift[0] * 0.75 and drift[1] < 5e-3


def test_mass_conservation():
    m = setup(O.OracleModule(), 3, 'seeded', visc2=1e5)
    mass0 = float(m.h[0, 0] @ m.areacell)
    for _ in range(5):
        m.sw_rk4()
    assert abs(float(m.h[0, 0] @ m.areacell) - mass0) / mass0 < 1e-14


def test_adjoint_consumes_seeds():
    m = setup(O.OracleModule(), 2, 'tc5', ad=True)
    m.pv_edge_ad = np.ones_like(m.pv_edge_ad)
    m.tend_u_ad = np.ones_like(m.tend_u_ad)
    m.u_ad[0, 0] = 1.0
    m.sw_rk4_adj()
    assert not m.pv_edge_ad.any() and not m.tend_u_ad.any()
    assert not m.u_ad[1].any() and m.u_ad[0].any()


def test_tracer_transport_oracle():
    """Tracer transport in the oracle's sw_rk4 (config_advect_tracers): off, the tracers are only
    carried (the reference's behaviour); on, a constant tracer stays constant, its tendency is
    exactly tend_h, and the tracer mass sum(areaCell h tracer) is conserved to rounding."""
    m = setup(O.OracleModule(), 3, 'tc5', ntracers=2)
    rng = np.random.default_rng(5)
    m.tracers[0, 0, 0] = 1.0
    m.tracers[0, 1, 0] = 1.0 + 0.1 * rng.standard_normal(m.tracers.shape[-1])
    t0 = m.tracers.copy()
    m.sw_rk4()
    assert np.array_equal(m.tracers[0], t0[0]) and np.array_equal(m.tracers[1], t0[0])

    m = setup(O.OracleModule(), 3, 'tc5', ntracers=2)
    m.tracers[0] = t0[0]
    m.config_advect_tracers = 1
    area = np.asarray(m.areacell).ravel()
    mass0 = (area * m.h[0, 0] * m.tracers[0, 1, 0]).sum()
    for _ in range(4):
        m.sw_rk4()
    mass1 = (area * m.h[0, 0] * m.tracers[0, 1, 0]).sum()
    assert abs(mass1 - mass0) / abs(mass0) < 1e-13
    assert np.abs(m.tracers[0, 0, 0] - 1.0).max() < 1e-14
    assert np.array_equal(m.tracers[0], m.tracers[1])
    assert not np.array_equal(m.tracers[0, 1, 0], t0[0, 1, 0])
    m.solve_diagnostics()
    m.compute_tend()
    m.compute_scalar_tend()
    assert np.array_equal(m.tend_tracer[0, 0], m.tend_h[0])
