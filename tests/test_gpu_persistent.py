"""The persistent forward kernel (one cooperative launch for all the steps of sw_rk4_steps /
mpsw_forward, grid barriers between the phases of a stage) against the per-step graphs of the
four forward kernels: the same per-entity arithmetic, so the states agree bit for bit, in FP64
and with FP32 stencils, with the physics switches it covers (del4 viscosity runs the graphs)."""
import os

import numpy as np
import pytest

from helpers import setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu


def run(phys, precision, nsteps, persistent):
    old = os.environ.get('MPSW_PERSIST')
    os.environ['MPSW_PERSIST'] = '1' if persistent else '0'
    try:
        g = setup(MpasSwModule(), 4, 'seeded', dt=300.0, **phys)
        g.sw_rk4_steps(nsteps, precision)
        out = (g.u.copy(), g.h.copy())
        if precision == 0:
            out += (g.tend_u.copy(), g.tend_h.copy())
        return out
    finally:
        if old is None:
            del os.environ['MPSW_PERSIST']
        else:
            os.environ['MPSW_PERSIST'] = old


@pytest.mark.parametrize('precision', [0, 1])
@pytest.mark.parametrize('phys', [dict(), dict(visc2=2.0e5, drag=True, wind=True)])
def test_persistent_forward_matches_step_graphs(phys, precision):
    a = run(phys, precision, 10, True)
    b = run(phys, precision, 10, False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.isfinite(a[0]).all() and np.isfinite(a[1]).all()


def test_persistent_forward_zero_steps_leaves_state():
    """No step: time level 1 keeps the state (and time level 2 receives it, as after sw_rk4)."""
    g = setup(MpasSwModule(), 3, 'seeded')
    u0, h0 = g.u[0].copy(), g.h[0].copy()
    g.sw_rk4_steps(0, 1)
    assert np.array_equal(g.u[0], u0) and np.array_equal(g.h[0], h0)
    assert np.array_equal(g.u[1], u0) and np.array_equal(g.h[1], h0)
