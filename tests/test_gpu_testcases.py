"""Williamson test cases 1, 2, 5 and 6 set up by GPU kernels (mpsw_sw_test_case,
csrc/mpsw_testcases.cu) against the host set-up of mpsw/testcases.py, which restates
src/mpas_sw_testcases.f90: the same fields to the last bits of the device's sin / cos / pow, and
the GPU set-up timed on the level-8 mesh (655362 cells)."""
import time

import numpy as np
import pytest

import oracle as O
from helpers import configure, mesh
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu

FIELDS = ('u', 'h', 'fedge', 'fvertex', 'h_s', 'loncell', 'xcell', 'dvedge', 'areacell', 'kiteareasonvertex')


def loaded(level):
    m = MpasSwModule()
    O.load_mesh(m, mesh(level), 2)
    configure(m)
    return m


@pytest.mark.parametrize('tc', [1, 2, 5, 6])
def test_device_test_case_matches_host(tc):
    host, dev = loaded(3), loaded(3)
    getattr(host, 'sw_test_case_%d' % tc)()
    dev.sw_test_case_device(tc)
    for k in FIELDS + ('tracers',):
        a, b = np.asarray(getattr(dev, k)), np.asarray(getattr(host, k))
        scale = max(np.abs(b).max(), 1e-300)
        # u is a difference of stream-function values ~1e8 apart from zero: their last-bit
        # differences become ~1e-14 of u
        tol = 1e-13 if k == 'u' else 4e-15
        assert np.abs(a - b).max() <= tol * scale, (tc, k, np.abs(a - b).max() / scale)


def test_device_test_case_level8_timing():
    m = loaded(8)
    t0 = time.perf_counter()
    m.sw_test_case_device(5)
    dt = time.perf_counter() - t0
    print('test case 5 on the level-8 mesh (GPU kernels, host scaling and copies): %.3f s' % dt)
    assert np.isfinite(np.asarray(m.h)).all()
