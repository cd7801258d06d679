"""Host-side behaviour of the drop-in module (module_sw_mpas.mpas_sw_module): the f2py
attribute protocol used by src/mpas_sw_driver.py works, and the Williamson test-case set-ups
agree with the oracle's restatement of src/mpas_sw_testcases.f90."""
import numpy as np
import pytest

import oracle as O
from helpers import mesh
from module_sw_mpas import MpasSwModule


def loaded(level=2):
    m = MpasSwModule()
    O.load_mesh(m, mesh(level))
    return m


def test_attribute_protocol():
    m = loaded()
    assert m.u.shape == (2, 1, 480) and m.u.flags.f_contiguous
    assert m.cellsonedge.dtype == np.int32 and m.cellsonedge.min() == 1
    assert m.u_tl is None                      # unallocated allocatable
    m.var_allocation_tlm()
    assert m.u_tl.shape == (2, 1, 480)
    m.xcell[()] *= m.a                         # in-place scaling as mpsw_init_real does
    assert abs(m.xcell).max() > 1e6
    ref = m.u
    m.u[0, 0] = 1.5
    assert ref is m.u and np.all(m.u[0, 0] == 1.5)
    m.config_dt = 900.
    assert float(m.config_dt) == 900.
    m.config_bottom_drag = True
    assert int(m.config_bottom_drag) == 1
    assert int(m.config_advect_tracers) == 0   # tracers carried, as in the reference
    m.config_advect_tracers = 1
    assert int(m.config_advect_tracers) == 1 and m.tracers.shape == (2, 1, 1, 162)
    with pytest.raises(ValueError):
        m.cellsonedge = np.zeros((3, 480), dtype=np.int32)
    with pytest.raises(AttributeError):
        m.not_a_module_variable


@pytest.mark.parametrize('case', [1, 2, 5, 6])
def test_test_cases_match_oracle(case):
    g, o = loaded(), O.OracleModule()
    O.load_mesh(o, mesh(2))
    getattr(g, f'sw_test_case_{case}')()
    getattr(o, f'sw_test_case_{case}')()
    for n in ('u', 'h', 'h_s', 'fvertex', 'fedge', 'areacell', 'dcedge', 'kiteareasonvertex'):
        np.testing.assert_allclose(getattr(g, n), getattr(o, n), rtol=1e-14, atol=1e-12, err_msg=n)
