"""Failure reporting on the GPU without a GPU fault: a NaN placed in the host-side input makes the
tendency kernels raise the engine's non-finite flag, and the routine returns MPSW_ERR_NONFINITE
(6) instead of carrying NaNs on silently as the reference's Fortran does; the next call with a
clean input succeeds (the flag is cleared per call)."""
import numpy as np
import pytest

from helpers import setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def test_forward_step_reports_nonfinite_state():
    m = setup(MpasSwModule(), 3, 'seeded', dt=600.0)
    u0, h0 = m.u[0, 0].copy(), m.h[0, 0].copy()
    bad = u0.copy()
    bad[17] = np.nan
    m.u[0, 0] = bad
    with pytest.raises(RuntimeError, match=r'\(6\).*non-finite'):
        m.sw_rk4()
    m.u[0, 0] = u0
    m.h[0, 0] = h0
    m.sw_rk4()  # a clean state steps again
    assert np.isfinite(m.u[0, 0]).all()


@pytest.mark.parametrize('prec_name', ['FP64', 'FP32'])
def test_window_sweeps_report_nonfinite_members(prec_name):
    from mpsw import torch_api
    prec = getattr(torch_api, prec_name)
    m = setup(MpasSwModule(), 3, 'seeded', dt=600.0)
    e = torch_api.Engine(m)
    B = 4
    rng = np.random.default_rng(1)
    du = torch.tensor(rng.standard_normal((int(m.nedges), B)) * 0.1, device='cuda')
    dh = torch.tensor(rng.standard_normal((int(m.ncells), B)), device='cuda')
    w = e.window(6, ckpt_every=2)
    bad = du.clone()
    bad[40, 2] = float('inf')
    with pytest.raises(RuntimeError, match=r'\(6\).*non-finite'):
        w.tl(bad, dh, prec)
    with pytest.raises(RuntimeError, match=r'\(6\).*non-finite'):
        w.ad(bad, dh, prec)
    tu, th = w.tl(du, dh, prec)  # clean members sweep again
    assert torch.isfinite(tu).all() and torch.isfinite(th).all()
