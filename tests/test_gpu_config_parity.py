"""Parity at the size of the benchmark configurations, against the oracle (the C restatement of
the reference Fortran) and through the reference's own checks.

* One day of the plain FP64 forward on the level-5 mesh (10242 cells, 288 steps of 300 s, seeded
  balanced flow over a flat bottom): within 1e-12 of the oracle after one step and 1e-9 after the
  day (src/mpas_sw_module.f90:528-635, driven as src/mpas_sw_driver.py:279-289).
* The FP64 window on that day: the dot-product test <L dx, y> = <dx, L^T y> to 1e-12
  (src/mpas_sw_module.f90:1006-1218 does it for one stage), and the tangent linear against
  nonlinear finite differences for relative perturbations 1e-2 .. 1e-8 as the reference's
  check_tlm does (src/mpas_sw_driver.py:335-377).
* The window adjoint against the oracle's per-step sw_rk4_adj (src/mpas_sw_module.f90:783-1002).
* The batched FP32-stencil windows within 1e-4 relative L2 of the FP64 window on levels 5 and 6.
"""
import numpy as np
import pytest

import oracle as O
from helpers import maxrel, setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

DT5, DAY5 = 300.0, 288


@pytest.fixture(scope='module')
def day5():
    """Oracle and engine modules on the level-5 day's initial state, and the oracle's states
    after 1 and 288 steps."""
    o = setup(O.OracleModule(), 5, 'balanced', dt=DT5)
    g = setup(MpasSwModule(), 5, 'balanced', dt=DT5, tl=True, ad=True)
    u0, h0 = o.u[0, 0].copy(), o.h[0, 0].copy()
    o.sw_rk4()
    one = (o.u[0, 0].copy(), o.h[0, 0].copy())
    for _ in range(DAY5 - 1):
        o.sw_rk4()
    day = (o.u[0, 0].copy(), o.h[0, 0].copy())
    return g, (u0, h0), one, day


def test_forward_one_day_level5(day5):
    g, (u0, h0), one, day = day5
    g.u[0, 0], g.h[0, 0] = u0, h0
    g.sw_rk4()
    assert maxrel(g.u[0, 0], one[0]) <= 1e-12
    assert maxrel(g.h[0, 0], one[1]) <= 1e-12
    g.sw_rk4_steps(DAY5 - 1)
    assert maxrel(g.u[0, 0], day[0]) <= 1e-9
    assert maxrel(g.h[0, 0], day[1]) <= 1e-9
    g.u[0, 0], g.h[0, 0] = u0, h0


def _members(n, B, seed, scale):
    rng = np.random.default_rng(seed)
    return torch.tensor(rng.standard_normal((n, B)) * scale, device='cuda')


def test_window_dot_product_one_day_level5(day5):
    from mpsw.torch_api import FP64, Engine
    g, (u0, h0), _, _ = day5
    g.u[0, 0], g.h[0, 0] = u0, h0
    e = Engine(g)
    B = 4
    du, dh = _members(int(g.nedges), B, 1, 0.1), _members(int(g.ncells), B, 2, 1.0)
    yu, yh = _members(int(g.nedges), B, 3, 0.1), _members(int(g.ncells), B, 4, 1.0)
    w = e.window(DAY5, ckpt_every=16)
    tu, th = w.tl(du, dh, FP64)
    au, ah = w.ad(yu, yh, FP64)
    lhs = (tu * yu).sum(0) + (th * yh).sum(0)
    rhs = (du * au).sum(0) + (dh * ah).sum(0)
    assert torch.all((lhs - rhs).abs() / lhs.abs() <= 1e-12), (lhs, rhs)


def test_tangent_linear_vs_finite_differences_level5(day5):
    """check_tlm: perturb the whole initial state by a factor (1 + eps), run the nonlinear day,
    and compare (M(x (1 + eps)) - M(x)) with the tangent linear of eps x, at the reference's
    probe point (index 500) and over the whole field."""
    from mpsw.torch_api import FP64, Engine
    g, (u0, h0), _, _ = day5
    g.u[0, 0], g.h[0, 0] = u0, h0
    g.sw_rk4_steps(DAY5)
    day = (g.u[0, 0].copy(), g.h[0, 0].copy())
    g.u[0, 0], g.h[0, 0] = u0, h0
    e = Engine(g)
    w = e.window(DAY5, ckpt_every=16)
    tu, th = w.tl(torch.tensor(u0, device='cuda')[:, None], torch.tensor(h0, device='cuda')[:, None], FP64)
    tu, th = tu[:, 0].cpu().numpy(), th[:, 0].cpu().numpy()  # L x, so L (eps x) = eps L x
    errs = []
    for k in range(2, 9):
        eps = 10.0 ** -k
        g.u[0, 0], g.h[0, 0] = u0 * (1 + eps), h0 * (1 + eps)
        g.sw_rk4_steps(DAY5)
        du, dh = g.u[0, 0] - day[0], g.h[0, 0] - day[1]
        r_point = (dh[500] / (eps * th[500]), du[500] / (eps * tu[500]))
        r_field = (np.dot(dh, th) / (eps * np.dot(th, th)), np.dot(du, tu) / (eps * np.dot(tu, tu)))
        errs.append((eps, max(abs(r - 1) for r in r_point + r_field)))
    g.u[0, 0], g.h[0, 0] = u0, h0
    print('TL vs finite differences, |ratio - 1| by eps:', errs)
    # the ratio converges to 1 at first order in eps until rounding takes over
    e2, e4 = dict(errs)[1e-2], dict(errs)[1e-4]
    assert e4 < 1e-3 and e4 < 0.05 * e2, errs
    assert min(err for eps, err in errs) < 1e-5, errs


def test_window_adjoint_vs_oracle_level5():
    """24 steps of the window's FP64 adjoint against the oracle's sw_rk4_adj, step by step from
    the end of the window (each step linearised about its own start state)."""
    from mpsw.torch_api import FP64, Engine
    nsteps = 24
    o = setup(O.OracleModule(), 5, 'balanced', dt=DT5, ad=True)
    g = setup(MpasSwModule(), 5, 'balanced', dt=DT5, ad=True)
    rng = np.random.default_rng(5)
    au = rng.standard_normal(int(g.nedges)) * 0.1
    ah = rng.standard_normal(int(g.ncells))
    states = []
    for _ in range(nsteps):
        states.append((o.u[0, 0].copy(), o.h[0, 0].copy()))
        o.sw_rk4()
    o.u_ad[0, 0], o.h_ad[0, 0] = au, ah
    for n in reversed(range(nsteps)):
        o.u[0, 0], o.h[0, 0] = states[n]
        o.sw_rk4_adj()
    e = Engine(g)
    w = e.window(nsteps, ckpt_every=8)
    ru, rh = w.ad(torch.tensor(au, device='cuda')[:, None], torch.tensor(ah, device='cuda')[:, None], FP64)
    assert maxrel(ru[:, 0].cpu().numpy(), o.u_ad[0, 0]) <= 1e-10
    assert maxrel(rh[:, 0].cpu().numpy(), o.h_ad[0, 0]) <= 1e-10


@pytest.mark.parametrize('level,dt,nsteps', [(5, 300.0, 288), (6, 150.0, 96)])
def test_fp32_window_within_bar(level, dt, nsteps):
    """Batched FP32-stencil / FP64-accumulation TL and AD windows (64 members, the member kernels
    the sweeps run by default) within 1e-4 relative L2 of the FP64 window, member by member."""
    from mpsw.torch_api import FP32, FP64, Engine
    g = setup(MpasSwModule(), level, 'seeded', dt=dt)
    e = Engine(g)
    B = 64
    du, dh = _members(int(g.nedges), B, 6, 0.1), _members(int(g.ncells), B, 7, 1.0)
    out = {}
    for prec in (FP32, FP64):
        w = e.window(nsteps, ckpt_every=16)
        tu, th = w.tl(du, dh, prec)
        out[prec] = (tu, th) + w.ad(tu, th, prec)
    num = torch.sqrt(sum(((a - b) ** 2).sum(0) for a, b in zip(out[FP32], out[FP64])))
    den = torch.sqrt(sum((b ** 2).sum(0) for b in out[FP64]))
    assert float((num / den).max()) <= 1e-4
