"""Batched device-resident windows (B members on the trailing dimension) and the autograd
step: FP64 windows agree with the single-member module path, the FP64 window's tangent linear
and adjoint pass the dot-product test, and the FP32-stencil / FP64-accumulation windows stay
within 1e-4 relative L2 error of the FP64 window (the bar for the FP32-stencil form)."""
import numpy as np
import pytest

from helpers import rel, setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def engine(level=3, **cfg):
    from mpsw.torch_api import Engine
    m = setup(MpasSwModule(), level, 'seeded', tl=True, ad=True, **cfg)
    return m, Engine(m)


def members(m, B, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    du = torch.tensor(rng.standard_normal((int(m.nedges), B)) * 0.1 * scale, device='cuda')
    dh = torch.tensor(rng.standard_normal((int(m.ncells), B)) * scale, device='cuda')
    return du, dh


@pytest.mark.parametrize('cfg', [dict(), dict(visc2=2e5, visc4=1e15, drag=True)])
def test_window_tl_matches_module_tlm(cfg):
    m, e = engine(**cfg)
    nsteps, B = 5, 3
    du, dh = members(m, B, 1)
    w = e.window(nsteps, ckpt_every=2)
    tu, th = w.tl(du, dh)
    u0, h0 = m.u[0, 0].copy(), m.h[0, 0].copy()
    for b in range(B):
        m.u[0, 0], m.h[0, 0] = u0, h0
        m.u_tl[0, 0] = du[:, b].cpu().numpy()
        m.h_tl[0, 0] = dh[:, b].cpu().numpy()
        for _ in range(nsteps):
            m.sw_rk4_tlm()
        assert np.array_equal(tu[:, b].cpu().numpy(), m.u_tl[0, 0])
        assert np.array_equal(th[:, b].cpu().numpy(), m.h_tl[0, 0])


def test_window_ad_matches_module_adj():
    m, e = engine(visc2=1e5)
    nsteps, B = 4, 2
    au, ah = members(m, B, 2)
    u0, h0 = m.u[0, 0].copy(), m.h[0, 0].copy()
    states = []
    for _ in range(nsteps):
        states.append((m.u[0, 0].copy(), m.h[0, 0].copy()))
        m.sw_rk4()
    m.u[0, 0], m.h[0, 0] = u0, h0
    w = e.window(nsteps, ckpt_every=3)
    ru, rh = w.ad(au, ah)
    for b in range(B):
        m.u_ad[0, 0] = au[:, b].cpu().numpy()
        m.h_ad[0, 0] = ah[:, b].cpu().numpy()
        for n in reversed(range(nsteps)):
            m.u[0, 0], m.h[0, 0] = states[n]
            m.sw_rk4_adj()
        assert rel(ru[:, b].cpu().numpy(), m.u_ad[0, 0]) < 1e-13
        assert rel(rh[:, b].cpu().numpy(), m.h_ad[0, 0]) < 1e-13


@pytest.mark.parametrize('cfg', [dict(), dict(visc2=1e5, visc4=5e14, drag=True, wind=True)])
def test_window_dot_product_and_fp32(cfg):
    m, e = engine(level=4, dt=300.0, **cfg)
    nsteps, B = 24, 4
    du, dh = members(m, B, 3)
    w = e.window(nsteps, ckpt_every=5)
    tu, th = w.tl(du, dh)
    yu, yh = members(m, B, 4)
    au, ah = w.ad(yu, yh)
    lhs = (tu * yu).sum(0) + (th * yh).sum(0)
    rhs = (du * au).sum(0) + (dh * ah).sum(0)
    assert torch.all((lhs - rhs).abs() / lhs.abs() < 1e-12), (lhs, rhs)
    from mpsw.torch_api import FP32
    tu32, th32 = w.tl(du, dh, precision=FP32)
    au32, ah32 = w.ad(yu, yh, precision=FP32)
    for b in range(B):
        for a, r in ((tu32, tu), (th32, th), (au32, au), (ah32, ah)):
            assert rel(a[:, b].cpu().numpy(), r[:, b].cpu().numpy()) < 1e-4


def test_autograd_step_matches_adjoint_and_fd():
    from mpsw.torch_api import rk4_step
    m, e = engine()
    u = torch.tensor(m.u[0, 0].copy(), device='cuda', requires_grad=True)
    h = torch.tensor(m.h[0, 0].copy(), device='cuda', requires_grad=True)
    u1, h1 = rk4_step(u, h, e)
    u2, h2 = rk4_step(u1, h1, e)
    rng = np.random.default_rng(9)
    wu = torch.tensor(rng.standard_normal(u2.shape), device='cuda')
    wh = torch.tensor(rng.standard_normal(h2.shape), device='cuda')
    J = (wu * u2).sum() + (wh * h2).sum()
    J.backward()
    du = torch.tensor(rng.standard_normal(u.shape) * 0.01, device='cuda')
    dh = torch.tensor(rng.standard_normal(h.shape) * 0.01, device='cuda')
    eps = 1e-4
    with torch.no_grad():
        jp = [(wu * a).sum() + (wh * b).sum() for a, b in [rk4_step(*rk4_step(u + eps * du, h + eps * dh, e), e)]][0]
        jm = [(wu * a).sum() + (wh * b).sum() for a, b in [rk4_step(*rk4_step(u - eps * du, h - eps * dh, e), e)]][0]
    fd = float((jp - jm) / (2 * eps))
    ad = float((u.grad * du).sum() + (h.grad * dh).sum())
    assert abs(fd - ad) / abs(ad) < 1e-6


@pytest.mark.parametrize('precision', [0, 1])
def test_stored_and_recomputed_stages_identical(precision):
    """Sweeps over stored stage linearisation points equal sweeps that recompute the stages
    from checkpoints, bit for bit, in both precisions (4 members: vector width 4 in FP32)."""
    m, e = engine(visc2=1e5, visc4=5e14, drag=True)
    nsteps, B = 7, 4
    du, dh = members(m, B, 5)
    au, ah = members(m, B, 6)
    out = {}
    for storage in (0, 3):
        w = e.window(nsteps, ckpt_every=3, storage=storage)
        out[storage] = w.tl(du, dh, precision) + w.ad(au, ah, precision)
    for a, b in zip(out[0], out[3]):
        assert torch.equal(a, b)


@pytest.mark.parametrize('precision', [0, 1])
def test_member_width_does_not_change_results(precision):
    """A 4-member sweep (several members per thread) and one-member sweeps (one member per
    thread) give the same numbers: the per-member arithmetic does not depend on the width."""
    m, e = engine(visc2=1e5)
    nsteps, B = 3, 4
    du, dh = members(m, B, 7)
    au, ah = members(m, B, 8)
    w = e.window(nsteps, ckpt_every=2)
    tu, th = w.tl(du, dh, precision)
    ru, rh = w.ad(au, ah, precision)
    for b in range(B):
        t1 = w.tl(du[:, b:b + 1].contiguous(), dh[:, b:b + 1].contiguous(), precision)
        r1 = w.ad(au[:, b:b + 1].contiguous(), ah[:, b:b + 1].contiguous(), precision)
        for x, y in zip(t1 + r1, (tu, th, ru, rh)):
            if precision == 0:
                assert torch.equal(x[:, 0], y[:, b])
            else:  # FP32 stencils are compiled with contraction: allow one rounding per op
                assert rel(x[:, 0].cpu().numpy(), y[:, b].cpu().numpy()) < 1e-6


def test_tuning_cache_file(tmp_path, monkeypatch):
    """The autotuner writes its choice for (mesh, precision, B) to MPSW_TUNE_CACHE, and an engine
    finding the key there takes it from the file."""
    import ctypes
    from mpsw import _lib
    cache = tmp_path / 'tune.txt'
    monkeypatch.setenv('MPSW_TUNE_CACHE', str(cache))
    m, e = engine(level=2)
    du, dh = members(m, 8, 11)
    w = e.window(2, ckpt_every=1)
    w.tl(du, dh, 1)
    lines = cache.read_text().split('\n')
    key_lines = [l for l in lines if l.strip()]
    assert len(key_lines) == 1 and key_lines[0].split()[0].endswith('|1|8')
    # a different choice under the same key in the file is taken by a new engine
    vals = [8, 64] * 8
    cache.write_text(key_lines[0].split()[0] + ' ' + ' '.join(map(str, vals)) + '\n')
    m2, e2 = engine(level=2)
    w2 = e2.window(2, ckpt_every=1)
    a = w2.tl(du, dh, 1)
    out = (ctypes.c_int * 16)()
    e2.h.check(_lib.load().mpsw_window_tuning(e2.h.ptr, 1, 8, out), 'tuning')
    assert list(out) == vals
    b = w.tl(du, dh, 1)
    for x, y in zip(a, b):  # FP32 stencils: the launch choice may move a rounding, no more
        assert rel(x.cpu().numpy(), y.cpu().numpy()) < 1e-6
