"""Fused FP32 member stages: one kernel per tangent-linear or adjoint RK stage over halo tiles
(csrc/mpsw_fused.cuh, tiles from csrc/mpsw_tiles.cpp) against the split member kernels.

Each entity's intermediates are formed by the same expression whichever tile computes them, so
the results do not depend on the tile size; they agree with the split FP32 kernels to FP32
rounding and with the FP64 window within the FP32-stencil bar (1e-4 relative L2)."""
import os

import numpy as np
import pytest

from helpers import setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

TOL_SPLIT = 1e-5   # fused vs split FP32 member kernels (FP32 roundings in another order)
TOL_FP64 = 1e-4    # FP32 stencils vs the FP64 window


def engine(level, env, **cfg):
    """A module whose device mesh (and fused tiles) is built with the environment `env`."""
    from mpsw.torch_api import Engine
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        m = setup(MpasSwModule(), level, 'seeded', dt=300.0, **cfg)
        return m, Engine(m)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def members(m, B, seed):
    rng = np.random.default_rng(seed)
    du = torch.tensor(rng.standard_normal((int(m.nedges), B)) * 0.1, device='cuda')
    dh = torch.tensor(rng.standard_normal((int(m.ncells), B)), device='cuda')
    return du, dh


def sweep(e, du, dh, yu, yh, prec, nsteps=8, storage=-1):
    w = e.window(nsteps, ckpt_every=3, storage=storage)
    return w.tl(du, dh, prec) + w.ad(yu, yh, prec)


def relmax(a, b):
    num = torch.sqrt(sum(((x - y) ** 2).sum(0) for x, y in zip(a, b)))
    den = torch.sqrt(sum((y ** 2).sum(0) for y in b))
    return float((num / den).max())


@pytest.mark.parametrize('level', [4, 5])
def test_fused_matches_split_and_fp64(level):
    from mpsw.torch_api import FP32, FP64
    B = 8
    mf, ef = engine(level, {'MPSW_FUSED': '1'})
    ms, es = engine(level, {'MPSW_FUSED': '0'})
    du, dh = members(mf, B, 1)
    yu, yh = members(mf, B, 2)
    fused = sweep(ef, du, dh, yu, yh, FP32)
    split = sweep(es, du, dh, yu, yh, FP32)
    ref = sweep(es, du, dh, yu, yh, FP64)
    assert relmax(fused[:2], split[:2]) < TOL_SPLIT
    assert relmax(fused[2:], split[2:]) < TOL_SPLIT
    assert relmax(fused[:2], ref[:2]) < TOL_FP64
    assert relmax(fused[2:], ref[2:]) < TOL_FP64


def test_fused_independent_of_tile_size_and_storage():
    from mpsw.torch_api import FP32
    B = 8
    outs = []
    for K in (17, 64, 200):
        m, e = engine(4, {'MPSW_FUSED': '1', 'MPSW_FUSED_K': str(K)})
        du, dh = members(m, B, 3)
        yu, yh = members(m, B, 4)
        outs.append(sweep(e, du, dh, yu, yh, FP32))
    outs.append(sweep(e, du, dh, yu, yh, FP32, storage=0))  # stages recomputed from checkpoints
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert torch.equal(a, b)


@pytest.mark.parametrize('nt', ['256', '1024'])
def test_fused_members_per_chunk_and_block_size(nt):
    """Chunks of 4, 8 and 16 members and blocks of 256 or 1024 threads give the same results (the
    chunk changes only which members a thread holds; FP32 contraction may differ per build)."""
    from mpsw.torch_api import FP32
    B = 16
    res = []
    for M in ('4', '8', '16'):
        m, e = engine(4, {'MPSW_FUSED': '1', 'MPSW_FUSED_M': M, 'MPSW_FUSED_NT': nt})
        du, dh = members(m, B, 5)
        yu, yh = members(m, B, 6)
        res.append(sweep(e, du, dh, yu, yh, FP32))
    assert relmax(res[0], res[1]) < 1e-6
    assert relmax(res[0], res[2]) < 1e-6


def test_split_kernels_serve_other_physics(tmp_path, monkeypatch):
    """With viscosity, drag and wind the window runs the split kernels whatever MPSW_FUSED says.
    Both engines take their launch choices from one tuning cache: FP32 contraction may differ
    between member widths, so the comparison is bit for bit only with the same choices."""
    from mpsw.torch_api import FP32
    monkeypatch.setenv('MPSW_TUNE_CACHE', str(tmp_path / 'tune.txt'))
    B = 8
    cfg = dict(visc2=1e5, visc4=5e14, drag=True, wind=True)
    mf, ef = engine(4, {'MPSW_FUSED': '1'}, **cfg)
    ms, es = engine(4, {'MPSW_FUSED': '0'}, **cfg)
    du, dh = members(mf, B, 7)
    yu, yh = members(mf, B, 8)
    for a, b in zip(sweep(ef, du, dh, yu, yh, FP32), sweep(es, du, dh, yu, yh, FP32)):
        assert torch.equal(a, b)


def test_fused_dot_product():
    """FP32 fused tangent linear and adjoint are transposes up to FP32 rounding."""
    from mpsw.torch_api import FP32
    B = 8
    m, e = engine(5, {'MPSW_FUSED': '1'})
    du, dh = members(m, B, 9)
    yu, yh = members(m, B, 10)
    tu, th, au, ah = sweep(e, du, dh, yu, yh, FP32, nsteps=12)
    lhs = (tu * yu).sum(0) + (th * yh).sum(0)
    rhs = (du * au).sum(0) + (dh * ah).sum(0)
    assert torch.all((lhs - rhs).abs() / lhs.abs() < 1e-5), (lhs, rhs)
