"""Binomial checkpointing of long windows (mpsw_window_snapshots): the adjoint sweep reversed with
a few snapshot states gives exactly what the stored-stage and two-level sweeps give, and it
recomputes the least number of nonlinear steps its schedule allows (Griewank's revolve bound,
checked against a brute-force minimum over every first advance)."""
from functools import lru_cache

import numpy as np
import pytest

from helpers import setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@lru_cache(maxsize=None)
def least_steps(n, s):
    """Fewest forward steps to reverse n steps from a held start state with s free slots."""
    if n <= 1:
        return 0
    if s == 0:
        return n * (n - 1) // 2
    return min(m + least_steps(n - m, s - 1) + least_steps(m, s) for m in range(1, n))


@pytest.mark.parametrize('prec_name', ['FP64', 'FP32'])
def test_binomial_matches_stored_and_two_level(prec_name):
    from mpsw import torch_api
    prec = getattr(torch_api, prec_name)
    m = setup(MpasSwModule(), 3, 'seeded', dt=600.0)
    e = torch_api.Engine(m)
    nsteps, B = 120, 4
    rng = np.random.default_rng(3)
    au = torch.tensor(rng.standard_normal((int(m.nedges), B)) * 0.1, device='cuda')
    ah = torch.tensor(rng.standard_normal((int(m.ncells), B)), device='cuda')
    runs = {}
    for name, kw in [('stored', dict(storage=-1)), ('two-level', dict(storage=0, ckpt_every=10)),
                     ('binomial', dict(storage=0, snapshots=4))]:
        w = e.window(nsteps, **kw)
        runs[name] = w.ad(au, ah, prec) + (w.forward_steps(),)
    for name in ('two-level', 'binomial'):
        assert torch.equal(runs[name][0], runs['stored'][0]), name
        assert torch.equal(runs[name][1], runs['stored'][1]), name
    assert runs['stored'][2] == 0
    assert runs['two-level'][2] == nsteps - nsteps // 10
    assert runs['binomial'][2] == least_steps(nsteps, 4)
    e.window(1, snapshots=0)  # back to the default for the module's other users
