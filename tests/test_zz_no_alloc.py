"""mpsw_compute_tend_noalloc: the tendency entry point for callers that may not allocate
device memory (it keeps its diagnostics in a fixed array inside the library instead).

It must give what the allocating entry point, mpsw_compute_tend, gives for the same state, and
what the oracle's sw_compute_tend gives, on consecutive calls that reuse the shared scratch;
the calls must leave the device's free memory unchanged (nothing allocated, nothing loaded);
and it must refuse a mesh whose diagnostics do not fit in that scratch.  This file is
collected last so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import pytest

import oracle as O
from helpers import maxrel, setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

TOL = 1e-13      # the parity tolerance of the FP64 forward stencils (tests/test_gpu_parity.py)
TOL_ORACLE = 1e-12


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize('phys', [dict(), dict(visc2=2e5, visc4=1e15, drag=True, wind=True)])
def test_noalloc_tendencies_match_compute_tend(phys):
    from mpsw.torch_api import Engine
    m = setup(MpasSwModule(), 4, 'seeded', **phys)
    o = setup(O.OracleModule(), 4, 'seeded', **phys)
    o.compute_tend()                                  # the oracle's sw_compute_tend
    e = Engine(m)
    m.compute_tend()                                  # the allocating entry point
    ref_u, ref_h = m.tend_u[0].copy(), m.tend_h[0].copy()
    u = e.to_internal(torch.tensor(m.u[0, 0], device='cuda'), 1)
    h = e.to_internal(torch.tensor(m.h[0, 0], device='cuda'), 0)
    tu = torch.empty_like(u)
    th = torch.empty_like(h)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = m.handle.lib
    for call in range(2):                             # the second call reuses dirty scratch
        tu.fill_(float('nan'))
        th.fill_(float('nan'))
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = L.mpsw_compute_tend_noalloc(m.handle.ptr, _p(u), _p(h), _p(tu), _p(th), stream)
        assert rc == 0, L.mpsw_last_error(m.handle.ptr)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (call, free0, free1)   # the call took no device memory
        got_u = e.to_reference(tu, 1)[:, 0].cpu().numpy()
        got_h = e.to_reference(th, 0)[:, 0].cpu().numpy()
        assert maxrel(got_u, ref_u) <= TOL, call
        assert maxrel(got_h, ref_h) <= TOL, call
        assert maxrel(got_u, o.tend_u[0]) <= TOL_ORACLE, call
        assert maxrel(got_h, o.tend_h[0]) <= TOL_ORACLE, call


def test_noalloc_refuses_meshes_beyond_its_scratch():
    m = setup(MpasSwModule(), 7, 'tc5')               # 163842 cells: needs about 2.46M doubles
    u = torch.zeros(int(m.nedges), dtype=torch.float64, device='cuda')
    h = torch.zeros(int(m.ncells), dtype=torch.float64, device='cuda')
    L = m.handle.lib
    rc = L.mpsw_compute_tend_noalloc(m.handle.ptr, _p(u), _p(h), _p(u), _p(h), None)
    assert rc != 0
    assert b'maximum' in L.mpsw_last_error(m.handle.ptr)
