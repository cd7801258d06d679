"""Host-side pieces of bench.py: the algorithmic byte model of the member kernels and the
DRAM traffic read back from the committed ncu summaries (both summary formats)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def sizes(level):
    c = 10 * 4 ** level + 2
    return c, 3 * c - 6, 2 * c - 4


def test_kernel_bytes_model():
    nC, nE, nV = sizes(5)
    S = 10 * nE - 60
    fp32 = {k: bench.kernel_bytes(k, nC, nE, nV, S, 64, 4) for k in ('tl_stage', 'ad_stage', 'tl_edge_tend')}
    fp64 = {k: bench.kernel_bytes(k, nC, nE, nV, S, 64, 8) for k in ('tl_stage', 'ad_stage', 'tl_edge_tend')}
    # the level-5, 64-member figure: 3 E-rows gathered + 2 cell rows + the RK bookkeeping of a
    # middle stage (rounded input read, provisional state and tendency written) + lists and base
    assert fp32['tl_edge_tend'] == 55747104
    assert all(fp64[k] > fp32[k] for k in fp32)
    # members dominate: doubling B nearly doubles a stage's bytes
    assert 1.9 < bench.kernel_bytes('ad_stage', nC, nE, nV, S, 128, 4) / fp32['ad_stage'] < 2.0


@pytest.mark.parametrize('level', [5, 7])
def test_traffic_from_profiles(level):
    t = bench.traffic_of('tl_edge_tend', level, 64)
    alg = bench.kernel_bytes('tl_edge_tend', *sizes(level), 10 * sizes(level)[1] - 60, 64, 4)
    assert t is not None and 0.5 * alg < t < 1.5 * alg
    assert bench.traffic_of('no_such_kernel', level, 64) is None
