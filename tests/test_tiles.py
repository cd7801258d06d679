"""Host checks of the halo tiles of the fused member stages (csrc/mpsw_tiles.cpp): every cell and
every edge is owned by exactly one tile, the builder's own check that no phase of a stage reads
outside its tile passes for several tile sizes, and a block's shared memory stays within the
227 KB a B200 block may use at the default tile size.  The builder is compiled from the package's
sources with g++ (it is host code) through tests/tile_check.cpp."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import mesh

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), 'mpas-sw-tl-ad_b200', 'csrc')


@pytest.fixture(scope='module')
def lib(tmp_path_factory):
    gxx = shutil.which('g++')
    if not gxx:
        pytest.skip('no g++')
    out = str(tmp_path_factory.mktemp('tiles') / 'libtilecheck.so')
    subprocess.run([gxx, '-O2', '-std=c++17', '-shared', '-fPIC', '-I' + CSRC,
                    '-x', 'c++', os.path.join(CSRC, 'mpsw_setup.cpp'),
                    '-x', 'c++', os.path.join(CSRC, 'mpsw_tiles.cpp'),
                    '-x', 'c++', os.path.join(HERE, 'tile_check.cpp'), '-o', out], check=True)
    return ctypes.CDLL(out)


def check(lib, level, K, adjoint, budget_kb=100):
    m = mesh(level)
    keep = []

    def p(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(ctypes.c_void_p)
    xyz = (ctypes.c_void_p * 9)(*[p(m[k], np.float64) for k in ('xCell', 'yCell', 'zCell', 'xEdge', 'yEdge',
                                                               'zEdge', 'xVertex', 'yVertex', 'zVertex')])
    out = np.zeros(7, dtype=np.int64)
    err = ctypes.create_string_buffer(512)
    rc = lib.tile_check(ctypes.c_int(m['nCells']), ctypes.c_int(m['nEdges']), ctypes.c_int(m['nVertices']),
                        ctypes.c_int(m['maxEdges']), ctypes.c_int(m['maxEdges2']),
                        *[p(m[k], np.int32) for k in ('cellsOnEdge', 'verticesOnEdge', 'edgesOnEdge',
                                                     'nEdgesOnEdge', 'edgesOnCell', 'nEdgesOnCell',
                                                     'cellsOnVertex', 'edgesOnVertex')],
                        *[p(m[k], np.float64) for k in ('weightsOnEdge', 'kiteAreasOnVertex', 'dcEdge', 'dvEdge',
                                                       'areaCell', 'areaTriangle')],
                        xyz, ctypes.c_int(K), ctypes.c_int(budget_kb), ctypes.c_int(int(adjoint)),
                        out.ctypes.data_as(ctypes.c_void_p), err, ctypes.c_int(512))
    assert rc == 0, err.value.decode()
    return m, out


@pytest.mark.parametrize('adjoint', [False, True])
@pytest.mark.parametrize('level,K', [(2, 1), (3, 17), (4, 64), (5, 64), (5, 200)])
def test_tiles_cover_the_mesh_once(lib, level, K, adjoint):
    m, out = check(lib, level, K, adjoint)
    ntiles, sc, se, bad_c, bad_e = out[:5]
    assert ntiles >= (m['nCells'] + K - 1) // K   # runs of at most K cells
    assert sc == m['nCells'] and se == m['nEdges']
    assert bad_c == 0 and bad_e == 0


@pytest.mark.parametrize('adjoint', [False, True])
def test_tiles_fit_the_shared_memory_budget(lib, adjoint):
    _, out = check(lib, 6, 1024, adjoint, budget_kb=100)
    assert out[5] <= 100 * 1024
    _, out = check(lib, 6, 1024, adjoint, budget_kb=60)
    assert out[5] <= 60 * 1024
