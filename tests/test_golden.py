"""Golden vectors (tests/golden/golden_L*.npz, written by tests/golden/make_golden.py).

CPU: the mesh generator and the oracle reproduce the recorded numbers bit for bit, and the
recorded tangent-linear / adjoint pairs satisfy the dot-product identity.  GPU: the engine,
driven through the f2py-style module from the recorded inputs, reproduces them: forward and
tangent-linear bit for bit, the adjoint (gathers in another order than the reference's
scatters) within 1e-11 of the largest value."""
import os

import numpy as np
import pytest

import oracle as O
from helpers import maxrel, mesh

HERE = os.path.dirname(os.path.abspath(__file__))
import sys  # noqa: E402
sys.path.insert(0, os.path.join(HERE, 'golden'))
import make_golden as G  # noqa: E402

LEVELS = G.LEVELS
EXACT = ('tc5_u1', 'tc5_h1', 'tc5_u12', 'tc5_h12', 'seeded_u1', 'seeded_h1', 'seeded_utl1',
         'seeded_htl1')
ADJOINT = ('seeded_uad0', 'seeded_had0')


def golden(level):
    with np.load(G.path(level)) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize('level', LEVELS)
def test_mesh_matches_golden_hash(level):
    assert G.mesh_hash(mesh(level)) == str(golden(level)['mesh_sha256'])


@pytest.mark.parametrize('level', LEVELS)
def test_golden_dot_products(level):
    g = golden(level)
    lhs = g['seeded_utl1'] @ g['seeded_au'] + g['seeded_htl1'] @ g['seeded_ah']
    rhs = g['seeded_du'] @ g['seeded_uad0'] + g['seeded_dh'] @ g['seeded_had0']
    assert abs(lhs - rhs) / abs(lhs) < 1e-12
    l, r = g['seeded_link']
    assert abs(l - r) / abs(l) < 1e-12


@pytest.mark.parametrize('level', LEVELS)
def test_oracle_reproduces_golden(level):
    O.build()
    g = golden(level)
    out = G.compute(O.OracleModule, level, inputs=g)
    for k, v in g.items():
        assert np.array_equal(out[k], v), k


@pytest.mark.gpu
@pytest.mark.parametrize('level', LEVELS)
def test_engine_reproduces_golden(level):
    from module_sw_mpas import MpasSwModule
    g = golden(level)
    out = G.compute(MpasSwModule, level, inputs=g)
    for k in EXACT:
        assert np.array_equal(out[k], g[k]), k
    for k in ADJOINT:
        assert maxrel(out[k], g[k]) <= 1e-11, k
    l, r = out['seeded_link']
    gl, gr = g['seeded_link']
    assert abs(l - gl) / abs(gl) < 1e-12 and abs(r - gr) / abs(gr) < 1e-11
