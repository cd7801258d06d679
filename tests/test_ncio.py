"""netCDF grid and trajectory files (mpsw/ncio.py): an MPAS grid file written from a generated
mesh reads back unchanged, a module loaded from the file (the reference driver's read_dims +
read_vars, src/mpas_sw_driver.py:33-119) integrates exactly like one loaded from the mesh, and
the forward demo's trajectory file (demo/run-fwd.py:51-64) round-trips and drives the adjoint
demo's step-by-step reload (demo/run-adj.py:44-45)."""
import numpy as np
import pytest

import oracle as O
from helpers import configure, mesh, setup
from mpsw import ncio


@pytest.mark.parametrize('level', [1, 3])
def test_grid_round_trip(tmp_path, level):
    m = mesh(level)
    path = tmp_path / 'grid.nc'
    ncio.write_grid(str(path), m)
    g = ncio.read_grid(str(path))
    for d in ncio.DIMS:
        assert g[d] == m[d]
    for k in ncio.GRID_VARS:
        a, b = np.asarray(g[k]), np.asarray(m[k])
        assert a.shape == b.shape and np.array_equal(a, b), k
    assert g['on_a_sphere'] and g['sphere_radius'] == 1.0 and g['nVertLevels'] == 1


def test_module_from_grid_file_matches(tmp_path):
    path = tmp_path / 'grid.nc'
    ncio.write_grid(str(path), mesh(2))
    a = O.OracleModule()
    ncio.load_grid(a, str(path))
    configure(a, dt=600.0)
    a.sw_test_case_5()
    a.sw_mpas_init_block()
    b = setup(O.OracleModule(), 2, 'tc5', dt=600.0)
    for _ in range(3):
        a.sw_rk4()
        b.sw_rk4()
    assert np.array_equal(a.u, b.u) and np.array_equal(a.h, b.h)


def test_trajectory_file_round_trip_and_adjoint_reload(tmp_path):
    m = setup(O.OracleModule(), 2, 'tc5', ad=True, dt=600.0)
    w = ncio.TrajectoryWriter(str(tmp_path / 'state.nc'))
    states = []
    for _ in range(4):
        w.append(m)
        states.append((m.u[0, 0].copy(), m.h[0, 0].copy()))
        m.sw_rk4()
    w.write()
    t = ncio.read_trajectory(str(tmp_path / 'state.nc'))
    assert t['u'].shape == (4, m.nedges) and t['h'].shape == (4, m.ncells)
    for i, (u, h) in enumerate(states):
        assert np.array_equal(t['u'][i], u) and np.array_equal(t['h'][i], h)
    assert np.allclose(t['latCell'], np.asarray(m.latcell).ravel() * 180 / np.pi, atol=1e-5)
    # the adjoint demo's loop: reload the state of each step from the file, then sw_rk4_adj
    ref = setup(O.OracleModule(), 2, 'tc5', ad=True, dt=600.0)
    m.u_ad[0, 0, 0] = ref.u_ad[0, 0, 0] = 1.0
    m.h_ad[0, 0, 0] = ref.h_ad[0, 0, 0] = 1.0
    for i in reversed(range(4)):
        m.u[0, 0], m.h[0, 0] = t['u'][i], t['h'][i]
        ref.u[0, 0], ref.h[0, 0] = states[i]
        m.sw_rk4_adj()
        ref.sw_rk4_adj()
    assert np.array_equal(m.u_ad, ref.u_ad) and np.array_equal(m.h_ad, ref.h_ad)


def test_rejects_non_classic_files(tmp_path):
    p = tmp_path / 'x.nc'
    p.write_bytes(b'\x89HDF\r\n\x1a\n' + b'\0' * 64)
    with pytest.raises(ValueError, match='netCDF'):
        ncio.read_grid(str(p))


@pytest.mark.gpu
def test_engine_from_grid_file_matches_oracle(tmp_path):
    """The f2py-compatible engine module loaded from an MPAS grid file reproduces the oracle
    loaded from the same file, bit for bit, over a few steps."""
    from module_sw_mpas import MpasSwModule
    path = tmp_path / 'grid.nc'
    ncio.write_grid(str(path), mesh(3))
    mods = []
    for make in (O.OracleModule, MpasSwModule):
        m = make()
        ncio.load_grid(m, str(path))
        configure(m, dt=600.0)
        m.sw_test_case_5()
        mods.append(m)
    o, g = mods
    g.u[0, 0], g.h[0, 0], g.h_s = o.u[0, 0], o.h[0, 0], o.h_s  # same initial state, bit for bit
    g.fvertex, g.fedge = o.fvertex, o.fedge
    for m in mods:
        m.sw_mpas_init_block()
        for _ in range(3):
            m.sw_rk4()
    assert np.array_equal(g.u[0, 0], o.u[0, 0]) and np.array_equal(g.h[0, 0], o.h[0, 0])
