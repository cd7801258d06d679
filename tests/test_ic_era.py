"""Box average of a latitude-longitude field onto mesh points (ERA5 initialisation,
src/grid2mpas.f90): the oracle's restatement on a hand-checked case and its edge behaviour; the
GPU kernel (mpsw_grid_to_points) bit-identical to the oracle on a 1-degree grid and level-3
cells and edges; and the driver's real-data initial condition built from it."""
import numpy as np
import pytest

import oracle as O
from helpers import mesh


def test_oracle_box_average_by_hand():
    lat1d = np.array([10.0, 0.0, -10.0])          # descending, as ERA5
    lon1d = np.array([0.0, 90.0, 180.0, 270.0])
    grid = np.arange(12.0).reshape(3, 4)
    # interior point nearest (1, 1): the full 3 x 3 block (rows 0-2, columns 0-2)
    assert O.grid_to_points(lat1d, lon1d, grid, [1.0], [95.0])[0] == grid[0:3, 0:3].mean()
    # corner point nearest (0, 0): clamped 2 x 2 block
    assert O.grid_to_points(lat1d, lon1d, grid, [40.0], [-5.0])[0] == grid[0:2, 0:2].sum() / 4.0
    # ties go to the first index (minloc): 5 is as far from 10 as from 0
    assert O.grid_to_points(lat1d, lon1d, grid, [5.0], [0.0])[0] == grid[0:2, 0:2].sum() / 4.0


def era_like(nlat=181, nlon=360, seed=0):
    rng = np.random.default_rng(seed)
    lat1d = np.linspace(90.0, -90.0, nlat)
    lon1d = np.arange(nlon) * (360.0 / nlon)
    lon2, lat2 = np.meshgrid(lon1d, lat1d)
    field = 5500.0 + 300.0 * np.cos(np.radians(lat2)) * np.sin(2 * np.radians(lon2)) + rng.standard_normal(lon2.shape)
    return lat1d, lon1d, field


@pytest.mark.gpu
def test_gpu_box_average_matches_oracle():
    from mpsw import ic
    lat1d, lon1d, field = era_like()
    m = mesh(3)
    r2d = 180.0 / np.pi
    for lat, lon in ((m['latCell'], m['lonCell']), (m['latEdge'], m['lonEdge'])):
        lat, lon = lat * r2d, lon * r2d
        got = ic.era_to_mpas(lat1d, lon1d, field, lat, lon)
        lon_w = np.where(lon < 0, lon + 360.0, lon)  # longitudes into the axis range (the fix)
        ref = O.grid_to_points(lat1d, lon1d, field, lat, lon_w)
        assert np.array_equal(got, ref)


@pytest.mark.gpu
def test_real_data_initial_condition_runs():
    """Test case 7 of the reference driver from synthetic reanalysis fields: balanced-looking
    geopotential and winds averaged onto a level-3 mesh, then a few steps stay finite."""
    from module_sw_mpas import MpasSwModule
    from helpers import configure
    from mpsw import ic
    m = MpasSwModule()
    O.load_mesh(m, mesh(3))
    configure(m, dt=600.0, tc=7)
    lat1d, lon1d, z = era_like(seed=1)
    z = (z - 5500.0) * 9.80616 + 5500.0 * 9.80616
    u = 10.0 * np.cos(np.radians(lat1d))[:, None] * np.ones((1, lon1d.size))
    v = np.zeros_like(u)
    ic.init_real(m, lat1d, lon1d, z, u, v)
    assert abs(np.mean(m.h[0, 0]) - 5500.0) < 50.0
    m.sw_mpas_init_block()
    for _ in range(3):
        m.sw_rk4()
    assert np.all(np.isfinite(m.h[0, 0])) and np.all(np.isfinite(m.u[0, 0]))
