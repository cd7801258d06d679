"""Seeded synthetic initial conditions for the benchmark workloads.

The reference initialises either from Williamson test cases (``src/mpas_sw_testcases.f90``) or
from an ERA5 file (``src/mpas_sw_driver.py:164-217``) that is not distributed.  The benchmark
workloads replace ERA5 with a seeded balanced flow:

* stream function psi = sum_{n=1..nmax} sum_m c_nm Y_nm (real, orthonormal spherical harmonics),
  c_nm ~ N(0,1) n^-3, drawn with ``numpy.random.default_rng(seed)`` in (n, m=-n..n) order;
* normal velocity u = -(psi(v2) - psi(v1)) / dvEdge, the discrete k x grad(psi) . n that the
  test cases use (``src/mpas_sw_testcases.f90:197-201``), scaled so that max|u| = umax;
* thickness h = h0 + f psi / g on cells (geostrophic balance), f = 2 Omega sin(lat);
* optional topography: Gaussian mountains b, with h reduced by b and h_s = b.

All lengths follow the reference's constants (``src/mpas_sw_module.f90:8-11``).
"""
from __future__ import annotations

import numpy as np

A_EARTH = 6371229.0
OMEGA = 7.29212e-5
GRAVITY = 9.80616

_SCALE_LEN = ('xCell', 'yCell', 'zCell', 'xVertex', 'yVertex', 'zVertex', 'xEdge', 'yEdge',
              'zEdge', 'dvEdge', 'dcEdge')
_SCALE_AREA = ('areaCell', 'areaTriangle', 'kiteAreasOnVertex')


def scale_mesh(mesh: dict, radius: float = A_EARTH) -> dict:
    """Copy of a unit-sphere mesh with lengths scaled by ``radius`` and areas by ``radius**2``
    (the scaling every initialisation path applies, ``src/mpas_sw_driver.py:166-179``)."""
    out = dict(mesh)
    for k in _SCALE_LEN:
        out[k] = mesh[k] * radius
    for k in _SCALE_AREA:
        out[k] = mesh[k] * radius ** 2.0
    return out


def _real_sph_harm_sum(coef, lat, lon, nmax):
    """sum_{n,m} coef[n][m] Y_nm(lat, lon) with orthonormal real spherical harmonics.

    Associated Legendre functions by the standard stable three-term recurrence in n for each m.
    """
    x = np.sin(lat)                      # cos(colatitude)
    s = np.cos(lat)                      # sin(colatitude)
    out = np.zeros_like(lat)
    pmm = np.full_like(lat, np.sqrt(1.0 / (4.0 * np.pi)))
    for m in range(0, nmax + 1):
        if m > 0:
            pmm = pmm * s * np.sqrt((2.0 * m + 1.0) / (2.0 * m))
        cm = np.cos(m * lon)
        sm = np.sin(m * lon)
        pnm2, pnm1 = None, pmm
        for n in range(m, nmax + 1):
            if n == m:
                p = pmm
            elif n == m + 1:
                p = np.sqrt(2.0 * m + 3.0) * x * pmm
            else:
                an = np.sqrt((4.0 * n * n - 1.0) / (n * n - m * m))
                bn = np.sqrt(((n - 1.0) ** 2 - m * m) / (4.0 * (n - 1.0) ** 2 - 1.0))
                p = an * (x * pnm1 - bn * pnm2)
            if n >= 1:
                if m == 0:
                    out += coef[(n, 0)] * p
                else:
                    out += np.sqrt(2.0) * p * (coef[(n, m)] * cm + coef[(n, -m)] * sm)
            if n > m:
                pnm2, pnm1 = pnm1, p
            else:
                pnm1 = p
    return out


def balanced_flow(mesh: dict, seed: int, nmax: int = 20, umax: float = 40.0,
                  h0: float = 5500.0) -> dict:
    """Seeded geostrophically balanced state on a mesh already scaled by the Earth radius.

    Returns ``h`` (nCells), ``u`` (nEdges), ``fVertex``, ``fEdge``, ``fCell``.
    """
    rng = np.random.default_rng(seed)
    coef = {}
    for n in range(1, nmax + 1):
        c = rng.standard_normal(2 * n + 1) * float(n) ** -3.0
        for i, m in enumerate(range(-n, n + 1)):
            coef[(n, m)] = c[i]
    psi_v = _real_sph_harm_sum(coef, mesh['latVertex'], mesh['lonVertex'], nmax)
    psi_c = _real_sph_harm_sum(coef, mesh['latCell'], mesh['lonCell'], nmax)
    v1 = mesh['verticesOnEdge'][:, 0] - 1
    v2 = mesh['verticesOnEdge'][:, 1] - 1
    u = -(psi_v[v2] - psi_v[v1]) / mesh['dvEdge']
    scale = umax / np.abs(u).max()
    u = u * scale
    psi_c = psi_c * scale
    fC = 2.0 * OMEGA * np.sin(mesh['latCell'])
    h = h0 + fC * psi_c / GRAVITY
    return {'h': h, 'u': u, 'fCell': fC,
            'fVertex': 2.0 * OMEGA * np.sin(mesh['latVertex']),
            'fEdge': 2.0 * OMEGA * np.sin(mesh['latEdge'])}


def _great_circle(lat1, lon1, lat2, lon2, radius):
    arg = np.sqrt(np.sin(0.5 * (lat2 - lat1)) ** 2
                  + np.cos(lat1) * np.cos(lat2) * np.sin(0.5 * (lon2 - lon1)) ** 2)
    return 2.0 * radius * np.arcsin(np.minimum(arg, 1.0))


def _random_centres(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    lon = rng.uniform(0.0, 2.0 * np.pi, n)
    return np.arcsin(z), lon


def mountains(mesh: dict, seed: int, count: int = 8, hmin: float = 500.0, hmax: float = 2000.0,
              wmin: float = 500e3, wmax: float = 1500e3) -> np.ndarray:
    """Seeded sum of ``count`` Gaussian mountains on cells: b = sum H exp(-(d/W)^2)."""
    rng = np.random.default_rng(seed)
    lat0, lon0 = _random_centres(rng, count)
    H = rng.uniform(hmin, hmax, count)
    W = rng.uniform(wmin, wmax, count)
    b = np.zeros(mesh['nCells'])
    for k in range(count):
        d = _great_circle(lat0[k], lon0[k], mesh['latCell'], mesh['lonCell'], A_EARTH)
        b += H[k] * np.exp(-(d / W[k]) ** 2)
    return b


def perturbation(mesh: dict, seed: int, count: int = 1, h_std: float = 1.0,
                 u_std: float = 0.1):
    """``count`` i.i.d. perturbations: h' ~ N(0, h_std) per cell, u' ~ N(0, u_std) per edge.

    Shapes (nCells, count) and (nEdges, count): the member index is the trailing dimension.
    """
    rng = np.random.default_rng(seed)
    dh = rng.standard_normal((mesh['nCells'], count)) * h_std
    du = rng.standard_normal((mesh['nEdges'], count)) * u_std
    return dh, du


def cap_masks(mesh: dict, seed: int, count: int, rmin: float = 500e3,
              rmax: float = 1500e3) -> np.ndarray:
    """``count`` spherical-cap masks on cells (radius U(rmin, rmax), uniform random centre),
    shape (nCells, count), values 0/1."""
    rng = np.random.default_rng(seed)
    lat0, lon0 = _random_centres(rng, count)
    r = rng.uniform(rmin, rmax, count)
    out = np.zeros((mesh['nCells'], count))
    for k in range(count):
        d = _great_circle(lat0[k], lon0[k], mesh['latCell'], mesh['lonCell'], A_EARTH)
        out[:, k] = (d < r[k]).astype(np.float64)
    return out


def workload(level: int, seed: int = 0, topography: bool = False):
    """Scaled mesh plus the seeded balanced state (and mountains) for one benchmark workload."""
    from .mesh import icosahedral_mesh
    unit = icosahedral_mesh(level)
    mesh = scale_mesh(unit)
    st = balanced_flow(mesh, seed)
    h_s = np.zeros(mesh['nCells'])
    if topography:
        h_s = mountains(mesh, seed + 1000)
        st['h'] = st['h'] - h_s
    st['h_s'] = h_s
    return unit, mesh, st


# ---- real-data initialisation (the reference driver's test case 7) ------------------------------
def era_to_mpas(lat_grid, lon_grid, var_grid, lat, lon, handle=None):
    """A regular latitude-longitude field (degrees; 1-D axes or the 2-D meshgrid of them) averaged
    onto points (degrees) by the GPU box average of ``mpsw_grid_to_points``, as the reference's
    era2mpas / grid2mpas (src/mpas_sw_driver.py:147-158, src/grid2mpas.f90:21-70): longitudes
    are taken into [0, 360) for the points and the grid (the reference shifts them into the
    latitudes instead, a slip fixed here), and points whose average is NaN get the mean of the
    others.  Returns a float64 numpy array."""
    import ctypes

    import torch

    from . import _lib
    lat_grid, lon_grid = np.asarray(lat_grid, dtype=np.float64), np.asarray(lon_grid, dtype=np.float64)
    lat1d = lat_grid[:, 0] if lat_grid.ndim == 2 else lat_grid
    lon1d = lon_grid[0, :] if lon_grid.ndim == 2 else lon_grid
    lon1d = np.where(lon1d < 0, lon1d + 360.0, lon1d)
    pts_lon = np.asarray(lon, dtype=np.float64).ravel().copy()
    pts_lon[pts_lon < 0] += 360.0
    pts_lat = np.asarray(lat, dtype=np.float64).ravel()
    grid = np.ascontiguousarray(var_grid, dtype=np.float64)
    if grid.shape != (lat1d.size, lon1d.size):
        raise ValueError('field shape %s does not match the axes (%d, %d)' % (grid.shape, lat1d.size, lon1d.size))
    own = handle is None
    h = _lib.Handle() if own else handle
    try:
        dev = [torch.tensor(np.ascontiguousarray(x), device='cuda') for x in (lat1d, lon1d, grid, pts_lat, pts_lon)]
        out = torch.empty(pts_lat.size, dtype=torch.float64, device='cuda')
        p = [ctypes.c_void_p(x.data_ptr()) for x in dev]
        h.call('mpsw_grid_to_points', lat1d.size, lon1d.size, p[0], p[1], p[2], pts_lat.size, p[3], p[4],
               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        var = out.cpu().numpy()
    finally:
        if own:
            h.close()
    bad = np.isnan(var)
    if bad.any():
        var[bad] = var[~bad].mean()
    return var


def init_real(module, lat_grid, lon_grid, z_grid, u_grid, v_grid):
    """The reference driver's real-data initial condition (mpsw_init_real, src/mpas_sw_driver.py:
    161-216) on a module loaded with a unit-sphere grid: mesh scaled to the Earth's radius,
    Coriolis parameters, h from the geopotential z / g and the normal wind from the zonal and
    meridional winds rotated by angleEdge, each averaged onto the mesh by ``era_to_mpas``.
    The fields are one time of the reanalysis, (nlat, nlon) in degrees."""
    a = A_EARTH
    for k in ('xcell', 'ycell', 'zcell', 'xvertex', 'yvertex', 'zvertex', 'xedge', 'yedge', 'zedge',
              'dvedge', 'dcedge'):
        setattr(module, k, np.asarray(getattr(module, k)) * a)
    for k in ('areacell', 'areatriangle', 'kiteareasonvertex'):
        setattr(module, k, np.asarray(getattr(module, k)) * a ** 2.0)
    alpha = 0.0
    late, lone = np.asarray(module.latedge), np.asarray(module.lonedge)
    latv, lonv = np.asarray(module.latvertex), np.asarray(module.lonvertex)
    module.fedge = 2.0 * OMEGA * (-np.cos(lone) * np.cos(late) * np.sin(alpha) + np.sin(late) * np.cos(alpha))
    module.fvertex = 2.0 * OMEGA * (-np.cos(lonv) * np.cos(latv) * np.sin(alpha) + np.sin(latv) * np.cos(alpha))
    r2d = 180.0 / np.pi
    latc, lonc = np.asarray(module.latcell).ravel() * r2d, np.asarray(module.loncell).ravel() * r2d
    module.h[0, 0] = era_to_mpas(lat_grid, lon_grid, np.asarray(z_grid) / GRAVITY, latc, lonc)
    ue = era_to_mpas(lat_grid, lon_grid, u_grid, late.ravel() * r2d, lone.ravel() * r2d)
    ve = era_to_mpas(lat_grid, lon_grid, v_grid, late.ravel() * r2d, lone.ravel() * r2d)
    ang = np.asarray(module.angleedge).ravel()
    module.u[0, 0] = np.cos(ang) * ue + np.sin(ang) * ve
