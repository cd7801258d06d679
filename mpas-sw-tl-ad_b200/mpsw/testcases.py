"""Williamson et al. (1992, J. Comput. Phys. 102) shallow-water test cases 1, 2, 5 and 6 as the
reference module sets them up (``src/mpas_sw_testcases.f90``): each scales the unit-sphere
mesh by the Earth radius, then fills u (normal velocity from a vertex stream function), h,
and, for cases 2 and 5, the Coriolis parameters.  Case 5 also sets the mountain h_s and tracer
1; case 6 leaves fEdge/fVertex untouched, as the reference does.

They operate on a module object with the f2py attribute surface (``mpas_sw_module``), host
side, in FP64 numpy.
"""
from __future__ import annotations

import numpy as np

PII = 3.141592653589793
A = 6371229.0
OMEGA = 7.29212e-5
GRAVITY = 9.80616


def _scale_mesh(m):
    for n in ('xcell', 'ycell', 'zcell', 'xvertex', 'yvertex', 'zvertex', 'xedge', 'yedge',
              'zedge', 'dvedge', 'dcedge'):
        arr = getattr(m, n)
        arr[...] = arr * A
    for n in ('areacell', 'areatriangle', 'kiteareasonvertex'):
        arr = getattr(m, n)
        arr[...] = arr * A ** 2.0


def _wind_from_psi(m, psi):
    v1 = m.verticesonedge[0] - 1
    v2 = m.verticesonedge[1] - 1
    m.u[0, 0, :] = -1.0 * (psi[v2] - psi[v1]) / m.dvedge


def _solid_body_psi(m, u0, alpha):
    lat, lon = m.latvertex, m.lonvertex
    return -A * u0 * (np.sin(lat) * np.cos(alpha) - np.cos(lon) * np.cos(lat) * np.sin(alpha))


def _coriolis(m, alpha):
    m.fedge[:] = 2.0 * OMEGA * (-np.cos(m.lonedge) * np.cos(m.latedge) * np.sin(alpha)
                                + np.sin(m.latedge) * np.cos(alpha))
    m.fvertex[:] = 2.0 * OMEGA * (-np.cos(m.lonvertex) * np.cos(m.latvertex) * np.sin(alpha)
                                  + np.sin(m.latvertex) * np.cos(alpha))


def _sphere_distance(lat1, lon1, lat2, lon2, radius):
    arg = np.sqrt(np.sin(0.5 * (lat2 - lat1)) ** 2
                  + np.cos(lat1) * np.cos(lat2) * np.sin(0.5 * (lon2 - lon1)) ** 2)
    return 2. * radius * np.arcsin(arg)


def test_case_1(m):
    """Advection of a cosine bell over the pole (wind frozen during the run)."""
    u0 = 2.0 * PII * A / (12.0 * 86400.0)
    h0, theta_c, lambda_c, alpha = 1000.0, 0.0, 3.0 * PII / 2.0, PII / 4.0
    _scale_mesh(m)
    _wind_from_psi(m, _solid_body_psi(m, u0, alpha))
    r = _sphere_distance(theta_c, lambda_c, m.latcell, m.loncell, A)
    m.h[0, 0, :] = np.where(r < A / 3.0, (h0 / 2.0) * (1.0 + np.cos(PII * r * 3.0 / A)), h0 / 2.0)


def _geostrophic_h(m, u0, gh0, alpha):
    x = (-np.cos(m.loncell) * np.cos(m.latcell) * np.sin(alpha) + np.sin(m.latcell) * np.cos(alpha))
    return (gh0 - (A * OMEGA * u0 + 0.5 * u0 ** 2.0) * x ** 2.0) / GRAVITY


def test_case_2(m):
    """Global steady-state nonlinear zonal geostrophic flow."""
    u0 = 2.0 * PII * A / (12.0 * 86400.0)
    gh0, alpha = 29400.0, 0.0
    _scale_mesh(m)
    _wind_from_psi(m, _solid_body_psi(m, u0, alpha))
    _coriolis(m, alpha)
    m.h[0, 0, :] = _geostrophic_h(m, u0, gh0, alpha)


def test_case_5(m):
    """Zonal flow over an isolated mountain."""
    u0, gh0, hs0 = 20., 5960.0 * GRAVITY, 2000.
    theta_c, lambda_c, rr, alpha = PII / 6.0, 3.0 * PII / 2.0, PII / 9.0, 0.0
    _scale_mesh(m)
    _wind_from_psi(m, _solid_body_psi(m, u0, alpha))
    _coriolis(m, alpha)
    lon = m.loncell
    lon[lon < 0.0] += 2.0 * PII
    r = np.sqrt(np.minimum(rr ** 2.0, (lon - lambda_c) ** 2.0 + (m.latcell - theta_c) ** 2.0))
    m.h_s[:] = hs0 * (1.0 - r / rr)
    if m.tracers is not None and m.tracers.shape[1] >= 1:
        m.tracers[0, 0, 0, :] = 1.0 - r / rr
    if m.tracers is not None and m.tracers.shape[1] > 1:
        r2 = np.sqrt(np.minimum(rr ** 2.0, (lon - lambda_c) ** 2.0
                                + (m.latcell - theta_c - PII / 6.0) ** 2.0))
        m.tracers[0, 1, 0, :] = 1.0 - r2 / rr
    m.h[0, 0, :] = _geostrophic_h(m, u0, gh0, alpha) - m.h_s


def test_case_6(m):
    """Rossby-Haurwitz wave (wavenumber 4).  As in the reference, fEdge/fVertex are not set."""
    h0, w, K, R = 8000.0, 7.848e-6, 7.848e-6, 4.0
    _scale_mesh(m)
    lat, lon = m.latvertex, m.lonvertex
    psi = -A * A * w * np.sin(lat) + A * A * K * (np.cos(lat) ** R) * np.sin(lat) * np.cos(R * lon)
    _wind_from_psi(m, psi)
    c = np.cos(m.latcell)
    aa = (0.5 * w * (2.0 * OMEGA + w) * c ** 2.0
          + 0.25 * K ** 2.0 * c ** (2.0 * R) * ((R + 1.0) * c ** 2.0 + 2.0 * R ** 2.0 - R - 2.0
                                                - 2.0 * R ** 2.0 * c ** (-2.0)))
    bb = (2.0 * (OMEGA + w) * K / ((R + 1.0) * (R + 2.0))) * c ** R * (
        (R ** 2.0 + 2.0 * R + 2.0) - ((R + 1.0) * c) ** 2.0)
    cc = 0.25 * K ** 2.0 * c ** (2.0 * R) * ((R + 1.0) * c ** 2.0 - R - 2.0)
    lonc = m.loncell
    m.h[0, 0, :] = (GRAVITY * h0 + A * A * aa + A * A * bb * np.cos(R * lonc)
                    + A * A * cc * np.cos(2.0 * R * lonc)) / GRAVITY
