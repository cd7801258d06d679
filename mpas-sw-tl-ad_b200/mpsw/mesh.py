"""Quasi-uniform spherical Voronoi (TRiSK) mesh from a recursively bisected icosahedron.

The reference reads its mesh from an MPAS grid file (``src/mpas_sw_driver.py:64-119``); no such
file ships with it, so this module builds one.  The output is a dict keyed by the MPAS netCDF
variable names, laid out exactly as ``infile[name][()]`` would return them (C order, first axis
the mesh entity, 1-based indices, 0 in unused slots), so that ``arr.T`` is what the reference
driver assigns to the f2py module (``mpsw.cellsonedge = infile['cellsOnEdge'][()].T``).

Conventions (the ones the reference stencils rely on):

* the normal of edge e points from ``cellsOnEdge(1,e)`` to ``cellsOnEdge(2,e)``
  (divergence sign, ``src/mpas_sw_dyncore.f90:222-236``);
* the tangent t = k x n points from ``verticesOnEdge(1,e)`` to ``verticesOnEdge(2,e)``
  (circulation sign, ``src/mpas_sw_dyncore.f90:208-214``);
* ``edgesOnCell``/``verticesOnCell``/``cellsOnCell`` run counter-clockwise seen from outside;
  ``verticesOnCell(i)`` is the vertex shared by ``edgesOnCell(i)`` and ``edgesOnCell(i+1)``;
* ``cellsOnVertex`` runs counter-clockwise; ``edgesOnVertex(i)`` joins ``cellsOnVertex(i)`` and
  ``cellsOnVertex(i+1)``; ``kiteAreasOnVertex(i,v)`` is the part of triangle v inside
  ``cellsOnVertex(i,v)``;
* ``areaTriangle`` and ``areaCell`` are the exact sums of their kites, so the kite fractions of a
  cell add up to one to rounding;
* ``weightsOnEdge``/``edgesOnEdge`` are the TRiSK tangential-velocity weights
  (Thuburn et al. 2009, J. Comput. Phys. 228; Ringler et al. 2010, J. Comput. Phys. 229),
  derived here from the kite mass balance: for edge e of cell i and another edge e' of i reached
  by going m steps counter-clockwise from e, ``w = n_{e,i} n_{e',i} (1/2 - sum_{j<m} R_{i,j})
  dvEdge(e') / dcEdge(e)`` with R the kite fractions of the vertices passed.  ``v = sum w u``
  is then the velocity component along t, the weights are antisymmetric after scaling by
  ``dcEdge*dvEdge`` (energy-neutral Coriolis term) and, on every vertex, the circulation of the
  reconstructed v equals minus the kite-weighted sum of the cell divergences of u (the TRiSK
  steady-geostrophic-mode identity), exactly to rounding.

Geometry is on the unit sphere, as MPAS grid files are; the test-case/IC code scales it by the
Earth radius (``src/mpas_sw_testcases.f90:173-186``).
"""
from __future__ import annotations

import numpy as np

MAX_EDGES = 6
MAX_EDGES2 = 12
VERTEX_DEGREE = 3


def _normalize(x):
    return x / np.linalg.norm(x, axis=-1, keepdims=True)


def _arc(a, b):
    """Great-circle distance between unit vectors (rows)."""
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=-1), np.einsum('ij,ij->i', a, b))


def _tri_area(a, b, c):
    """Signed area of the spherical triangle (a,b,c) on the unit sphere (positive if CCW)."""
    num = np.einsum('ij,ij->i', a, np.cross(b, c))
    den = 1.0 + np.einsum('ij,ij->i', a, b) + np.einsum('ij,ij->i', b, c) + np.einsum('ij,ij->i', c, a)
    return 2.0 * np.arctan2(num, den)


def _icosahedron():
    p = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p),
                  (0, -1, -p), (0, 1, -p), (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)],
                 dtype=np.float64)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9),
                  (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2),
                  (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
                  (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    return _normalize(v), f


def _bisect(P, F):
    nP = P.shape[0]
    nF = F.shape[0]
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    es = np.sort(e, axis=1)
    key = es[:, 0] * nP + es[:, 1]
    uk, inv = np.unique(key, return_inverse=True)
    a, b = uk // nP, uk % nP
    mid = _normalize(P[a] + P[b])
    m = nP + inv
    m01, m12, m20 = m[:nF], m[nF:2 * nF], m[2 * nF:]
    f0, f1, f2 = F[:, 0], F[:, 1], F[:, 2]
    newF = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([m01, f1, m12], 1),
                           np.stack([m20, m12, f2], 1), np.stack([m01, m12, m20], 1)])
    return np.concatenate([P, mid]), newF


def _tangent_basis(r):
    """Right-handed tangent basis (e1, e2) at unit vectors r with e1 x e2 = r."""
    ref = np.zeros_like(r)
    ref[:, 2] = 1.0
    polar = np.abs(r[:, 2]) > 0.9
    ref[polar] = (1.0, 0.0, 0.0)
    e1 = _normalize(np.cross(ref, r))
    e2 = np.cross(r, e1)
    return e1, e2


def _latlon(x):
    lat = np.arcsin(np.clip(x[:, 2], -1.0, 1.0))
    lon = np.arctan2(x[:, 1], x[:, 0])
    lon = np.where(lon < 0.0, lon + 2.0 * np.pi, lon)
    return lat, lon


def icosahedral_mesh(level: int) -> dict:
    """Build the level-``level`` bisected-icosahedron TRiSK mesh.

    Counts: nCells = 10*4**level + 2, nEdges = 30*4**level, nVertices = 20*4**level.
    Returns the MPAS grid-file variables (see module docstring) plus the dimension sizes.
    """
    P, F = _icosahedron()
    for _ in range(level):
        P, F = _bisect(P, F)
    N, V = P.shape[0], F.shape[0]

    # counter-clockwise triangles seen from outside
    a, b, c = P[F[:, 0]], P[F[:, 1]], P[F[:, 2]]
    orient = np.einsum('ij,ij->i', np.cross(b - a, c - a), a + b + c)
    F = np.where((orient < 0)[:, None], F[:, [0, 2, 1]], F)
    a, b, c = P[F[:, 0]], P[F[:, 1]], P[F[:, 2]]
    xV = _normalize(np.cross(b - a, c - a))            # circumcentre on the sphere

    # ---- edges: directed triangle sides (F[:,i] -> F[:,i+1]) ----
    dsrc = np.concatenate([F[:, 0], F[:, 1], F[:, 2]])
    ddst = np.concatenate([F[:, 1], F[:, 2], F[:, 0]])
    dface = np.tile(np.arange(V), 3)
    lo, hi = np.minimum(dsrc, ddst), np.maximum(dsrc, ddst)
    key = lo * N + hi
    order = np.argsort(key, kind='stable')
    E = order.size // 2
    first, second = order[0::2], order[1::2]
    assert np.all(key[first] == key[second])
    edge_of_directed = np.empty(order.size, dtype=np.int64)
    edge_of_directed[first] = np.arange(E)
    edge_of_directed[second] = np.arange(E)
    c1 = lo[first]
    c2 = hi[first]
    # the face in which c1 -> c2 appears counter-clockwise lies to the left of n, i.e. on the
    # t = k x n side: that circumcentre is verticesOnEdge(2)
    fwd_is_first = dsrc[first] == c1
    face_fwd = np.where(fwd_is_first, dface[first], dface[second])
    face_bwd = np.where(fwd_is_first, dface[second], dface[first])
    v1, v2 = face_bwd, face_fwd

    xC = P
    xE = _normalize(xC[c1] + xC[c2])
    dc = _arc(xC[c1], xC[c2])
    dv = _arc(xV[v1], xV[v2])

    # ---- vertices: cellsOnVertex (CCW), edgesOnVertex(i) between cov(i) and cov(i+1) ----
    cov = F.copy()
    eov = np.stack([edge_of_directed[0 * V:1 * V], edge_of_directed[1 * V:2 * V],
                    edge_of_directed[2 * V:3 * V]], 1)

    # kites: quadrilateral (c_i, mid(c_i,c_{i+1}), vertex, mid(c_{i-1},c_i))
    kites = np.empty((V, 3))
    for i in range(3):
        ci = xC[cov[:, i]]
        cn = xC[cov[:, (i + 1) % 3]]
        cp = xC[cov[:, (i + 2) % 3]]
        mn = _normalize(ci + cn)
        mp = _normalize(cp + ci)
        kites[:, i] = _tri_area(ci, mn, xV) + _tri_area(ci, xV, mp)
    areaTriangle = kites[:, 0] + kites[:, 1] + kites[:, 2]
    areaCell = np.zeros(N)
    for i in range(3):
        np.add.at(areaCell, cov[:, i], kites[:, i])

    # ---- cells: edgesOnCell counter-clockwise ----
    ce = np.concatenate([c1, c2])
    ee = np.concatenate([np.arange(E), np.arange(E)])
    o = np.argsort(ce, kind='stable')
    nEoC = np.bincount(ce, minlength=N)
    start = np.concatenate([[0], np.cumsum(nEoC)[:-1]])
    slot = np.arange(o.size) - start[ce[o]]
    eoc = np.full((N, MAX_EDGES), -1, dtype=np.int64)
    eoc[ce[o], slot] = ee[o]
    e1b, e2b = _tangent_basis(xC)
    ang = np.full((N, MAX_EDGES), np.inf)
    valid = eoc >= 0
    d = xE[np.where(valid, eoc, 0)] - xC[:, None, :]
    ang_v = np.arctan2(np.einsum('nkj,nj->nk', d, e2b), np.einsum('nkj,nj->nk', d, e1b))
    ang[valid] = ang_v[valid]
    srt = np.argsort(ang, axis=1)
    eoc = np.take_along_axis(eoc, srt, axis=1)

    rows = np.arange(N)
    voc = np.full((N, MAX_EDGES), -1, dtype=np.int64)
    coc = np.full((N, MAX_EDGES), -1, dtype=np.int64)
    for i in range(MAX_EDGES):
        has = i < nEoC
        ea = eoc[:, i]
        eb = eoc[rows, (i + 1) % np.maximum(nEoC, 1)]
        ea_ = np.where(has, ea, 0)
        eb_ = np.where(has, eb, 0)
        va1, va2 = v1[ea_], v2[ea_]
        vb1, vb2 = v1[eb_], v2[eb_]
        common = np.where((va1 == vb1) | (va1 == vb2), va1, va2)
        voc[has, i] = common[has]
        other = np.where(c1[ea_] == rows, c2[ea_], c1[ea_])
        coc[has, i] = other[has]

    # kite fraction of each (cell, vertex slot)
    R = np.zeros((N, MAX_EDGES))
    for i in range(MAX_EDGES):
        has = i < nEoC
        vv = np.where(has, voc[:, i], 0)
        corner = np.argmax(cov[vv] == rows[:, None], axis=1)
        R[has, i] = kites[vv, corner][has] / areaCell[has]

    # ---- TRiSK weights ----
    nEoE = nEoC[c1] + nEoC[c2] - 2
    eoe = np.full((E, MAX_EDGES2), -1, dtype=np.int64)
    woe = np.zeros((E, MAX_EDGES2))
    for p in range(MAX_EDGES):
        hasp = p < nEoC
        cc = rows[hasp]
        n = nEoC[hasp]
        e = eoc[hasp, p]
        side1 = c1[e] == cc
        sgn_e = np.where(side1, 1.0, -1.0)
        base = np.where(side1, 0, nEoC[c1[e]] - 1)
        cum = np.zeros(cc.size)
        for m in range(1, MAX_EDGES):
            hasm = m < n
            j = (p + m - 1) % n
            cum = cum + R[cc, j]
            ep = eoc[cc, (p + m) % n]
            sgn_ep = np.where(c1[ep] == cc, 1.0, -1.0)
            w = sgn_e * sgn_ep * (0.5 - cum) * dv[ep] / dc[e]
            s = base + m - 1
            eoe[e[hasm], s[hasm]] = ep[hasm]
            woe[e[hasm], s[hasm]] = w[hasm]

    latC, lonC = _latlon(xC)
    latE, lonE = _latlon(xE)
    latV, lonV = _latlon(xV)
    east = np.stack([-np.sin(lonE), np.cos(lonE), np.zeros(E)], 1)
    north = np.cross(xE, east)
    nrm = _normalize(xC[c2] - xC[c1])
    angleEdge = np.arctan2(np.einsum('ij,ij->i', nrm, north), np.einsum('ij,ij->i', nrm, east))

    def one(x):  # 1-based, 0 in unused slots
        return np.where(x >= 0, x + 1, 0).astype(np.int32)

    return {
        'nCells': N, 'nEdges': E, 'nVertices': V, 'maxEdges': MAX_EDGES,
        'maxEdges2': MAX_EDGES2, 'vertexDegree': VERTEX_DEGREE,
        'xCell': xC[:, 0].copy(), 'yCell': xC[:, 1].copy(), 'zCell': xC[:, 2].copy(),
        'latCell': latC, 'lonCell': lonC,
        'xEdge': xE[:, 0].copy(), 'yEdge': xE[:, 1].copy(), 'zEdge': xE[:, 2].copy(),
        'latEdge': latE, 'lonEdge': lonE,
        'xVertex': xV[:, 0].copy(), 'yVertex': xV[:, 1].copy(), 'zVertex': xV[:, 2].copy(),
        'latVertex': latV, 'lonVertex': lonV,
        'cellsOnEdge': one(np.stack([c1, c2], 1)),
        'verticesOnEdge': one(np.stack([v1, v2], 1)),
        'nEdgesOnCell': nEoC.astype(np.int32),
        'nEdgesOnEdge': nEoE.astype(np.int32),
        'edgesOnCell': one(eoc), 'verticesOnCell': one(voc), 'cellsOnCell': one(coc),
        'edgesOnEdge': one(eoe), 'weightsOnEdge': woe,
        'cellsOnVertex': one(cov), 'edgesOnVertex': one(eov),
        'kiteAreasOnVertex': kites, 'areaTriangle': areaTriangle, 'areaCell': areaCell,
        'dcEdge': dc, 'dvEdge': dv, 'angleEdge': angleEdge,
        'meshDensity': np.ones(N),
    }
