"""TRiSK mesh generator invariants (mpsw.mesh): counts, areas, orientation conventions the
reference stencils rely on (src/mpas_sw_dyncore.f90:208-242), and the TRiSK identities."""
import numpy as np
import pytest

from helpers import mesh


@pytest.mark.parametrize('level', [0, 1, 2, 3, 4])
def test_counts_and_areas(level):
    m = mesh(level)
    assert m['nCells'] == 10 * 4 ** level + 2
    assert m['nEdges'] == 30 * 4 ** level
    assert m['nVertices'] == 20 * 4 ** level
    assert abs(m['areaCell'].sum() - 4 * np.pi) < 1e-12
    assert abs(m['areaTriangle'].sum() - 4 * np.pi) < 1e-12
    assert m['kiteAreasOnVertex'].min() > 0
    assert np.all((m['nEdgesOnCell'] == 5) | (m['nEdgesOnCell'] == 6))
    assert (m['nEdgesOnCell'] == 5).sum() == 12
    assert np.array_equal(m['nEdgesOnEdge'], m['nEdgesOnCell'][m['cellsOnEdge'][:, 0] - 1]
                          + m['nEdgesOnCell'][m['cellsOnEdge'][:, 1] - 1] - 2)


def test_orientation_conventions():
    m = mesh(3)
    xc = np.stack([m['xCell'], m['yCell'], m['zCell']], 1)
    xv = np.stack([m['xVertex'], m['yVertex'], m['zVertex']], 1)
    xe = np.stack([m['xEdge'], m['yEdge'], m['zEdge']], 1)
    c1, c2 = m['cellsOnEdge'][:, 0] - 1, m['cellsOnEdge'][:, 1] - 1
    v1, v2 = m['verticesOnEdge'][:, 0] - 1, m['verticesOnEdge'][:, 1] - 1
    n = xc[c2] - xc[c1]
    t = np.cross(xe, n)
    # t = k x n points from verticesOnEdge(1) to verticesOnEdge(2)
    assert np.all(np.einsum('ij,ij->i', t, xv[v2] - xv[v1]) > 0)
    # edgesOnVertex(i) joins cellsOnVertex(i) and cellsOnVertex(i+1)
    cov, eov = m['cellsOnVertex'] - 1, m['edgesOnVertex'] - 1
    for i in range(3):
        a, b = cov[:, i], cov[:, (i + 1) % 3]
        e = eov[:, i]
        assert np.all(((c1[e] == a) & (c2[e] == b)) | ((c1[e] == b) & (c2[e] == a)))


def test_trisk_identities():
    """weightsOnEdge: energy-neutral (antisymmetric after dc*dv scaling) and the
    steady-geostrophic-mode identity curl(v) = -sum_i kite_i div_i(u) on every vertex."""
    m = mesh(3)
    E, N, V = m['nEdges'], m['nCells'], m['nVertices']
    dc, dv = m['dcEdge'], m['dvEdge']
    eoe, w, ne = m['edgesOnEdge'] - 1, m['weightsOnEdge'], m['nEdgesOnEdge']
    wmax = np.abs(w).max()
    for e in range(E):
        for j in range(ne[e]):
            ep = eoe[e, j]
            jj = np.where(eoe[ep, :ne[ep]] == e)[0]
            assert len(jj) == 1
            assert abs(dc[e] * dv[e] * w[e, j] + dc[ep] * dv[ep] * w[ep, jj[0]]) < 1e-13 * wmax
    rng = np.random.default_rng(0)
    u = rng.standard_normal(E)
    v = np.zeros(E)
    for j in range(12):
        msk = j < ne
        v[msk] += w[msk, j] * u[eoe[msk, j]]
    c1, c2 = m['cellsOnEdge'][:, 0] - 1, m['cellsOnEdge'][:, 1] - 1
    v1, v2 = m['verticesOnEdge'][:, 0] - 1, m['verticesOnEdge'][:, 1] - 1
    circ = np.zeros(V)
    np.add.at(circ, v1, -dc * v)
    np.add.at(circ, v2, dc * v)
    div = np.zeros(N)
    np.add.at(div, c1, u * dv)
    np.add.at(div, c2, -u * dv)
    div /= m['areaCell']
    rem = (m['kiteAreasOnVertex'] * div[m['cellsOnVertex'] - 1]).sum(1)
    assert np.abs(circ + rem).max() < 1e-13 * np.abs(rem).max()


def test_tangential_reconstruction_converges():
    """v = sum w u approximates the tangential component of a solid-body rotation."""
    errs = []
    for level in (3, 4, 5):
        m = mesh(level)
        xe = np.stack([m['xEdge'], m['yEdge'], m['zEdge']], 1)
        xc = np.stack([m['xCell'], m['yCell'], m['zCell']], 1)
        c1, c2 = m['cellsOnEdge'][:, 0] - 1, m['cellsOnEdge'][:, 1] - 1
        n = xc[c2] - xc[c1]
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        vel = np.cross(np.array([0.3, -0.5, 0.8])[None, :], xe)
        u = np.einsum('ij,ij->i', vel, n)
        vex = np.einsum('ij,ij->i', vel, np.cross(xe, n))
        v = np.zeros(m['nEdges'])
        for j in range(12):
            msk = j < m['nEdgesOnEdge']
            v[msk] += m['weightsOnEdge'][msk, j] * u[m['edgesOnEdge'][msk, j] - 1]
        errs.append(np.sqrt(np.mean((v - vex) ** 2)) / np.sqrt(np.mean(vex ** 2)))
    assert errs[-1] < 0.05 and errs[-1] < errs[0]


def test_deterministic():
    a, b = mesh(2), __import__('mpsw.mesh', fromlist=['x']).icosahedral_mesh(2)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
