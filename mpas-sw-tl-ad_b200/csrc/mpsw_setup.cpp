// Host set-up of the engine; see mpsw_setup.h.  Compiled without FMA contraction so that the
// geometry it derives is bit-identical to what the reference's sw_mpas_init_block computes.
#include "mpsw_setup.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <sstream>

#include "mpsw_internal.h"

namespace mpsw {

namespace {

// column-major, 1-based accessors for the reference layout
inline int ri(const int *p, int ld, int i, int j) { return p[(size_t)(i - 1) + (size_t)ld * (j - 1)]; }
inline double rd(const double *p, int ld, int i, int j) { return p[(size_t)(i - 1) + (size_t)ld * (j - 1)]; }

std::string fmt(const char *what, long long a, long long b) {
  std::ostringstream s;
  s << what << " (" << a << ", " << b << ")";
  return s.str();
}

// --- 3-D Hilbert key: J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707 (2004):
// transform axes to the transposed Hilbert index, then interleave its bits.
uint64_t hilbert3(uint32_t x0, uint32_t x1, uint32_t x2, int bits) {
  uint32_t X[3] = {x0, x1, x2};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
    for (int i = 0; i < 3; i++) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; i++) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; i++) X[i] ^= t;
  uint64_t key = 0;
  for (int b = bits - 1; b >= 0; b--)
    for (int i = 0; i < 3; i++) key = (key << 1) | ((X[i] >> b) & 1u);
  return key;
}

// reference index -> internal index, ordering points along the Hilbert curve of their
// direction (positions are normalised, so unit and Earth-radius meshes order identically)
std::vector<int> hilbert_perm(int n, const double *x, const double *y, const double *z, int sfc) {
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  if (sfc && x && y && z) {
    const int bits = 20;
    const double scale = (double)((1u << bits) - 1);
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; i++) {
      double r = std::sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
      if (!(r > 0)) r = 1.0;
      const uint32_t q0 = (uint32_t)((x[i] / r + 1.0) * 0.5 * scale);
      const uint32_t q1 = (uint32_t)((y[i] / r + 1.0) * 0.5 * scale);
      const uint32_t q2 = (uint32_t)((z[i] / r + 1.0) * 0.5 * scale);
      key[i] = hilbert3(q0, q1, q2, bits);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
  }
  std::vector<int> perm(n);
  for (int k = 0; k < n; k++) perm[order[k]] = k;
  return perm;
}

// --- geometry (src/mpas_sw_operators.f90) ---------------------------------------------------
void unit_vec(double *x) {
  const double mag = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  x[0] = x[0] / mag;
  x[1] = x[1] / mag;
  x[2] = x[2] / mag;
}

// Partial-pivoting Gaussian elimination with row scaling (the reference's elgs/mpas_legs,
// T. Pang 2001), column-major n x n matrix a, pivot order in idx; solves in place for b.
void pivot_solve(std::vector<double> &a, int n, std::vector<double> &b, std::vector<double> &x,
                 std::vector<int> &idx) {
  auto A = [&](int i, int j) -> double & { return a[(size_t)i + (size_t)n * j]; };
  std::vector<double> scale(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  for (int i = 0; i < n; i++) {
    double c1 = 0.0;
    for (int j = 0; j < n; j++) c1 = std::fmax(c1, std::fabs(A(i, j)));
    scale[i] = c1;
  }
  int k = 0;
  for (int j = 0; j < n - 1; j++) {
    double best = 0.0;
    for (int i = j; i < n; i++) {
      const double p = std::fabs(A(idx[i], j)) / scale[idx[i]];
      if (p > best) {
        best = p;
        k = i;
      }
    }
    std::swap(idx[j], idx[k]);
    for (int i = j + 1; i < n; i++) {
      const double pj = A(idx[i], j) / A(idx[j], j);
      A(idx[i], j) = pj;
      for (int kk = j + 1; kk < n; kk++) A(idx[i], kk) = A(idx[i], kk) - pj * A(idx[j], kk);
    }
  }
  for (int i = 0; i < n - 1; i++)
    for (int j = i + 1; j < n; j++) b[idx[j]] = b[idx[j]] - A(idx[j], i) * b[idx[i]];
  x[n - 1] = b[idx[n - 1]] / A(idx[n - 1], n - 1);
  for (int i = n - 2; i >= 0; i--) {
    x[i] = b[idx[i]];
    for (int j = i + 1; j < n; j++) x[i] = x[i] - A(idx[i], j) * x[j];
    x[i] = x[i] / A(idx[i], i);
  }
}

// Coefficients of the RBF reconstruction of a cell-centred vector from edge-normal components
// (inverse multiquadric kernel, constant vector in the tangent plane; src/mpas_sw_operators.f90:413-527).
void rbf_cell(int n, const double *loc /*n x 3 row-major*/, const double *nrm /*n x 3*/,
              const double *centre, double alpha, const double plane[2][3], double *coef /*n x 3*/) {
  const int ms = n + 2;
  std::vector<double> ps(2 * n), pu(2 * n);
  double pd[2];
  for (int i = 0; i < n; i++)
    for (int d = 0; d < 2; d++) {
      double s = 0.0, t = 0.0;
      for (int k = 0; k < 3; k++) {
        s = s + loc[3 * i + k] * plane[d][k];
        t = t + nrm[3 * i + k] * plane[d][k];
      }
      ps[2 * i + d] = s;
      pu[2 * i + d] = t;
    }
  for (int d = 0; d < 2; d++) {
    double s = 0.0;
    for (int k = 0; k < 3; k++) s = s + centre[k] * plane[d][k];
    pd[d] = s;
  }
  std::vector<double> mat((size_t)ms * ms, 0.0), rhs((size_t)2 * ms, 0.0);
  auto M = [&](int i, int j) -> double & { return mat[(size_t)i + (size_t)ms * j]; };
  const double a2 = alpha * alpha;
  for (int j = 0; j < n; j++)
    for (int i = j; i < n; i++) {
      double rs = 0.0, dot = 0.0;
      for (int d = 0; d < 2; d++) {
        const double df = ps[2 * i + d] - ps[2 * j + d];
        rs = rs + df * df;
        dot = dot + pu[2 * i + d] * pu[2 * j + d];
      }
      rs = rs / a2;
      M(i, j) = (1.0 / std::sqrt(1.0 + rs)) * dot;
      M(j, i) = M(i, j);
    }
  for (int j = 0; j < n; j++) {
    double rs = 0.0;
    for (int d = 0; d < 2; d++) {
      const double df = pd[d] - ps[2 * j + d];
      rs = rs + df * df;
    }
    rs = rs / a2;
    const double rb = 1.0 / std::sqrt(1.0 + rs);
    for (int d = 0; d < 2; d++) rhs[j + (size_t)ms * d] = rb * pu[2 * j + d];
  }
  for (int i = 0; i < n; i++)
    for (int d = 0; d < 2; d++) {
      M(i, n + d) = pu[2 * i + d];
      M(n + d, i) = M(i, n + d);
    }
  rhs[n] = 1.0;
  rhs[(n + 1) + (size_t)ms] = 1.0;
  std::vector<double> mcopy = mat, b0(rhs.begin(), rhs.begin() + ms), b1(rhs.begin() + ms, rhs.end());
  std::vector<double> x0(ms), x1(ms);
  std::vector<int> idx(ms);
  pivot_solve(mat, ms, b0, x0, idx);
  pivot_solve(mcopy, ms, b1, x1, idx);
  for (int k = 0; k < 3; k++)
    for (int p = 0; p < n; p++) coef[3 * p + k] = plane[0][k] * x0[p] + plane[1][k] * x1[p];
}

}  // namespace

std::string validate_mesh(const RefMesh &m) {
  if (m.nC <= 0 || m.nE <= 0 || m.nV <= 0) return "mesh dimensions must be positive";
  if (m.maxEdges < 3 || m.maxEdges > MAXE) return fmt("maxEdges out of supported range [3, 10]", m.maxEdges, MAXE);
  if (m.maxEdges2 < 1 || m.maxEdges2 > MAXE2) return fmt("maxEdges2 out of supported range [1, 20]", m.maxEdges2, MAXE2);
  if (m.vd != VDEG) return fmt("vertexDegree must be 3", m.vd, VDEG);
  const void *req[] = {m.cellsOnEdge, m.verticesOnEdge, m.edgesOnEdge, m.nEdgesOnEdge, m.edgesOnCell,
                       m.nEdgesOnCell, m.cellsOnVertex, m.edgesOnVertex, m.weightsOnEdge,
                       m.kiteAreasOnVertex, m.dcEdge, m.dvEdge, m.areaCell, m.areaTriangle};
  for (const void *p : req)
    if (!p) return "a required mesh array has not been set";
  for (int e = 1; e <= m.nE; e++) {
    for (int i = 1; i <= 2; i++) {
      const int c = ri(m.cellsOnEdge, 2, i, e), v = ri(m.verticesOnEdge, 2, i, e);
      if (c < 1 || c > m.nC) return fmt("cellsOnEdge out of range at edge", e, c);
      if (v < 1 || v > m.nV) return fmt("verticesOnEdge out of range at edge", e, v);
    }
    if (ri(m.cellsOnEdge, 2, 1, e) == ri(m.cellsOnEdge, 2, 2, e)) return fmt("edge joins a cell to itself", e, 0);
    const int n = m.nEdgesOnEdge[e - 1];
    if (n < 0 || n > m.maxEdges2) return fmt("nEdgesOnEdge out of range at edge", e, n);
    for (int j = 1; j <= n; j++) {
      const int x = ri(m.edgesOnEdge, m.maxEdges2, j, e);
      if (x < 1 || x > m.nE) return fmt("edgesOnEdge out of range at edge", e, x);
    }
    if (!(m.dcEdge[e - 1] != 0.0) || !(m.dvEdge[e - 1] != 0.0)) return fmt("zero dcEdge/dvEdge at edge", e, 0);
  }
  for (int c = 1; c <= m.nC; c++) {
    const int n = m.nEdgesOnCell[c - 1];
    if (n < 3 || n > m.maxEdges) return fmt("nEdgesOnCell out of range at cell", c, n);
    for (int i = 1; i <= n; i++) {
      const int x = ri(m.edgesOnCell, m.maxEdges, i, c);
      if (x < 1 || x > m.nE) return fmt("edgesOnCell out of range at cell", c, x);
    }
    if (!(m.areaCell[c - 1] != 0.0)) return fmt("zero areaCell at cell", c, 0);
  }
  for (int v = 1; v <= m.nV; v++) {
    for (int i = 1; i <= m.vd; i++) {
      const int c = ri(m.cellsOnVertex, m.vd, i, v), e = ri(m.edgesOnVertex, m.vd, i, v);
      if (c < 1 || c > m.nC) return fmt("cellsOnVertex out of range at vertex", v, c);
      if (e < 1 || e > m.nE) return fmt("edgesOnVertex out of range at vertex", v, e);
    }
    if (!(m.areaTriangle[v - 1] != 0.0)) return fmt("zero areaTriangle at vertex", v, 0);
  }
  return "";
}

void compute_geometry(const RefMesh &m, RefGeometry *g) {
  const int nC = m.nC, nE = m.nE, mE = m.maxEdges;
  g->meshScalingDel2.assign(nE, 1.0);
  g->meshScalingDel4.assign(nE, 1.0);
  if (m.h_ScaleWithMesh && m.meshDensity) {
    for (int e = 1; e <= nE; e++) {
      const double md = (m.meshDensity[ri(m.cellsOnEdge, 2, 1, e) - 1] +
                         m.meshDensity[ri(m.cellsOnEdge, 2, 2, e) - 1]) / 2.0;
      g->meshScalingDel2[e - 1] = 1.0 / std::pow(md, 5.0 / 12.0);
      g->meshScalingDel4[e - 1] = 1.0 / std::pow(md, 5.0 / 6.0);
    }
  }
  g->localVerticalUnitVectors.assign((size_t)3 * nC, 0.0);
  g->edgeNormalVectors.assign((size_t)3 * nE, 0.0);
  g->cellTangentPlane.assign((size_t)6 * nC, 0.0);
  g->coeffs_reconstruct.assign((size_t)3 * mE * nC, 0.0);
  if (!m.xCell || !m.xEdge) return;
  for (int c = 0; c < nC; c++) {
    double *l = &g->localVerticalUnitVectors[3 * (size_t)c];
    if (m.on_a_sphere) {
      l[0] = m.xCell[c];
      l[1] = m.yCell[c];
      l[2] = m.zCell[c];
      unit_vec(l);
    } else {
      l[0] = 0.;
      l[1] = 0.;
      l[2] = 1.;
    }
  }
  for (int e = 1; e <= nE; e++) {
    const int c1 = ri(m.cellsOnEdge, 2, 1, e) - 1, c2 = ri(m.cellsOnEdge, 2, 2, e) - 1;
    double *n = &g->edgeNormalVectors[3 * (size_t)(e - 1)];
    n[0] = m.xCell[c2] - m.xCell[c1];
    n[1] = m.yCell[c2] - m.yCell[c1];
    n[2] = m.zCell[c2] - m.zCell[c1];
    unit_vec(n);
  }
  for (int c = 1; c <= nC; c++) {
    const int e = ri(m.edgesOnCell, mE, 1, c) - 1;
    const double *r = &g->localVerticalUnitVectors[3 * (size_t)(c - 1)];
    const double *n = &g->edgeNormalVectors[3 * (size_t)e];
    const double nd = 0.0 + n[0] * r[0] + n[1] * r[1] + n[2] * r[2];
    double xh[3], yh[3];
    for (int k = 0; k < 3; k++) xh[k] = n[k] - nd * r[k];
    unit_vec(xh);
    yh[0] = r[1] * xh[2] - r[2] * xh[1];
    yh[1] = r[2] * xh[0] - r[0] * xh[2];
    yh[2] = r[0] * xh[1] - r[1] * xh[0];
    unit_vec(yh);
    for (int k = 0; k < 3; k++) {
      g->cellTangentPlane[k + 3 * (0 + 2 * (size_t)(c - 1))] = xh[k];
      g->cellTangentPlane[k + 3 * (1 + 2 * (size_t)(c - 1))] = yh[k];
    }
  }
  std::vector<double> loc, nrm, cf;
  for (int c = 1; c <= nC; c++) {
    const int n = m.nEdgesOnCell[c - 1];
    const double centre[3] = {m.xCell[c - 1], m.yCell[c - 1], m.zCell[c - 1]};
    loc.assign(3 * n, 0.0);
    nrm.assign(3 * n, 0.0);
    cf.assign(3 * n, 0.0);
    for (int i = 0; i < n; i++) {
      const int e = ri(m.edgesOnCell, mE, i + 1, c) - 1;
      loc[3 * i + 0] = m.xEdge[e];
      loc[3 * i + 1] = m.yEdge[e];
      loc[3 * i + 2] = m.zEdge[e];
      for (int k = 0; k < 3; k++) nrm[3 * i + k] = g->edgeNormalVectors[3 * (size_t)e + k];
    }
    double alpha = 0.0;
    for (int i = 0; i < n; i++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++) {
        const double d = centre[k] - loc[3 * i + k];
        s = s + d * d;
      }
      alpha = alpha + std::sqrt(s);
    }
    alpha = alpha / n;
    double plane[2][3];
    for (int k = 0; k < 3; k++) {
      plane[0][k] = g->cellTangentPlane[k + 3 * (0 + 2 * (size_t)(c - 1))];
      plane[1][k] = g->cellTangentPlane[k + 3 * (1 + 2 * (size_t)(c - 1))];
    }
    rbf_cell(n, loc.data(), nrm.data(), centre, alpha, plane, cf.data());
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++)
        g->coeffs_reconstruct[k + 3 * ((size_t)i + (size_t)mE * (c - 1))] = cf[3 * i + k];
  }
}

std::string build_mesh(const RefMesh &m, const RefGeometry &g, int sfc, BuiltMesh *o) {
  const int nC = m.nC, nE = m.nE, nV = m.nV, mE = m.maxEdges, mE2 = m.maxEdges2;
  o->nC = nC;
  o->nE = nE;
  o->nV = nV;
  o->perm_c = hilbert_perm(nC, m.xCell, m.yCell, m.zCell, sfc);
  o->perm_e = hilbert_perm(nE, m.xEdge, m.yEdge, m.zEdge, sfc);
  o->perm_v = hilbert_perm(nV, m.xVertex, m.yVertex, m.zVertex, sfc);
  const std::vector<int> &pc = o->perm_c, &pe = o->perm_e, &pv = o->perm_v;

  // transposed lists in reference scatter order
  std::vector<std::vector<std::pair<int, int>>> c_e(nC), v_e(nV);
  std::vector<std::vector<std::pair<int, double>>> c_v(nC);
  std::vector<std::vector<int>> e_v(nE);
  for (int e = 1; e <= nE; e++) {
    c_e[ri(m.cellsOnEdge, 2, 1, e) - 1].push_back({e - 1, +1});
    c_e[ri(m.cellsOnEdge, 2, 2, e) - 1].push_back({e - 1, -1});
    v_e[ri(m.verticesOnEdge, 2, 1, e) - 1].push_back({e - 1, -1});
    v_e[ri(m.verticesOnEdge, 2, 2, e) - 1].push_back({e - 1, +1});
  }
  for (int v = 1; v <= nV; v++)
    for (int i = 1; i <= VDEG; i++) {
      c_v[ri(m.cellsOnVertex, VDEG, i, v) - 1].push_back({v - 1, rd(m.kiteAreasOnVertex, VDEG, i, v)});
      e_v[ri(m.edgesOnVertex, VDEG, i, v) - 1].push_back(v - 1);
    }

  o->c_n.assign(nC, 0);
  o->c_eoc.assign((size_t)MAXE * nC, 0);
  o->c_es.assign((size_t)MAXE * nC, 0);
  o->c_vs.assign((size_t)MAXE * nC, 0);
  o->c_esg.assign((size_t)MAXE * nC, 0);
  o->c_vk.assign((size_t)MAXE * nC, 0.0);
  o->c_area.assign(nC, 0.0);
  o->c_hs.assign(nC, 0.0);
  o->c_coef.assign((size_t)3 * MAXE * nC, 0.0);
  o->c_trig.assign((size_t)4 * nC, 0.0);
  for (int c = 0; c < nC; c++) {
    const int ci = pc[c], n = m.nEdgesOnCell[c];
    if ((int)c_e[c].size() != n) return fmt("cell edge count disagrees with nEdgesOnCell at cell", c + 1, (long long)c_e[c].size());
    if ((int)c_v[c].size() != n) return fmt("cell vertex count disagrees with nEdgesOnCell at cell", c + 1, (long long)c_v[c].size());
    o->c_n[ci] = n;
    for (int i = 0; i < n; i++) {
      o->c_eoc[(size_t)i * nC + ci] = pe[ri(m.edgesOnCell, mE, i + 1, c + 1) - 1];
      o->c_es[(size_t)i * nC + ci] = pe[c_e[c][i].first];
      o->c_esg[(size_t)i * nC + ci] = (signed char)c_e[c][i].second;
      o->c_vs[(size_t)i * nC + ci] = pv[c_v[c][i].first];
      o->c_vk[(size_t)i * nC + ci] = c_v[c][i].second;
      for (int k = 0; k < 3; k++)
        o->c_coef[((size_t)k * MAXE + i) * nC + ci] = g.coeffs_reconstruct[k + 3 * ((size_t)i + (size_t)mE * c)];
    }
    o->c_area[ci] = m.areaCell[c];
    o->c_hs[ci] = m.h_s ? m.h_s[c] : 0.0;
    if (m.latCell && m.lonCell) {
      o->c_trig[ci] = std::cos(m.latCell[c]);
      o->c_trig[(size_t)nC + ci] = std::sin(m.latCell[c]);
      o->c_trig[(size_t)2 * nC + ci] = std::cos(m.lonCell[c]);
      o->c_trig[(size_t)3 * nC + ci] = std::sin(m.lonCell[c]);
    }
  }

  o->e_c1.assign(nE, 0); o->e_c2.assign(nE, 0); o->e_v1.assign(nE, 0); o->e_v2.assign(nE, 0);
  o->e_va.assign(nE, 0); o->e_vb.assign(nE, 0); o->e_slot1.assign(nE, 0); o->e_slot2.assign(nE, 0);
  o->e_n.assign(nE, 0);
  o->e_eoe.assign((size_t)MAXE2 * nE, 0);
  o->e_rev.assign((size_t)MAXE2 * nE, 0);
  o->e_w.assign((size_t)MAXE2 * nE, 0.0);
  o->e_wrev.assign((size_t)MAXE2 * nE, 0.0);
  o->e_dc.assign(nE, 0.0); o->e_dv.assign(nE, 0.0); o->e_sc2.assign(nE, 1.0); o->e_sc4.assign(nE, 1.0);
  o->e_usrc.assign(nE, 0.0);
  for (int e = 0; e < nE; e++) {
    const int ei = pe[e];
    const int c1 = ri(m.cellsOnEdge, 2, 1, e + 1) - 1, c2 = ri(m.cellsOnEdge, 2, 2, e + 1) - 1;
    o->e_c1[ei] = pc[c1];
    o->e_c2[ei] = pc[c2];
    o->e_v1[ei] = pv[ri(m.verticesOnEdge, 2, 1, e + 1) - 1];
    o->e_v2[ei] = pv[ri(m.verticesOnEdge, 2, 2, e + 1) - 1];
    if (e_v[e].size() != 2) return fmt("edge is not listed by exactly two vertices in edgesOnVertex", e + 1, (long long)e_v[e].size());
    o->e_va[ei] = pv[e_v[e][0]];
    o->e_vb[ei] = pv[e_v[e][1]];
    int s1 = -1, s2 = -1;
    for (int i = 0; i < m.nEdgesOnCell[c1]; i++)
      if (ri(m.edgesOnCell, mE, i + 1, c1 + 1) == e + 1) s1 = i;
    for (int i = 0; i < m.nEdgesOnCell[c2]; i++)
      if (ri(m.edgesOnCell, mE, i + 1, c2 + 1) == e + 1) s2 = i;
    if (s1 < 0 || s2 < 0) return fmt("edge missing from edgesOnCell of one of its cells", e + 1, s1 < 0 ? c1 + 1 : c2 + 1);
    o->e_slot1[ei] = s1;
    o->e_slot2[ei] = s2;
    const int n = m.nEdgesOnEdge[e];
    o->e_n[ei] = n;
    for (int j = 0; j < n; j++) {
      const int nb = ri(m.edgesOnEdge, mE2, j + 1, e + 1) - 1;
      int r = -1;
      for (int k = 0; k < m.nEdgesOnEdge[nb]; k++)
        if (ri(m.edgesOnEdge, mE2, k + 1, nb + 1) == e + 1) { r = k; break; }
      if (r < 0) return fmt("edgesOnEdge is not symmetric between edges", e + 1, nb + 1);
      o->e_eoe[(size_t)j * nE + ei] = pe[nb];
      o->e_rev[(size_t)j * nE + ei] = r;
      o->e_w[(size_t)j * nE + ei] = rd(m.weightsOnEdge, mE2, j + 1, e + 1);
      o->e_wrev[(size_t)j * nE + ei] = rd(m.weightsOnEdge, mE2, r + 1, nb + 1);
    }
    o->e_dc[ei] = m.dcEdge[e];
    o->e_dv[ei] = m.dvEdge[e];
    o->e_sc2[ei] = g.meshScalingDel2.empty() ? 1.0 : g.meshScalingDel2[e];
    o->e_sc4[ei] = g.meshScalingDel4.empty() ? 1.0 : g.meshScalingDel4[e];
    o->e_usrc[ei] = m.u_src ? m.u_src[e] : 0.0;
  }

  o->v_es.assign((size_t)VDEG * nV, 0);
  o->v_esg.assign((size_t)VDEG * nV, 0);
  o->v_c.assign((size_t)VDEG * nV, 0);
  o->v_e.assign((size_t)VDEG * nV, 0);
  o->v_k.assign((size_t)VDEG * nV, 0.0);
  o->v_area.assign(nV, 0.0);
  o->v_f.assign(nV, 0.0);
  for (int v = 0; v < nV; v++) {
    const int vi = pv[v];
    if (v_e[v].size() != VDEG) return fmt("vertex is not an endpoint of exactly three edges", v + 1, (long long)v_e[v].size());
    for (int k = 0; k < VDEG; k++) {
      o->v_es[(size_t)k * nV + vi] = pe[v_e[v][k].first];
      o->v_esg[(size_t)k * nV + vi] = (signed char)v_e[v][k].second;
      o->v_c[(size_t)k * nV + vi] = pc[ri(m.cellsOnVertex, VDEG, k + 1, v + 1) - 1];
      o->v_e[(size_t)k * nV + vi] = pe[ri(m.edgesOnVertex, VDEG, k + 1, v + 1) - 1];
      o->v_k[(size_t)k * nV + vi] = rd(m.kiteAreasOnVertex, VDEG, k + 1, v + 1);
    }
    o->v_area[vi] = m.areaTriangle[v];
    o->v_f[vi] = m.fVertex ? m.fVertex[v] : 0.0;
  }
  return "";
}

}  // namespace mpsw
