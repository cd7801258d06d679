// Host-only check of the fused-stage tile builder (compiled by tests/test_tiles.py with g++ from
// the package's own set-up sources): builds the internal mesh from reference-layout arrays, then
// the tangent-linear and adjoint tiles, and reports what the test checks.
#include <cstring>
#include <vector>

#include "mpsw_setup.h"
#include "mpsw_tiles.h"

using namespace mpsw;

// out[0] tiles, out[1] owned cells summed over tiles, out[2] owned edges summed, out[3] cells
// owned twice or never, out[4] edges owned twice or never, out[5] shared-memory bytes (M = 4,
// the tiles' budget), out[6] (M = 8); returns 0 or 1 with the builder's message in err.
extern "C" int tile_check(int nC, int nE, int nV, int maxEdges, int maxEdges2, const int *coe, const int *voe,
                          const int *eoe, const int *neoe, const int *eoc, const int *neoc, const int *cov,
                          const int *eov, const double *w, const double *kites, const double *dc,
                          const double *dv, const double *ac, const double *at, const double *xyz[9], int K,
                          int budget_kb, int adjoint, long long *out, char *err, int errlen) {
  RefMesh r;
  r.nC = nC; r.nE = nE; r.nV = nV; r.maxEdges = maxEdges; r.maxEdges2 = maxEdges2; r.vd = 3;
  r.cellsOnEdge = coe; r.verticesOnEdge = voe; r.edgesOnEdge = eoe; r.nEdgesOnEdge = neoe;
  r.edgesOnCell = eoc; r.nEdgesOnCell = neoc; r.cellsOnVertex = cov; r.edgesOnVertex = eov;
  r.weightsOnEdge = w; r.kiteAreasOnVertex = kites; r.dcEdge = dc; r.dvEdge = dv; r.areaCell = ac;
  r.areaTriangle = at;
  r.xCell = xyz[0]; r.yCell = xyz[1]; r.zCell = xyz[2]; r.xEdge = xyz[3]; r.yEdge = xyz[4]; r.zEdge = xyz[5];
  r.xVertex = xyz[6]; r.yVertex = xyz[7]; r.zVertex = xyz[8];
  std::vector<double> fz(nV, 0.0);
  r.fVertex = fz.data();
  RefGeometry g;
  g.coeffs_reconstruct.assign((size_t)3 * maxEdges * nC, 0.0);
  BuiltMesh bm;
  std::string e = build_mesh(r, g, 1, &bm);
  TileSetHost t;
  if (e.empty()) e = build_tiles(bm, (size_t)budget_kb << 10, K, 4, adjoint != 0, &t);
  if (!e.empty()) {
    std::strncpy(err, e.c_str(), errlen - 1);
    err[errlen - 1] = 0;
    return 1;
  }
  std::vector<int> oc(nC, 0), oe(nE, 0);
  long long sc = 0, se = 0;
  for (int i = 0; i < t.ntiles; i++) {
    const int *cnt = &t.cnt[(size_t)i * kTileCounts];
    const int *off = &t.off[(size_t)i * 3];
    for (int k = 0; k < cnt[C_OWN]; k++) oc[t.gc[off[1] + k]]++;
    for (int k = 0; k < cnt[E_OWN]; k++) oe[t.ge[off[0] + k]]++;
    sc += cnt[C_OWN];
    se += cnt[E_OWN];
  }
  long long bc = 0, be = 0;
  for (int x : oc) bc += x != 1;
  for (int x : oe) be += x != 1;
  out[0] = t.ntiles; out[1] = sc; out[2] = se; out[3] = bc; out[4] = be;
  out[5] = (long long)t.smem[0]; out[6] = (long long)t.smem[1];
  return 0;
}
