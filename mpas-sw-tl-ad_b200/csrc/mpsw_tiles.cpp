// Host builder of the halo tiles of the fused member-stage kernels (see mpsw_tiles.h).
#include "mpsw_tiles.h"

#include <algorithm>
#include <sstream>

namespace mpsw {
namespace {

constexpr int kCellSlots = 6, kEoeSlots = 10;

// One local index space of a tile: entities join in layers; each layer is sorted by internal
// index before it is numbered, so the gathers of a layer walk memory in order.
struct Space {
  std::vector<int> &stamp, &loc;
  int tile;
  std::vector<int> list, pending;
  Space(std::vector<int> &s, std::vector<int> &l, int t) : stamp(s), loc(l), tile(t) {}
  void add(int g) {
    if (stamp[g] != tile) {
      stamp[g] = tile;
      loc[g] = -1;
      pending.push_back(g);
    }
  }
  int close() {
    std::sort(pending.begin(), pending.end());
    for (int g : pending) {
      loc[g] = (int)list.size();
      list.push_back(g);
    }
    pending.clear();
    return (int)list.size();
  }
  int local(int g) const { return stamp[g] == tile && loc[g] >= 0 ? loc[g] : -1; }
};

struct Builder {
  const BuiltMesh &m;
  std::vector<int> se, le, sc, lc, sv, lv;
  explicit Builder(const BuiltMesh &mesh)
      : m(mesh), se(mesh.nE, -1), le(mesh.nE, -1), sc(mesh.nC, -1), lc(mesh.nC, -1), sv(mesh.nV, -1),
        lv(mesh.nV, -1) {}
  int cn(int c) const { return m.c_n[c]; }
  int ces(int c, int k) const { return m.c_es[(size_t)k * m.nC + c]; }
  int cvs(int c, int k) const { return m.c_vs[(size_t)k * m.nC + c]; }
  int cnb(int c, int k) const {
    const int e = ces(c, k);
    return m.e_c1[e] == c ? m.e_c2[e] : m.e_c1[e];
  }
  int eoe(int e, int j) const { return m.e_eoe[(size_t)j * m.nE + e]; }
  int ves(int v, int k) const { return m.v_es[(size_t)k * m.nV + v]; }
  int vc(int v, int k) const { return m.v_c[(size_t)k * m.nV + v]; }
};

std::string fail(int tile, const char *what) {
  std::ostringstream s;
  s << "tile " << tile << ": " << what;
  return s.str();
}

}  // namespace

std::string build_tiles(const BuiltMesh &m, int K, bool adjoint, TileSetHost *o) {
  if (K < 1) return "tile size must be positive";
  for (int c = 0; c < m.nC; c++)
    if (m.c_n[c] > kCellSlots) return "fused tiles need at most 6 edges per cell";
  for (int e = 0; e < m.nE; e++)
    if (m.e_n[e] > kEoeSlots) return "fused tiles need at most 10 edgesOnEdge";
  Builder b(m);
  const int nC = m.nC, nE = m.nE;
  const int ntiles = (nC + K - 1) / K;
  // owned edges: those whose lower-numbered cell the tile owns (counting sort by tile)
  std::vector<int> first(ntiles + 1, 0), owned(nE);
  for (int e = 0; e < nE; e++) first[std::min(m.e_c1[e], m.e_c2[e]) / K + 1]++;
  for (int t = 0; t < ntiles; t++) first[t + 1] += first[t];
  {
    std::vector<int> fill(first.begin(), first.end() - 1);
    for (int e = 0; e < nE; e++) owned[fill[std::min(m.e_c1[e], m.e_c2[e]) / K]++] = e;
  }
  *o = TileSetHost();
  o->K = K;
  o->ntiles = ntiles;
  o->cnt.assign((size_t)ntiles * kTileCounts, 0);
  o->off.assign((size_t)ntiles * 3, 0);
  for (int t = 0; t < ntiles; t++) {
    Space E(b.se, b.le, t), C(b.sc, b.lc, t), V(b.sv, b.lv, t);
    int *cnt = &o->cnt[(size_t)t * kTileCounts];
    const int c0 = t * K, c1 = std::min(nC, c0 + K);
    for (int c = c0; c < c1; c++) C.add(c);
    cnt[C_OWN] = C.close();
    for (int i = first[t]; i < first[t + 1]; i++) E.add(owned[i]);
    cnt[E_OWN] = E.close();
    const std::vector<int> OE(E.list), OC(C.list);
    for (int e : OE) {
      C.add(m.e_c1[e]);
      C.add(m.e_c2[e]);
    }
    cnt[C_KE] = C.close();
    if (!adjoint) {
      for (int e : OE)
        for (int j = 0; j < m.e_n[e]; j++) E.add(b.eoe(e, j));
      cnt[E_MID] = E.close();
      for (int e : E.list) {
        C.add(m.e_c1[e]);
        C.add(m.e_c2[e]);
      }
      cnt[C_MID] = C.close();
      for (int c : C.list)
        for (int k = 0; k < b.cn(c); k++) V.add(b.cvs(c, k));
      for (int i = 0; i < cnt[E_MID]; i++) {
        V.add(m.e_v1[E.list[i]]);
        V.add(m.e_v2[E.list[i]]);
      }
      cnt[V_ALL] = V.close();
      for (int i = 0; i < cnt[E_MID]; i++)
        for (int j = 0; j < m.e_n[E.list[i]]; j++) E.add(b.eoe(E.list[i], j));
      for (int v : V.list)
        for (int k = 0; k < VDEG; k++) E.add(b.ves(v, k));
      for (int i = 0; i < cnt[C_KE]; i++)
        for (int k = 0; k < b.cn(C.list[i]); k++) E.add(b.ces(C.list[i], k));
      cnt[E_ALL] = E.close();
      for (int v : V.list)
        for (int k = 0; k < VDEG; k++) C.add(b.vc(v, k));
      for (int c : OC)
        for (int k = 0; k < b.cn(c); k++) C.add(b.cnb(c, k));
      cnt[C_ALL] = C.close();
    } else {
      for (int e : OE) {
        V.add(m.e_v1[e]);
        V.add(m.e_v2[e]);
      }
      for (int c : OC)
        for (int k = 0; k < b.cn(c); k++) V.add(b.cvs(c, k));
      cnt[V_ALL] = V.close();
      for (int v : V.list)
        for (int k = 0; k < VDEG; k++) C.add(b.vc(v, k));
      cnt[C_MID] = C.close();
      for (int e : OE)
        for (int j = 0; j < m.e_n[e]; j++) E.add(b.eoe(e, j));
      for (int c : C.list)
        for (int k = 0; k < b.cn(c); k++) E.add(b.ces(c, k));
      for (int v : V.list)
        for (int k = 0; k < VDEG; k++) E.add(b.ves(v, k));
      cnt[E_MID] = E.close();
      for (int i = 0; i < cnt[E_MID]; i++)
        for (int j = 0; j < m.e_n[E.list[i]]; j++) E.add(b.eoe(E.list[i], j));
      cnt[E_ALL] = E.close();
      for (int i = 0; i < cnt[E_MID]; i++) {
        C.add(m.e_c1[E.list[i]]);
        C.add(m.e_c2[E.list[i]]);
      }
      cnt[C_ALL] = C.close();
    }
    if (E.list.size() >= kNoLocal || C.list.size() >= kNoLocal || V.list.size() >= kNoLocal)
      return fail(t, "a local index space exceeds 65534 entities (use a smaller tile)");
    // records
    int *off = &o->off[(size_t)t * 3];
    off[0] = (int)o->ge.size();
    off[1] = (int)o->gc.size();
    off[2] = (int)o->gv.size();
    auto L = [](int x) { return x < 0 ? kNoLocal : (uint16_t)x; };
    for (int e : E.list) {
      o->ge.push_back(e);
      uint16_t r[kERec] = {};
      r[0] = L(C.local(m.e_c1[e]));
      r[1] = L(C.local(m.e_c2[e]));
      r[2] = L(V.local(m.e_v1[e]));
      r[3] = L(V.local(m.e_v2[e]));
      // slots past nEdgesOnEdge point at local edge 0: their weights are zero
      for (int j = 0; j < kEoeSlots; j++) r[4 + j] = j < m.e_n[e] ? L(E.local(b.eoe(e, j))) : 0;
      o->erec.insert(o->erec.end(), r, r + kERec);
    }
    for (int c : C.list) {
      o->gc.push_back(c);
      uint16_t r[kCRec] = {};
      for (int k = 0; k < kCellSlots; k++) {  // padded slots: local index 0, zero coefficients
        const bool in = k < b.cn(c);
        r[k] = in ? L(E.local(b.ces(c, k))) : 0;
        r[6 + k] = in ? L(V.local(b.cvs(c, k))) : 0;
        r[12 + k] = in ? L(C.local(b.cnb(c, k))) : 0;
      }
      o->crec.insert(o->crec.end(), r, r + kCRec);
    }
    for (int v : V.list) {
      o->gv.push_back(v);
      uint16_t r[kVRec] = {};
      for (int k = 0; k < VDEG; k++) {
        r[k] = L(E.local(b.ves(v, k)));
        r[3 + k] = L(C.local(b.vc(v, k)));
      }
      o->vrec.insert(o->vrec.end(), r, r + kVRec);
    }
    // every neighbour a phase reads must be in the tile, in the layer the phase needs
    const uint16_t *er = &o->erec[(size_t)off[0] * kERec];
    const uint16_t *cr = &o->crec[(size_t)off[1] * kCRec];
    const uint16_t *vr = &o->vrec[(size_t)off[2] * kVRec];
    auto below = [](uint16_t x, int n) { return x != kNoLocal && (int)x < n; };
    auto cells_ok = [&](int lo, int hi, int edges_below, bool verts, bool nbs) {
      for (int i = lo; i < hi; i++)
        for (int k = 0; k < b.cn(C.list[i]); k++) {
          if (!below(cr[(size_t)i * kCRec + k], edges_below)) return false;
          if (verts && cr[(size_t)i * kCRec + 6 + k] == kNoLocal) return false;
          if (nbs && cr[(size_t)i * kCRec + 12 + k] == kNoLocal) return false;
        }
      return true;
    };
    auto edges_ok = [&](int lo, int hi, int eoe_below, int cells_below, bool verts) {
      for (int i = lo; i < hi; i++) {
        const uint16_t *r = er + (size_t)i * kERec;
        if (!below(r[0], cells_below) || !below(r[1], cells_below)) return false;
        if (verts && (r[2] == kNoLocal || r[3] == kNoLocal)) return false;
        for (int j = 0; j < m.e_n[E.list[i]]; j++)
          if (!below(r[4 + j], eoe_below)) return false;
      }
      return true;
    };
    auto verts_ok = [&](int edges_below, int cells_below) {
      for (int i = 0; i < cnt[V_ALL]; i++)
        for (int k = 0; k < VDEG; k++)
          if (!below(vr[(size_t)i * kVRec + k], edges_below) || !below(vr[(size_t)i * kVRec + 3 + k], cells_below))
            return false;
      return true;
    };
    bool ok;
    if (!adjoint) {
      ok = verts_ok(cnt[E_ALL], cnt[C_ALL]) &&                            // pv_vertex'
           cells_ok(0, cnt[C_KE], cnt[E_ALL], false, false) &&            // ke'
           cells_ok(0, cnt[C_OWN], cnt[E_ALL], false, true) &&            // thickness tendency
           cells_ok(0, cnt[C_MID], cnt[E_ALL], true, false) &&            // pv_cell'
           edges_ok(0, cnt[E_MID], cnt[E_ALL], cnt[C_MID], true) &&       // pv_edge', fluxes
           edges_ok(0, cnt[E_OWN], cnt[E_MID], cnt[C_KE], true);          // normal-velocity tendency
    } else {
      ok = edges_ok(0, cnt[E_MID], cnt[E_ALL], cnt[C_ALL], false) &&      // edge adjoints
           cells_ok(0, cnt[C_MID], cnt[E_MID], false, false) &&           // pv_cell / ke adjoints
           verts_ok(cnt[E_MID], cnt[C_MID]) &&                            // vertex adjoints
           edges_ok(0, cnt[E_OWN], cnt[E_MID], cnt[C_KE], true) &&        // owned edges
           cells_ok(0, cnt[C_OWN], cnt[E_MID], true, false);              // owned cells
    }
    if (!ok) return fail(t, "a phase of the fused stage would read outside its tile");
    for (int k = 0; k < kTileCounts; k++) o->max_cnt[k] = std::max(o->max_cnt[k], cnt[k]);
    // shared memory of the stage's block: member rows (M floats each) and base values (floats),
    // in the order the kernels lay them out
    const size_t rows = adjoint ? (size_t)cnt[E_ALL] + cnt[C_ALL] + 3 * (size_t)cnt[E_MID] + cnt[E_OWN] +
                                      cnt[C_MID] + cnt[C_KE] + 2 * (size_t)cnt[V_ALL]
                                : (size_t)cnt[E_ALL] + cnt[C_ALL] + cnt[V_ALL] + cnt[C_MID] + cnt[C_KE] +
                                      2 * (size_t)cnt[E_MID] + cnt[E_OWN];
    const size_t floats = adjoint ? 3 * (size_t)cnt[E_ALL] + cnt[E_MID] : 2 * (size_t)cnt[E_ALL];
    for (int i = 0; i < 2; i++) o->smem[i] = std::max(o->smem[i], (rows * (4 << i) + floats) * sizeof(float));
  }
  return "";
}

void build_fused_coefficients(const BuiltMesh &m, FusedCoefHost *o) {
  const int nC = m.nC, nE = m.nE, nV = m.nV;
  *o = FusedCoefHost();
  for (auto *a : {&o->v_cc, &o->v_kr, &o->v_kc, &o->v_sr}) a->assign((size_t)VDEG * nV, 0.f);
  for (int k = 0; k < VDEG; k++)
    for (int v = 0; v < nV; v++) {
      const size_t i = (size_t)k * nV + v;
      const int e = m.v_es[i], c = m.v_c[i];
      o->v_cc[i] = (float)((double)m.v_esg[i] * m.e_dc[e] / m.v_area[v]);
      o->v_kr[i] = (float)(m.v_k[i] / m.v_area[v]);
      o->v_kc[i] = (float)(m.v_k[i] / m.c_area[c]);
      o->v_sr[i] = (float)((double)m.v_esg[i] / m.e_dv[e]);
    }
  for (auto *a : {&o->c_kr, &o->c_kec, &o->c_sdv, &o->c_src, &o->c_hk}) a->assign((size_t)kCellSlots * nC, 0.f);
  for (int k = 0; k < kCellSlots; k++)
    for (int c = 0; c < nC; c++) {
      if (k >= m.c_n[c]) continue;  // padded slots keep zero coefficients
      const size_t i = (size_t)k * nC + c;
      const int e = m.c_es[i];
      const double ra = 1.0 / m.c_area[c], sg = (double)m.c_esg[i];
      o->c_kr[i] = (float)(m.c_vk[i] * ra);
      o->c_kec[i] = (float)(0.25 * m.e_dc[e] * m.e_dv[e] * ra);
      o->c_sdv[i] = (float)(sg * m.e_dv[e] * ra);
      o->c_src[i] = (float)(sg / m.e_dc[e]);
      o->c_hk[i] = 0.5f;
    }
  o->e_rdv.assign(nE, 0.f);
  o->e_rdc.assign(nE, 0.f);
  for (int e = 0; e < nE; e++) {
    o->e_rdv[e] = (float)(1.0 / m.e_dv[e]);
    o->e_rdc[e] = (float)(1.0 / m.e_dc[e]);
  }
}

}  // namespace mpsw
