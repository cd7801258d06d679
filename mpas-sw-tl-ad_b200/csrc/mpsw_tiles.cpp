// Host builder of the halo tiles of the fused member-stage kernels (see mpsw_tiles.h).
#include "mpsw_tiles.h"

#include <algorithm>
#include <cstring>
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

// Every neighbour a phase of the stage reads must be in the tile, in the layer the phase needs
// (local index below that layer's count).
bool validate(const Builder &b, const BuiltMesh &m, const Space &E, const Space &C, const Space &V, const int *cnt,
              bool adjoint) {
  auto below = [](int x, int n) { return x >= 0 && x < n; };
  auto cells_ok = [&](int hi, int edges_below, bool verts, bool nbs) {
    for (int i = 0; i < hi; i++) {
      const int c = C.list[i];
      for (int k = 0; k < b.cn(c); k++) {
        if (!below(E.local(b.ces(c, k)), edges_below)) return false;
        if (verts && V.local(b.cvs(c, k)) < 0) return false;
        if (nbs && C.local(b.cnb(c, k)) < 0) return false;
      }
    }
    return true;
  };
  auto edges_ok = [&](int hi, int eoe_below, int cells_below, bool verts) {
    for (int i = 0; i < hi; i++) {
      const int e = E.list[i];
      if (!below(C.local(m.e_c1[e]), cells_below) || !below(C.local(m.e_c2[e]), cells_below)) return false;
      if (verts && (V.local(m.e_v1[e]) < 0 || V.local(m.e_v2[e]) < 0)) return false;
      for (int j = 0; j < m.e_n[e]; j++)
        if (!below(E.local(b.eoe(e, j)), eoe_below)) return false;
    }
    return true;
  };
  auto verts_ok = [&](int edges_below, int cells_below) {
    for (int v : V.list)
      for (int k = 0; k < VDEG; k++)
        if (!below(E.local(b.ves(v, k)), edges_below) || !below(C.local(b.vc(v, k)), cells_below)) return false;
    return true;
  };
  if (!adjoint)
    return verts_ok(cnt[E_ALL], cnt[C_ALL]) &&                  // pv_vertex'
           cells_ok(cnt[C_KE], cnt[E_ALL], false, false) &&     // ke'
           cells_ok(cnt[C_OWN], cnt[E_ALL], false, true) &&     // thickness tendency
           cells_ok(cnt[C_MID], cnt[E_ALL], true, false) &&     // pv_cell'
           edges_ok(cnt[E_MID], cnt[E_ALL], cnt[C_MID], true) &&  // pv_edge', fluxes
           edges_ok(cnt[E_OWN], cnt[E_MID], cnt[C_KE], true);     // normal-velocity tendency
  return edges_ok(cnt[E_MID], cnt[E_ALL], cnt[C_ALL], false) &&   // edge adjoints
         cells_ok(cnt[C_MID], cnt[E_MID], false, false) &&        // pv_cell / ke adjoints
         verts_ok(cnt[E_MID], cnt[C_MID]) &&                      // vertex adjoints
         edges_ok(cnt[E_OWN], cnt[E_MID], cnt[C_KE], true) &&     // owned edges
         cells_ok(cnt[C_OWN], cnt[E_MID], true, false);           // owned cells
}

// Append one tile's blob (BlobSection layout of blob_layout).  Local indices of neighbours
// outside the tile are kNoLocal (validate() has checked no phase reads them); slots past an
// entity's list length hold local index 0 with zero coefficients, so a phase may run all slots.
void pack_blob(const Builder &b, const BuiltMesh &m, const Space &E, const Space &C, const Space &V,
               const int *cnt, bool adjoint, std::vector<unsigned char> *blob) {
  int off[kBlobSections];
  const int size = blob_layout(cnt, adjoint, off);
  const size_t base = blob->size();
  blob->resize(base + size, 0);
  unsigned char *p = blob->data() + base;
  auto ints = [&](int sec) { return reinterpret_cast<int *>(p + off[sec]); };
  auto u16s = [&](int sec) { return reinterpret_cast<uint16_t *>(p + off[sec]); };
  auto flts = [&](int sec) { return reinterpret_cast<float *>(p + off[sec]); };
  auto L = [](int x) { return x < 0 ? kNoLocal : (uint16_t)x; };
  std::memcpy(ints(B_GE), E.list.data(), 4 * E.list.size());
  std::memcpy(ints(B_GC), C.list.data(), 4 * C.list.size());
  std::memcpy(ints(B_GV), V.list.data(), 4 * V.list.size());
  // records: vertex es[3] cs[3]; cell es[6] vs[6] nb[6]; edge c1 c2 v1 v2 eoe[10]
  for (int i = 0; i < cnt[V_ALL]; i++) {
    const int v = V.list[i];
    uint16_t *r = u16s(B_VREC) + (size_t)kVRec * i;
    for (int k = 0; k < VDEG; k++) {
      r[k] = L(E.local(b.ves(v, k)));
      r[3 + k] = L(C.local(b.vc(v, k)));
    }
  }
  for (int i = 0; i < cnt[C_MID]; i++) {
    const int c = C.list[i];
    uint16_t *r = u16s(B_CREC) + (size_t)kCRec * i;
    for (int k = 0; k < kCellSlots; k++) {
      const bool in = k < b.cn(c);
      r[k] = in ? L(E.local(b.ces(c, k))) : 0;
      r[6 + k] = in ? L(V.local(b.cvs(c, k))) : 0;
      r[12 + k] = in ? L(C.local(b.cnb(c, k))) : 0;
    }
  }
  for (int i = 0; i < cnt[E_MID]; i++) {
    const int e = E.list[i];
    uint16_t *r = u16s(B_EREC) + (size_t)kERec * i;
    r[0] = L(C.local(m.e_c1[e]));
    r[1] = L(C.local(m.e_c2[e]));
    r[2] = L(V.local(m.e_v1[e]));
    r[3] = L(V.local(m.e_v2[e]));
    for (int j = 0; j < kEoeSlots; j++) r[4 + j] = j < m.e_n[e] ? L(E.local(b.eoe(e, j))) : 0;
  }
  // coefficients, formed in FP64 and rounded once
  auto vslot = [&](int v, int k) { return (size_t)k * m.nV + v; };
  auto cslot = [&](int c, int k) { return (size_t)k * m.nC + c; };
  for (int i = 0; i < cnt[V_ALL]; i++) {
    const int v = V.list[i];
    float *q = flts(B_VCOEF) + 8 * (size_t)i;
    for (int k = 0; k < VDEG; k++) {
      const size_t s = vslot(v, k);
      const int e = m.v_es[s], c = m.v_c[s];
      if (!adjoint) {
        q[k] = (float)((double)m.v_esg[s] * m.e_dc[e] / m.v_area[v]);  // circulation -> vorticity'
        q[3 + k] = (float)(m.v_k[s] / m.v_area[v]);                       // h' -> h_vertex'
      } else {
        q[k] = (float)(m.v_k[s] / m.c_area[c]);                           // pv_cell_ad -> pv_vertex_ad
        q[3 + k] = (float)((double)m.v_esg[s] / m.e_dv[e]);               // gradPVt_ad -> pv_vertex_ad
      }
    }
    q[6] = (float)(adjoint ? 1.0 / m.v_area[v] : m.v_f[v]);
    q[7] = (float)(adjoint ? m.v_f[v] : 0.0);
  }
  for (int i = 0; i < cnt[C_MID]; i++) {
    const int c = C.list[i];
    float *q = flts(B_C1) + 8 * (size_t)i;
    for (int k = 0; k < b.cn(c); k++) {
      const size_t s = cslot(c, k);
      q[k] = adjoint ? (float)((double)m.c_esg[s] / m.e_dc[m.c_es[s]])  // gradPVn / ke / gravity adjoints
                     : (float)(m.c_vk[s] / m.c_area[c]);                // pv_vertex' -> pv_cell'
    }
    if (adjoint) {
      q[6] = (float)(1.0 / m.c_area[c]);
      q[7] = (float)m.c_area[c];
    }
  }
  if (!adjoint) {
    for (int i = 0; i < cnt[C_KE]; i++) {  // ke' coefficients 0.25 dcEdge dvEdge / areaCell
      const int c = C.list[i];
      float *q = flts(B_C2) + 8 * (size_t)i;
      for (int k = 0; k < b.cn(c); k++) {
        const int e = m.c_es[cslot(c, k)];
        q[k] = (float)(0.25 * m.e_dc[e] * m.e_dv[e] / m.c_area[c]);
      }
    }
    for (int i = 0; i < cnt[C_OWN]; i++) {  // thickness flux: sign dvEdge / areaCell
      const int c = C.list[i];
      float *q = flts(B_C3) + 8 * (size_t)i;
      for (int k = 0; k < b.cn(c); k++) {
        const size_t s = cslot(c, k);
        q[k] = (float)((double)m.c_esg[s] * m.e_dv[m.c_es[s]] / m.c_area[c]);
      }
    }
  } else {
    for (int i = 0; i < cnt[C_OWN]; i++) {  // owned cells: h_edge adjoint halves, kites
      const int c = C.list[i];
      float *q = flts(B_C2) + 16 * (size_t)i;
      for (int k = 0; k < b.cn(c); k++) {
        q[k] = 0.5f;
        q[6 + k] = (float)m.c_vk[cslot(c, k)];
      }
    }
  }
  for (int i = 0; i < cnt[E_MID]; i++) {
    const int e = E.list[i];
    float *q = flts(B_ECOEF) + (adjoint ? 24 : 12) * (size_t)i;
    for (int j = 0; j < kEoeSlots; j++) {
      q[j] = (float)m.e_w[(size_t)j * m.nE + e];  // zero past nEdgesOnEdge
      if (adjoint) q[10 + j] = (float)m.e_wrev[(size_t)j * m.nE + e];
    }
    if (!adjoint) {
      q[10] = (float)(1.0 / m.e_dv[e]);
      q[11] = (float)(1.0 / m.e_dc[e]);
    } else {
      q[20] = (float)m.e_dv[e];
      q[21] = (float)m.e_dc[e];
    }
  }
}

}  // namespace

// The local spaces of the tile that owns cells [c0, c1) and the edges whose lower-numbered cell
// is among them, layer by layer (TileLayer), into E, C, V; counts into cnt.
static void tile_spaces(const Builder &b, const BuiltMesh &m, int c0, int c1, bool adjoint, Space &E, Space &C,
                        Space &V, int *cnt) {
  for (int c = c0; c < c1; c++) C.add(c);
  cnt[C_OWN] = C.close();
  for (int c = c0; c < c1; c++)
    for (int k = 0; k < b.cn(c); k++) {
      const int e = b.ces(c, k), lo = std::min(m.e_c1[e], m.e_c2[e]);
      if (lo >= c0 && lo < c1) E.add(e);
    }
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
}

// Shared memory of a tile's block with M members per chunk: blob, base values, member rows.
static size_t tile_smem(const int *cnt, bool adjoint, int M) {
  int off[kBlobSections];
  return (size_t)blob_layout(cnt, adjoint, off) + 4 * (size_t)base_floats(cnt, adjoint) +
         (size_t)member_rows(cnt, adjoint) * M * sizeof(float);
}

std::string build_tiles(const BuiltMesh &m, size_t budget, int kmax, int M, bool adjoint, TileSetHost *o) {
  if (kmax < 1) return "tile size must be positive";
  for (int c = 0; c < m.nC; c++)
    if (m.c_n[c] > kCellSlots) return "fused tiles need at most 6 edges per cell";
  for (int e = 0; e < m.nE; e++)
    if (m.e_n[e] > kEoeSlots) return "fused tiles need at most 10 edgesOnEdge";
  Builder b(m);
  const int nC = m.nC;
  int stamp = 0;  // a fresh id for each trial build of the spaces
  int cnt[kTileCounts];
  // shared memory of the tile [c0, c1) with M members per chunk
  auto fits = [&](int c0, int c1) {
    Space E(b.se, b.le, stamp), C(b.sc, b.lc, stamp), V(b.sv, b.lv, stamp);
    stamp++;
    tile_spaces(b, m, c0, c1, adjoint, E, C, V, cnt);
    return tile_smem(cnt, adjoint, M) <= budget && E.list.size() < kNoLocal && C.list.size() < kNoLocal &&
           V.list.size() < kNoLocal;
  };
  // partition the cells into runs of the internal order: each run as long as its tile's shared
  // memory stays within the budget (and at most kmax cells), so tiles near a jump of the
  // Hilbert curve, whose halo is larger, own fewer cells
  std::vector<int> bounds{0};
  while (bounds.back() < nC) {
    const int c0 = bounds.back(), hi = std::min(nC, c0 + kmax);
    if (!fits(c0, c0 + 1)) return fail((int)bounds.size() - 1, "one cell's halo exceeds the shared-memory budget");
    int ok = c0 + 1, step = 1;
    while (ok < hi) {  // grow geometrically, then bisect
      const int t = std::min(hi, ok + step);
      if (!fits(c0, t)) {
        int lo = ok, bad = t;
        while (bad - lo > 1) {
          const int mid = (lo + bad) / 2;
          (fits(c0, mid) ? lo : bad) = mid;
        }
        ok = lo;
        break;
      }
      ok = t;
      step *= 2;
    }
    bounds.push_back(ok);
  }
  const int ntiles = (int)bounds.size() - 1;
  *o = TileSetHost();
  o->K = kmax;
  o->ntiles = ntiles;
  o->cnt.assign((size_t)ntiles * kTileCounts, 0);
  o->off.assign((size_t)ntiles * 3, 0);
  o->blob_off.assign(ntiles, 0);
  for (int t = 0; t < ntiles; t++) {
    Space E(b.se, b.le, stamp), C(b.sc, b.lc, stamp), V(b.sv, b.lv, stamp);
    stamp++;
    int *tc = &o->cnt[(size_t)t * kTileCounts];
    tile_spaces(b, m, bounds[t], bounds[t + 1], adjoint, E, C, V, tc);
    if (!validate(b, m, E, C, V, tc, adjoint)) return fail(t, "a phase of the fused stage would read outside its tile");
    for (int k = 0; k < kTileCounts; k++) o->max_cnt[k] = std::max(o->max_cnt[k], tc[k]);
    int *off = &o->off[(size_t)t * 3];
    off[0] = (int)o->ge.size();
    off[1] = (int)o->gc.size();
    off[2] = (int)o->gv.size();
    o->ge.insert(o->ge.end(), E.list.begin(), E.list.end());
    o->gc.insert(o->gc.end(), C.list.begin(), C.list.end());
    o->gv.insert(o->gv.end(), V.list.begin(), V.list.end());
    o->blob_off[t] = (long long)o->blob.size();
    pack_blob(b, m, E, C, V, tc, adjoint, &o->blob);
    for (int i = 0; i < 4; i++) o->smem[i] = std::max(o->smem[i], tile_smem(tc, adjoint, 4 << i));
  }
  return "";
}

}  // namespace mpsw
