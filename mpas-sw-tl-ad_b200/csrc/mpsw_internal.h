// Internal data layout of the B200 shallow-water engine.
//
// Everything on the device is in *internal order*: cells, edges and vertices are renumbered
// along a 3-D Hilbert curve of their positions so that neighbour gathers touch nearby
// addresses; the permutation is applied at the boundary (mpsw_set_var / mpsw_get_var and the
// to/from-internal kernels), so callers always see the reference's numbering.
//
// Connectivity is stored slot-major ([slot][n]) so that, for a fixed slot, consecutive
// threads read consecutive words.  Gather lists that replace the reference's scatter loops
// are sorted by the *reference* index of the scattering entity, so each gather performs the
// same additions in the same order as the reference loop (bit-identical FP64 results).
//
// Member arrays (tangent-linear / adjoint batches) are [n][B]: the B members of one cell,
// edge or vertex are contiguous, so a warp reading one neighbour reads B consecutive values
// and the connectivity word is a broadcast.
#pragma once

#include <cstddef>
#include <cstdint>

namespace mpsw {

constexpr int MAXE = 10;   // max edges (and vertices) of a cell
constexpr int MAXE2 = 20;  // max entries of edgesOnEdge
constexpr int VDEG = 3;    // vertexDegree (triangular dual mesh)

// Physical constants of the reference (src/mpas_sw_dyncore.f90:414,460).
constexpr double GRAVITY = 9.80616;
constexpr double RHO_REF = 1000.0;

template <typename R>
struct MeshDev {
  int nC, nE, nV;
  int max_eoe, max_eoc;        // largest nEdgesOnEdge and nEdgesOnCell of the mesh
  // cells
  const int *c_n;              // [N]      nEdgesOnCell
  const int *c_eoc;            // [MAXE][N] edgesOnCell, reference slot order
  const int *c_es;             // [MAXE][N] edges of the cell sorted by reference edge index
  const signed char *c_esg;    // [MAXE][N] +1 if the cell is cellsOnEdge(1) of that edge, else -1
  const int *c_vs;             // [MAXE][N] vertices of the cell sorted by reference vertex index
  const R *c_vk;               // [MAXE][N] kiteAreasOnVertex of (that vertex, this cell)
  const R *c_area;             // [N]
  const R *c_hs;               // [N]      h_s (bottom topography)
  const R *c_coef;             // [3][MAXE][N] coeffs_reconstruct
  const R *c_trig;             // [4][N]   cos(lat), sin(lat), cos(lon), sin(lon)
  // edges
  const int *e_c1, *e_c2;      // [E]      cellsOnEdge
  const int *e_v1, *e_v2;      // [E]      verticesOnEdge
  const int *e_va, *e_vb;      // [E]      the two vertices listing this edge, reference vertex order
  const int *e_slot1, *e_slot2;// [E]      slot of this edge in edgesOnCell of cell 1 / cell 2
  const int *e_n;              // [E]      nEdgesOnEdge
  const int *e_eoe;            // [MAXE2][E] edgesOnEdge
  const int *e_rev;            // [MAXE2][E] slot of this edge in the neighbour's edgesOnEdge
  const R *e_w;                // [MAXE2][E] weightsOnEdge
  const R *e_wrev;             // [MAXE2][E] weight of this edge in the neighbour's list (transpose)
  const R *e_dc, *e_dv;        // [E]
  const R *e_sc2, *e_sc4;      // [E]      meshScalingDel2/Del4
  const R *e_usrc;             // [E]      u_src
  // vertices
  const int *v_es;             // [3][V]   edges of the vertex sorted by reference edge index
  const signed char *v_esg;    // [3][V]   +1 if the vertex is verticesOnEdge(2) of that edge
  const int *v_c;              // [3][V]   cellsOnVertex (reference order)
  const R *v_k;                // [3][V]   kiteAreasOnVertex
  const int *v_e;              // [3][V]   edgesOnVertex (reference order)
  const R *v_area, *v_f;       // [V]      areaTriangle, fVertex
};

// Physics switches and scalars of one configuration (namelist, src/mpas_sw_module.f90:23-42).
template <typename R>
struct Phys {
  R dt, apvm, visc2, visc4;
  int wind, drag, tc1, sphere;
  // set to 1 by a tendency kernel that forms a non-finite (NaN / Inf) normal-velocity
  // tendency or adjoint; null: not checked
  int *bad = nullptr;
};

// Diagnostics of one state (B members, [n][B]); null pointers are not written.
template <typename R>
struct Diag {
  R *circ, *vort, *hv, *pvv;       // vertices
  R *div, *ke, *pc, *vc;           // cells
  R *v, *gpt, *pe, *gpn, *he;      // edges
  R *dsq_u;                        // edges    (del4 only)
  R *dsq_vort;                     // vertices (del4 only)
  R *dsq_div;                      // cells    (del4 only)
};

// Linearisation point of one RK stage (single trajectory, [n]).
template <typename R>
struct Base {
  const R *u, *he, *v, *gpt, *gpn, *pe;  // edges
  const R *vort, *hv;                    // vertices
  const R *ke;                           // cells (bottom drag only)
};

// RK4 bookkeeping of one stage for one prognostic field (src/mpas_sw_module.f90:590-611):
//   next    = x0 + c * tend   (provisional state of the next stage, omitted at stage 4)
//   acc_out = acc_in + w * tend
template <typename R, typename A>
struct RK {
  const A *x0;
  const A *acc_in;
  A *acc_out;
  R *next;
  A c, w;
  R off;      // next stores x - off (reference-depth offset of the reduced-precision h)
  int frozen; // test case 1: the wind stays at x0
  // Deferred accumulation (member sweeps): stages 1-3 store their tendency in t_out instead of
  // accumulating; the last stage (t_in[0] set) writes acc_out = (((x0 + wt[0] t_in[0]) +
  // wt[1] t_in[1]) + wt[2] t_in[2]) + w t, the same FP64 operations as accumulating stage by stage.
  R *t_out;
  const R *t_in[3];
  A wt[3];
  // FP32 members: the step's input rounded to R; when set, stages 1-3 form the next provisional
  // state as x0r + c t in R instead of reading the FP64 state x0
  const R *x0r;
};

// Input of one adjoint stage: its tendency adjoint, tu (edges) and th / areaCell (cells), as
// formed by the previous adjoint stage (or k_ad_tinit) from src/mpas_sw_module.f90:912-942:
// tend_ad = w * x2_ad + c * provis_ad(next stage) [+ seed].
template <typename R>
struct AdIn {
  const R *tu, *th;
};

// Adjoint seeds of the diagnostics (module *_ad arrays); single member only.
template <typename R>
struct AdSeeds {
  const R *v, *he, *hv, *pe, *pvv, *pc, *circ, *vort, *div, *ke, *vc, *gpn, *gpt;
};

// Edge/cell/vertex intermediates of one adjoint stage ([n][B]).
template <typename R>
struct AdWork {
  R *pe_ad, *he_ad, *ud, *gpn_ad, *gpt_ad, *v_ad;  // edges
  R *du_ad;                                       // edges    (del4)
  R *pc_ad, *ke_ad, *div_ad, *hd;                 // cells
  R *dd_ad;                                       // cells    (del4)
  R *hv_ad, *circ_ad;                             // vertices
  R *dc_ad;                                       // vertices (del4)
};

// Where the provisional-state adjoint `pad` of a stage goes.
//   AD_SET:   acc = pad              AD_ADD: acc = acc + pad
//   AD_FINAL: dst = (acc + x2) + pad (the step's input adjoint; dst may alias x2)
// and the tendency adjoint of the stage before it:
//   tu_next = wu * x2 + cu * pad     (AD_FINAL: wu * dst, the first stage of the next step)
//   th_next = (wh * x2 + ch * pad) / areaCell
enum AdMode { AD_SET = 0, AD_ADD = 1, AD_FINAL = 2 };
template <typename R, typename A>
struct AdOut {
  A *acc_u, *acc_h;
  const A *x2u, *x2h;
  A *dst_u, *dst_h;
  int mode;
  R *tu_next, *th_next;
  A wu, cu, wh, ch;
  // Deferred accumulation (member sweeps): instead of adding into acc, AD_SET / AD_ADD stages
  // store their contribution in pad_out_*, and AD_FINAL (pad_in_*[0] set) sums the three stored
  // contributions in stage order before adding x2 and its own: the same FP64 operations.
  R *pad_out_u, *pad_out_h;
  const R *pad_in_u[3], *pad_in_h[3];
  // FP32 members: x2 rounded to R.  When set, AD_SET / AD_ADD stages form tu_next / th_next from
  // it (four bytes a value instead of x2's eight), and AD_FINAL writes the rounding of its dst
  // there for the step before.
  R *x2r_u, *x2r_h;
};

// ---- fused member stages (mpsw_fused.cuh, tiles built by mpsw_tiles.cpp) ----------------
#ifdef __CUDACC__
#define MPSW_HD __host__ __device__
#else
#define MPSW_HD
#endif

// Prefix sizes of a tile's local spaces; the meaning of each layer for the tangent-linear and
// the adjoint stage is given in mpsw_tiles.h.
enum TileLayer { E_OWN, E_MID, E_ALL, C_OWN, C_KE, C_MID, C_ALL, V_ALL, kTileCounts };

// Sections of a tile's blob: everything a fused stage needs of the mesh for that tile, in the
// tile's local order, copied into shared memory once per tile.  Internal indices (ge, gc, gv),
// neighbour records as 16-bit local indices (vertex 16 B, cell 48 B, edge 32 B), and per-entity
// coefficient records of 8 / 16 / 12 / 24 floats (their content per stage: mpsw_tiles.cpp).
enum BlobSection { B_GE, B_GC, B_GV, B_VREC, B_CREC, B_EREC, B_VCOEF, B_C1, B_C2, B_C3, B_ECOEF, kBlobSections };

MPSW_HD inline int blob_up16(int x) { return (x + 15) & ~15; }

// Byte offsets of the sections of a tile's blob from its counts; returns the blob's size.
MPSW_HD inline int blob_layout(const int *cnt, bool adjoint, int *off) {
  int sz[kBlobSections];
  sz[B_GE] = 4 * cnt[E_ALL];
  sz[B_GC] = 4 * cnt[C_ALL];
  sz[B_GV] = 4 * cnt[V_ALL];
  sz[B_VREC] = 16 * cnt[V_ALL];
  sz[B_CREC] = 48 * cnt[C_MID];
  sz[B_EREC] = 32 * cnt[E_MID];
  sz[B_VCOEF] = 32 * cnt[V_ALL];
  sz[B_C1] = 32 * cnt[C_MID];
  sz[B_C2] = adjoint ? 64 * cnt[C_OWN] : 32 * cnt[C_KE];
  sz[B_C3] = adjoint ? 0 : 32 * cnt[C_OWN];
  sz[B_ECOEF] = (adjoint ? 96 : 48) * cnt[E_MID];
  int o = 0;
  for (int k = 0; k < kBlobSections; k++) {
    off[k] = o;
    o += blob_up16(sz[k]);
  }
  return o;
}

// Floats of the linearisation point a fused stage stages per tile (see mpsw_fused.cuh).
MPSW_HD inline int base_floats(const int *cnt, bool adjoint) {
  return blob_up16(4 * ((adjoint ? 3 : 2) * cnt[E_ALL] + (adjoint ? 3 : 4) * cnt[E_MID] + 2 * cnt[V_ALL])) / 4;
}

// Member rows (M floats each) of a fused stage's block: inputs double-buffered, then the
// stage's intermediates (see mpsw_fused.cuh).
MPSW_HD inline int member_rows(const int *cnt, bool adjoint) {
  const int in = 2 * (cnt[E_ALL] + cnt[C_ALL]);
  return adjoint ? in + 3 * cnt[E_MID] + cnt[E_OWN] + cnt[C_MID] + cnt[C_KE] + 2 * cnt[V_ALL]
                 : in + cnt[V_ALL] + cnt[C_MID] + cnt[C_KE] + 2 * cnt[E_MID] + cnt[E_OWN];
}

// Halo tiles on the device: per tile its counts and the byte offset of its blob.
struct TileSetDev {
  int ntiles = 0;
  const int *cnt = nullptr;
  const long long *blob_off = nullptr;
  const unsigned char *blob = nullptr;
  size_t smem[4] = {0, 0, 0, 0};  // dynamic shared memory of a block for 4, 8, 16, 32 members per chunk
};

struct FusedDev {
  bool ok = false;  // tiles built (meshes within 6 edgesOnCell, 10 edgesOnEdge)
  int M = 8;        // members per chunk the tiles were sized for (4, 8, 16 or 32)
  int nt = 512;     // threads per block (256, 512 or 1024)
  TileSetDev tl, ad;
};

// Up to kConvMax double arrays rounded to float by one launch (see convert_list).
constexpr int kConvMax = 10;
// up to kConvMax FP64 arrays, each rounded to FP32 into dst[i] and/or copied into dst64[i]
// (either may be null)
struct ConvList {
  const double *src[kConvMax];
  float *dst[kConvMax];
  double *dst64[kConvMax];
  long long n[kConvMax];
  int count;
};

}  // namespace mpsw
