// Fused tangent-linear and adjoint RK stages of B FP32 members: one kernel per stage.
//
// The split member kernels (mpsw_members.cuh) run a stage as four grid-wide passes (vertices,
// cells, edge diagnostics, edge tendencies) and pass pv_vertex', pv_cell', pv_edge', ke' and
// the flux rows between them through HBM, roughly tripling the bytes a stage must move.  Here
// one thread block computes a whole stage for one halo tile (mpsw_tiles.h: K owned cells and
// their owned edges) and a chunk of M members: it copies the tile's member inputs into shared
// memory once, forms every intermediate on the tile's halo in shared memory (the halo is
// recomputed by the neighbouring tiles, not exchanged), and writes only the stage's RK outputs.
// Each thread holds 4 members of one entity (float4 rows), so M / 4 threads share an entity.
//
// The arithmetic is the FP32 member arithmetic of the split kernels with the per-entity
// coefficients folded (sign x length / area and the like, formed once on the host), so results
// agree with them to FP32 rounding; every entity's value is the same expression whichever tile
// forms it, so results do not depend on the tile size.  Physics: the default configuration (no
// del2 / del4 viscosity, no bottom drag, no wind stress); the window uses the split kernels
// otherwise.
#pragma once

#include "mpsw_members.cuh"

namespace mpsw {

using F4 = Mv<float, 4>;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// 16-bit local indices packed two to a word (little endian: the lower index in the low half)
__device__ __forceinline__ int lo16(unsigned w) { return (int)(w & 0xFFFFu); }
__device__ __forceinline__ int hi16(unsigned w) { return (int)(w >> 16); }

// Local records of one tile (layout in mpsw_tiles.h: edge c1 c2 v1 v2 eoe[10]; cell es[6]
// vs[6] nb[6]; vertex es[3] cs[3]).
struct ERec {
  int c1, c2, v1, v2, eoe[10];
};
struct CRec {
  int es[6], vs[6], nb[6];
};
struct VRec {
  int es[3], cs[3];
};
__device__ __forceinline__ ERec load_erec(const uint16_t *p) {
  const uint4 a = *reinterpret_cast<const uint4 *>(p), b = *reinterpret_cast<const uint4 *>(p + 8);
  ERec r;
  r.c1 = lo16(a.x); r.c2 = hi16(a.x); r.v1 = lo16(a.y); r.v2 = hi16(a.y);
  r.eoe[0] = lo16(a.z); r.eoe[1] = hi16(a.z); r.eoe[2] = lo16(a.w); r.eoe[3] = hi16(a.w);
  r.eoe[4] = lo16(b.x); r.eoe[5] = hi16(b.x); r.eoe[6] = lo16(b.y); r.eoe[7] = hi16(b.y);
  r.eoe[8] = lo16(b.z); r.eoe[9] = hi16(b.z);
  return r;
}
__device__ __forceinline__ CRec load_crec(const uint16_t *p) {
  const uint4 a = *reinterpret_cast<const uint4 *>(p), b = *reinterpret_cast<const uint4 *>(p + 8),
              c = *reinterpret_cast<const uint4 *>(p + 16);
  const unsigned w[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
  auto at = [&](int q) { return (q & 1) ? hi16(w[q >> 1]) : lo16(w[q >> 1]); };
  CRec r;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    r.es[k] = at(k);
    r.vs[k] = at(6 + k);
    r.nb[k] = at(12 + k);
  }
  return r;
}
__device__ __forceinline__ VRec load_vrec(const uint16_t *p) {
  const uint4 a = *reinterpret_cast<const uint4 *>(p);
  VRec r;
  r.es[0] = lo16(a.x); r.es[1] = hi16(a.x); r.es[2] = lo16(a.y);
  r.cs[0] = hi16(a.y); r.cs[1] = lo16(a.z); r.cs[2] = hi16(a.z);
  return r;
}

// The tile of block `blockIdx.x` and its member chunk (the chunk varies fastest, so the blocks
// of one tile run side by side and share its records in L2).
struct TileView {
  int n[kTileCounts];
  const int *ge, *gc, *gv;
  const uint16_t *er, *cr, *vr;
  int b0;
};
__device__ __forceinline__ TileView tile_view(const TileSetDev &ts, int B, int M) {
  const int chunks = B / M;
  const int tile = blockIdx.x / chunks;
  TileView v;
  const int *n = ts.cnt + (size_t)tile * kTileCounts;
#pragma unroll
  for (int k = 0; k < kTileCounts; k++) v.n[k] = n[k];
  const int *off = ts.off + (size_t)tile * 3;
  v.ge = ts.ge + off[0];
  v.gc = ts.gc + off[1];
  v.gv = ts.gv + off[2];
  v.er = ts.erec + (size_t)off[0] * 16;
  v.cr = ts.crec + (size_t)off[1] * 24;
  v.vr = ts.vrec + (size_t)off[2] * 8;
  v.b0 = (blockIdx.x - tile * chunks) * M;
  return v;
}

// rows of M members in shared memory: row i, the thread's slot s (4 members)
#define ROW(arr, i) (arr)[(size_t)(i) * T + s]

// ----------------------------------------------------------------------------------------
// Tangent-linear stage: sw_compute_solve_diagnostics_tlm + sw_compute_tend_tlm
// (src/mpas_sw_dyncore_tlm.f90) at one linearisation point, and the RK bookkeeping.
// ----------------------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(256, 3) k_tl_fused(TileSetDev ts, FusedMesh fm, MeshDev<float> m, int B,
                                                     Base<float> bs, const float *__restrict__ ut,
                                                     const float *__restrict__ ht, float a, RK<float, double> rku,
                                                     RK<float, double> rkh, int *bad, int early) {
  constexpr int T = M / 4;
  const TileView tv = tile_view(ts, B, M);
  const int nEo = tv.n[E_OWN], nEm = tv.n[E_MID], nEa = tv.n[E_ALL], nCo = tv.n[C_OWN], nCk = tv.n[C_KE],
            nCm = tv.n[C_MID], nCa = tv.n[C_ALL], nVa = tv.n[V_ALL];
  const int nE = m.nE, nC = m.nC, nV = m.nV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F4 *sU = reinterpret_cast<F4 *>(smem_raw);
  F4 *sH = sU + (size_t)nEa * T, *sPV = sH + (size_t)nCa * T, *sPC = sPV + (size_t)nVa * T;
  F4 *sKE = sPC + (size_t)nCm * T, *sFA = sKE + (size_t)nCk * T, *sFB = sFA + (size_t)nEm * T;
  F4 *sPE = sFB + (size_t)nEm * T;
  float *sUB = reinterpret_cast<float *>(sPE + (size_t)nEo * T), *sHB = sUB + nEa;
  const int tid = threadIdx.x, nt = blockDim.x;
  // u and h_edge of the linearisation point on the tile's edges (shared by all members)
  if (!early) pdl_begin();
  for (int i = tid; i < nEa; i += nt) {
    const int g = tv.ge[i];
    sUB[i] = __ldg(bs.u + g);
    sHB[i] = __ldg(bs.he + g);
  }
  if (early) pdl_begin();
  // member inputs of the tile: u' on its edges, h' on its cells
  for (int x = tid; x < nEa * T; x += nt) {
    const int i = x / T, s = x - i * T;
    cp_async16(sU + x, ut + (size_t)tv.ge[i] * B + tv.b0 + 4 * s);
  }
  for (int x = tid; x < nCa * T; x += nt) {
    const int i = x / T, s = x - i * T;
    cp_async16(sH + x, ht + (size_t)tv.gc[i] * B + tv.b0 + 4 * s);
  }
  cp_async_wait_all();
  __syncthreads();

  // phase 1: pv_vertex' (:255-271, :344-360) on the tile's vertices; ke' (:274-316) on the
  // cells of owned edges; thickness tendency (:541-561) and its RK update on owned cells
  for (int x = tid; x < nVa * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gv[i];
    const VRec r = load_vrec(tv.vr + (size_t)i * 8);
    F4 circ = mv_fill<float, 4>(0.f), hh = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      circ = circ + __ldg(fm.v_cc + (size_t)k * nV + g) * ROW(sU, r.es[k]);
      hh = hh + __ldg(fm.v_kr + (size_t)k * nV + g) * ROW(sH, r.cs[k]);
    }
    const float rh = 1.f / __ldg(bs.hv + g);
    const float q = ((__ldg(m.v_f + g) + __ldg(bs.vort + g)) * rh) * rh;
    sPV[x] = circ * rh - hh * q;
  }
  for (int x = tid; x < nCk * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gc[i];
    const CRec r = load_crec(tv.cr + (size_t)i * 24);
    F4 ke = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 6; k++)
      ke = ke + (__ldg(fm.c_kec + (size_t)k * nC + g) * (2.f * sUB[r.es[k]])) * ROW(sU, r.es[k]);
    sKE[x] = ke;
  }
  for (int x = tid; x < nCo * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gc[i];
    const CRec r = load_crec(tv.cr + (size_t)i * 24);
    const F4 hc = ROW(sH, i);
    F4 th = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const int e = r.es[k];
      const F4 het = 0.5f * (hc + ROW(sH, r.nb[k]));
      th = th - __ldg(fm.c_sdv + (size_t)k * nC + g) * (ROW(sU, e) * sHB[e] + sUB[e] * het);
    }
    rk_members<float, double, 4>(rkh, (size_t)g * B + tv.b0 + 4 * s, th);
  }
  __syncthreads();

  // phase 2: pv_cell' (:397-421)
  for (int x = tid; x < nCm * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gc[i];
    const CRec r = load_crec(tv.cr + (size_t)i * 24);
    F4 pc = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 6; k++) pc = pc + __ldg(fm.c_kr + (size_t)k * nC + g) * ROW(sPV, r.vs[k]);
    sPC[x] = pc;
  }
  __syncthreads();

  // phase 3: v', gradPVt', gradPVn', pv_edge' with both APVM terms (:319-329, :364-393,
  // :425-445), h_edge' (:117-126), and the edge's thickness flux (u h_edge)' and PV flux
  // (u h_edge pv_edge)', which the normal-velocity tendency sums over edgesOnEdge
  for (int x = tid; x < nEm * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.ge[i];
    const ERec r = load_erec(tv.er + (size_t)i * 16);
    F4 vt = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int j = 0; j < 10; j++) vt = vt + __ldg(m.e_w + (size_t)j * nE + g) * ROW(sU, r.eoe[j]);
    const F4 p1 = ROW(sPV, r.v1), p2 = ROW(sPV, r.v2);
    const F4 gptt = (p2 - p1) * __ldg(fm.e_rdv + g);
    const F4 gpnt = (ROW(sPC, r.c2) - ROW(sPC, r.c1)) * __ldg(fm.e_rdc + g);
    const F4 uet = ROW(sU, i);
    const float ub = sUB[i], hb = sHB[i], pb = __ldg(bs.pe + g);
    const F4 pet = 0.5f * p1 + 0.5f * p2 - (a * __ldg(bs.gpt + g)) * vt - (a * __ldg(bs.v + g)) * gptt -
                   (a * __ldg(bs.gpn + g)) * uet - (a * ub) * gpnt;
    const F4 het = 0.5f * (ROW(sH, r.c1) + ROW(sH, r.c2));
    sFA[x] = uet * hb + ub * het;
    sFB[x] = (hb * pb) * uet + (ub * hb) * pet + (ub * pb) * het;
    if (i < nEo) sPE[x] = pet;
  }
  __syncthreads();

  // phase 4: normal-velocity tendency (:564-768) and its RK update on owned edges:
  // q' = 0.5 pv_edge sum w (u h_edge)'_j + 0.5 sum w (u h_edge pv_edge)'_j
  //      + 0.5 pv_edge' sum w u_j h_edge_j, minus the gradients of ke' and g h'
  for (int x = tid; x < nEo * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.ge[i];
    const ERec r = load_erec(tv.er + (size_t)i * 16);
    F4 f1 = mv_fill<float, 4>(0.f), f2 = mv_fill<float, 4>(0.f);
    float sb = 0.f;
#pragma unroll
    for (int j = 0; j < 10; j++) {
      const int k = r.eoe[j];
      const float w = __ldg(m.e_w + (size_t)j * nE + g);
      f1 = f1 + w * ROW(sFA, k);
      f2 = f2 + w * ROW(sFB, k);
      sb = sb + (w * sUB[k]) * sHB[k];
    }
    const F4 qt = (0.5f * __ldg(bs.pe + g)) * f1 + 0.5f * f2 + (0.5f * sb) * sPE[x];
    const F4 grad = (ROW(sKE, r.c2) - ROW(sKE, r.c1)) + float(GRAVITY) * (ROW(sH, r.c2) - ROW(sH, r.c1));
    const F4 tut = qt - grad * __ldg(fm.e_rdc + g);
#pragma unroll
    for (int q = 0; q < 4; q++) flag_nonfinite(bad, tut.x[q]);
    rk_members<float, double, 4>(rku, (size_t)g * B + tv.b0 + 4 * s, tut);
  }
}

// ----------------------------------------------------------------------------------------
// Adjoint stage: sw_compute_tend_adj followed by sw_compute_solve_diagnostics_adj
// (src/mpas_sw_dyncore_adj.f90) at one linearisation point, as gathers over the tile, and the
// adjoint RK bookkeeping (ad_emit).
// ----------------------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(256, 3) k_ad_fused(TileSetDev ts, FusedMesh fm, MeshDev<float> m, int B,
                                                     Base<float> bs, float a, AdIn<float> in,
                                                     AdOut<float, double> out, int *bad, int early) {
  constexpr int T = M / 4;
  const TileView tv = tile_view(ts, B, M);
  const int nEo = tv.n[E_OWN], nEm = tv.n[E_MID], nEa = tv.n[E_ALL], nCo = tv.n[C_OWN], nCk = tv.n[C_KE],
            nCm = tv.n[C_MID], nCa = tv.n[C_ALL], nVa = tv.n[V_ALL];
  const int nE = m.nE, nC = m.nC, nV = m.nV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F4 *sT = reinterpret_cast<F4 *>(smem_raw);
  F4 *sTh = sT + (size_t)nEa * T, *sPA = sTh + (size_t)nCa * T, *sHA = sPA + (size_t)nEm * T;
  F4 *sVT = sHA + (size_t)nEm * T, *sUD = sVT + (size_t)nEm * T, *sPC = sUD + (size_t)nEo * T;
  F4 *sKE = sPC + (size_t)nCm * T, *sVO = sKE + (size_t)nCk * T, *sHV = sVO + (size_t)nVa * T;
  float *sUB = reinterpret_cast<float *>(sHV + (size_t)nVa * T), *sHB = sUB + nEa, *sPB = sHB + nEa;
  float *sVB = sPB + nEa;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (!early) pdl_begin();
  for (int i = tid; i < nEa; i += nt) {
    const int g = tv.ge[i];
    sUB[i] = __ldg(bs.u + g);
    sHB[i] = __ldg(bs.he + g);
    sPB[i] = __ldg(bs.pe + g);
    if (i < nEm) sVB[i] = __ldg(bs.v + g);
  }
  if (early) pdl_begin();
  // tendency adjoints on the tile: tu on its edges, th (already over areaCell) on its cells
  for (int x = tid; x < nEa * T; x += nt) {
    const int i = x / T, s = x - i * T;
    cp_async16(sT + x, in.tu + (size_t)tv.ge[i] * B + tv.b0 + 4 * s);
  }
  for (int x = tid; x < nCa * T; x += nt) {
    const int i = x / T, s = x - i * T;
    cp_async16(sTh + x, in.th + (size_t)tv.gc[i] * B + tv.b0 + 4 * s);
  }
  cp_async_wait_all();
  __syncthreads();

  // phase 1, the edges whose adjoints the later phases gather: the q / workpv adjoint over the
  // transposed edgesOnEdge (:689-718) split into its thickness-flux part fa and PV-flux part fb,
  // the thickness-flux adjoint (:720-736), and from them pv_edge_ad, h_edge_ad, the direct u_ad
  // of the edge and the tangential-velocity adjoint of the APVM terms (:193-200, :235-242)
  for (int x = tid; x < nEm * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.ge[i];
    const ERec r = load_erec(tv.er + (size_t)i * 16);
    F4 fa = mv_fill<float, 4>(0.f), fb = mv_fill<float, 4>(0.f);
    float sb = 0.f;
#pragma unroll
    for (int j = 0; j < 10; j++) {
      const int k = r.eoe[j];
      const float wr = __ldg(m.e_wrev + (size_t)j * nE + g);
      const F4 tk = ROW(sT, k);
      fa = fa + (wr * sPB[k]) * tk;
      fb = fb + wr * tk;
      sb = sb + (__ldg(m.e_w + (size_t)j * nE + g) * sUB[k]) * sHB[k];
    }
    fa = 0.5f * fa;
    fb = 0.5f * fb;
    const F4 dth = ROW(sTh, r.c2) - ROW(sTh, r.c1);
    const float ub = sUB[i], hb = sHB[i], pb = sPB[i], dv = __ldg(m.e_dv + g);
    const F4 pa = (0.5f * sb) * ROW(sT, i) + (ub * hb) * fb;
    sPA[x] = pa;
    sHA[x] = ub * fa + (ub * pb) * fb + (ub * dv) * dth;
    sVT[x] = -(a * __ldg(bs.gpt + g)) * pa;
    if (i < nEo) sUD[x] = (dv * hb) * dth + hb * fa + (hb * pb) * fb - (a * __ldg(bs.gpn + g)) * pa;
  }
  __syncthreads();

  // phase 2, cells: gradPVn adjoint onto pv_cell (:202-213); ke adjoint of the gradient term
  // (:696-699), kept over areaCell (the ke' it transposes was)
  for (int x = tid; x < nCm * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gc[i];
    const CRec r = load_crec(tv.cr + (size_t)i * 24);
    F4 pc = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 6; k++)
      pc = pc + ((a * sUB[r.es[k]]) * __ldg(fm.c_src + (size_t)k * nC + g)) * ROW(sPA, r.es[k]);
    sPC[x] = pc;
    if (i < nCk) {
      F4 ke = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 6; k++) ke = ke + __ldg(fm.c_src + (size_t)k * nC + g) * ROW(sT, r.es[k]);
      sKE[x] = ke * (1.f / __ldg(m.c_area + g));
    }
  }
  __syncthreads();

  // phase 3, vertices: pv_cell and pv_edge / gradPVt adjoints onto pv_vertex (:215-262), then
  // pv_vertex onto vorticity and h_vertex (:268-292); both kept over areaTriangle
  for (int x = tid; x < nVa * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gv[i];
    const VRec r = load_vrec(tv.vr + (size_t)i * 8);
    F4 pv = mv_fill<float, 4>(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      pv = pv + __ldg(fm.v_kc + (size_t)k * nV + g) * ROW(sPC, r.cs[k]);
      pv = pv + (0.5f - (a * sVB[r.es[k]]) * __ldg(fm.v_sr + (size_t)k * nV + g)) * ROW(sPA, r.es[k]);
    }
    const float rh = 1.f / __ldg(bs.hv + g), ra = 1.f / __ldg(m.v_area + g);
    const float q = ((__ldg(m.v_f + g) + __ldg(bs.vort + g)) * rh) * rh;
    sVO[x] = (rh * ra) * pv;
    sHV[x] = -(q * ra) * pv;
  }
  __syncthreads();

  // phase 4: u_ad of owned edges (direct terms, transposed tangential velocity :296-303, ke
  // :306-317, circulation :350-355) and h_ad of owned cells (gravity, h_edge :358-369,
  // h_vertex :286-289), with the stage's RK bookkeeping
  for (int x = tid; x < nEo * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.ge[i];
    const ERec r = load_erec(tv.er + (size_t)i * 16);
    F4 pu = sUD[x];
#pragma unroll
    for (int j = 0; j < 10; j++) pu = pu + __ldg(m.e_wrev + (size_t)j * nE + g) * ROW(sVT, r.eoe[j]);
    const float dc = __ldg(m.e_dc + g), kc = ((0.5f * dc) * __ldg(m.e_dv + g)) * sUB[i];
    pu = pu + kc * (ROW(sKE, r.c1) + ROW(sKE, r.c2)) + dc * (ROW(sVO, r.v2) - ROW(sVO, r.v1));
#pragma unroll
    for (int q = 0; q < 4; q++) flag_nonfinite(bad, pu.x[q]);
    ad_emit<float, double, 4>(out, 1, (size_t)g * B + tv.b0 + 4 * s, pu, 1.f);
  }
  for (int x = tid; x < nCo * T; x += nt) {
    const int i = x / T, s = x - i * T, g = tv.gc[i];
    const CRec r = load_crec(tv.cr + (size_t)i * 24);
    const float area = __ldg(m.c_area + g);
    F4 ph = (float(GRAVITY) * area) * sKE[x];
#pragma unroll
    for (int k = 0; k < 6; k++) {
      ph = ph + __ldg(fm.c_hk + (size_t)k * nC + g) * ROW(sHA, r.es[k]);
      ph = ph + __ldg(m.c_vk + (size_t)k * nC + g) * ROW(sHV, r.vs[k]);
    }
    ad_emit<float, double, 4>(out, 0, (size_t)g * B + tv.b0 + 4 * s, ph, area);
  }
}

#undef ROW

}  // namespace mpsw
