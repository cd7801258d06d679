// Fused tangent-linear and adjoint RK stages of B FP32 members: one kernel per stage.
//
// The split member kernels (mpsw_members.cuh) run a stage as four grid-wide passes (vertices,
// cells, edge diagnostics, edge tendencies) and pass pv_vertex', pv_cell', pv_edge', ke' and
// the flux rows between them through HBM, roughly tripling the bytes a stage must move.  Here
// one thread block computes a whole stage for one halo tile (mpsw_tiles.h: K owned cells and
// their owned edges): it copies the tile's blob (neighbour records and coefficients) and the
// linearisation point on the tile into shared memory once, then walks the members in chunks of
// M: each chunk's member inputs are copied into shared memory (the next chunk's while the
// current one computes), every intermediate is formed on the tile's halo in shared memory (the
// halo is recomputed by the neighbouring tiles, not exchanged), and only the stage's RK outputs
// go to HBM.  Each thread holds 4 members of one entity (float4 rows), so M / 4 threads share
// an entity.
//
// The arithmetic is the FP32 member arithmetic of the split kernels with the per-entity
// coefficients folded (sign x length / area and the like, formed in FP64 on the host), so
// results agree with them to FP32 rounding; every entity's value is the same expression
// whichever tile forms it, so results do not depend on the tile size.  Physics: the default
// configuration (no del2 / del4 viscosity, no bottom drag, no wind stress); the window uses the
// split kernels otherwise.
#pragma once

#include "mpsw_members.cuh"

namespace mpsw {

using F4 = Mv<float, 4>;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// 16-bit local indices packed two to a word (little endian: the lower index in the low half)
__device__ __forceinline__ int lo16(unsigned w) { return (int)(w & 0xFFFFu); }
__device__ __forceinline__ int hi16(unsigned w) { return (int)(w >> 16); }

// Neighbour records of a tile (layout in mpsw_tiles.h: edge c1 c2 v1 v2 eoe[10]; cell es[6]
// vs[6] nb[6]; vertex es[3] cs[3]), read from shared memory.
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
// n floats of an entity's coefficient record in shared memory (16-byte aligned)
template <int N>
struct Coef {
  float f[N];
};
template <int N>
__device__ __forceinline__ Coef<N> load_coef(const float *p) {
  static_assert(N % 4 == 0, "coefficient records are whole float4s");
  Coef<N> c;
#pragma unroll
  for (int i = 0; i < N / 4; i++) {
    const float4 v = reinterpret_cast<const float4 *>(p)[i];
    c.f[4 * i] = v.x; c.f[4 * i + 1] = v.y; c.f[4 * i + 2] = v.z; c.f[4 * i + 3] = v.w;
  }
  return c;
}

// One block's tile in shared memory: counts, the blob's sections, and the base of the shared
// memory that follows the blob.
struct TileSmem {
  int n[kTileCounts];
  const int *ge, *gc, *gv;
  const uint16_t *vrec, *crec, *erec;
  const float *vco, *c1, *c2, *c3, *eco;
  unsigned char *rest;  // the linearisation point, then member rows
  int group, tile;
};

// Stage block `blockIdx.x`'s tile blob into shared memory (cp.async, one group) and wait for it.
__device__ __forceinline__ TileSmem stage_tile(const TileSetDev &ts, int groups, bool adjoint) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem t;
  t.tile = blockIdx.x / groups;
  t.group = blockIdx.x - t.tile * groups;
  const int *n = ts.cnt + (size_t)t.tile * kTileCounts;
#pragma unroll
  for (int k = 0; k < kTileCounts; k++) t.n[k] = n[k];
  int off[kBlobSections];
  const int bytes = blob_layout(t.n, adjoint, off);
  const unsigned char *g = ts.blob + ts.blob_off[t.tile];
  for (int x = 16 * threadIdx.x; x < bytes; x += 16 * blockDim.x) cp_async16(smem_raw + x, g + x);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  t.ge = reinterpret_cast<const int *>(smem_raw + off[B_GE]);
  t.gc = reinterpret_cast<const int *>(smem_raw + off[B_GC]);
  t.gv = reinterpret_cast<const int *>(smem_raw + off[B_GV]);
  t.vrec = reinterpret_cast<const uint16_t *>(smem_raw + off[B_VREC]);
  t.crec = reinterpret_cast<const uint16_t *>(smem_raw + off[B_CREC]);
  t.erec = reinterpret_cast<const uint16_t *>(smem_raw + off[B_EREC]);
  t.vco = reinterpret_cast<const float *>(smem_raw + off[B_VCOEF]);
  t.c1 = reinterpret_cast<const float *>(smem_raw + off[B_C1]);
  t.c2 = reinterpret_cast<const float *>(smem_raw + off[B_C2]);
  t.c3 = reinterpret_cast<const float *>(smem_raw + off[B_C3]);
  t.eco = reinterpret_cast<const float *>(smem_raw + off[B_ECOEF]);
  t.rest = smem_raw + bytes;
  return t;
}

// rows of M members in shared memory: row i, the thread's slot s (4 members)
#define ROW(arr, i) (arr)[(size_t)(i) * T + s]

// Copy chunk b0's member rows of the tile's edges (x over n_e rows) and cells into shared
// memory as one cp.async group.
template <int T>
__device__ __forceinline__ void prefetch_rows(const TileSmem &t, const float *xe, const float *xc, int B, int b0,
                                              F4 *se, F4 *sc) {
  const int ne = t.n[E_ALL] * T, nc = t.n[C_ALL] * T;
  for (int x = threadIdx.x; x < ne; x += blockDim.x) {
    const int i = x / T, s = x - i * T;
    cp_async16(se + x, xe + (size_t)t.ge[i] * B + b0 + 4 * s);
  }
  for (int x = threadIdx.x; x < nc; x += blockDim.x) {
    const int i = x / T, s = x - i * T;
    cp_async16(sc + x, xc + (size_t)t.gc[i] * B + b0 + 4 * s);
  }
  cp_async_commit();
}

// ----------------------------------------------------------------------------------------
// Tangent-linear stage: sw_compute_solve_diagnostics_tlm + sw_compute_tend_tlm
// (src/mpas_sw_dyncore_tlm.f90) at one linearisation point, and the RK bookkeeping.
// A block takes chunks [group * cpb, (group + 1) * cpb) of its tile's B / M member chunks.
// ----------------------------------------------------------------------------------------
template <int M, int NT>
__global__ void __launch_bounds__(NT, 1) k_tl_fused(TileSetDev ts, int B, int cpb, Base<float> bs,
                                                     const float *__restrict__ ut, const float *__restrict__ ht,
                                                     float a, RK<float, double> rku, RK<float, double> rkh,
                                                     int *bad, int early) {
  constexpr int T = M / 4;
  const TileSmem t = stage_tile(ts, (B / M) / cpb, false);
  const int nEo = t.n[E_OWN], nEm = t.n[E_MID], nEa = t.n[E_ALL], nCo = t.n[C_OWN], nCk = t.n[C_KE],
            nCm = t.n[C_MID], nCa = t.n[C_ALL], nVa = t.n[V_ALL];
  const int tid = threadIdx.x, nt = NT;
  // the linearisation point on the tile (shared by every member)
  float *sUB = reinterpret_cast<float *>(t.rest), *sHB = sUB + nEa, *sPB = sHB + nEa, *sGT = sPB + nEm;
  float *sVB = sGT + nEm, *sGN = sVB + nEm, *sHVB = sGN + nEm, *sVOB = sHVB + nVa;
  F4 *rows = reinterpret_cast<F4 *>(t.rest + 4 * (size_t)base_floats(t.n, false));
  const size_t in_rows = (size_t)(nEa + nCa) * T;  // one buffer of member inputs: u' rows, then h'
  F4 *sPV = rows + 2 * (size_t)(nEa + nCa) * T, *sPC = sPV + (size_t)nVa * T, *sKE = sPC + (size_t)nCm * T;
  F4 *sFA = sKE + (size_t)nCk * T, *sFB = sFA + (size_t)nEm * T, *sPE = sFB + (size_t)nEm * T;
  auto load_base = [&]() {
    for (int i = tid; i < nEa; i += nt) {
      const int g = t.ge[i];
      sUB[i] = __ldg(bs.u + g);
      sHB[i] = __ldg(bs.he + g);
      if (i < nEm) {
        sPB[i] = __ldg(bs.pe + g);
        sGT[i] = __ldg(bs.gpt + g);
        sVB[i] = __ldg(bs.v + g);
        sGN[i] = __ldg(bs.gpn + g);
      }
    }
    for (int i = tid; i < nVa; i += nt) {
      const int g = t.gv[i];
      sHVB[i] = __ldg(bs.hv + g);
      sVOB[i] = __ldg(bs.vort + g);
    }
  };
  if (early) load_base();  // stored linearisation points: no kernel before this one writes them
  pdl_begin();
  if (!early) load_base();
  const int c0 = t.group * cpb;
  prefetch_rows<T>(t, ut, ht, B, c0 * M, rows, rows + (size_t)nEa * T);
  for (int ci = 0; ci < cpb; ci++) {
    const int buf = ci & 1, b0 = (c0 + ci) * M;
    if (ci + 1 < cpb) {
      F4 *nx = rows + (buf ^ 1) * in_rows;
      prefetch_rows<T>(t, ut, ht, B, b0 + M, nx, nx + (size_t)nEa * T);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const F4 *U = rows + buf * in_rows, *H = U + (size_t)nEa * T;

    // phase 1: pv_vertex' (:255-271, :344-360) on the tile's vertices; ke' (:274-316) on the
    // cells of owned edges; thickness tendency (:541-561) and its RK update on owned cells
    for (int x = tid; x < nVa * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const VRec r = load_vrec(t.vrec + 8 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.vco + 8 * (size_t)i);  // sign dc / area x3, kite / area x3, f
      F4 circ = mv_fill<float, 4>(0.f), hh = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        circ = circ + q.f[k] * ROW(U, r.es[k]);
        hh = hh + q.f[3 + k] * ROW(H, r.cs[k]);
      }
      const float rh = 1.f / sHVB[i];
      const float qq = ((q.f[6] + sVOB[i]) * rh) * rh;
      sPV[x] = circ * rh - hh * qq;
    }
    for (int x = tid; x < nCk * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const CRec r = load_crec(t.crec + 24 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.c2 + 8 * (size_t)i);  // 0.25 dc dv / area
      F4 ke = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 6; k++) ke = ke + (q.f[k] * (2.f * sUB[r.es[k]])) * ROW(U, r.es[k]);
      sKE[x] = ke;
    }
    for (int x = tid; x < nCo * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const CRec r = load_crec(t.crec + 24 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.c3 + 8 * (size_t)i);  // sign dv / area
      const F4 hc = ROW(H, i);
      F4 th = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const int e = r.es[k];
        const F4 het = 0.5f * (hc + ROW(H, r.nb[k]));
        th = th - q.f[k] * (ROW(U, e) * sHB[e] + sUB[e] * het);
      }
      rk_members<float, double, 4>(rkh, (size_t)t.gc[i] * B + b0 + 4 * s, th);
    }
    __syncthreads();

    // phase 2: pv_cell' (:397-421)
    for (int x = tid; x < nCm * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const CRec r = load_crec(t.crec + 24 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.c1 + 8 * (size_t)i);  // kite / area
      F4 pc = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 6; k++) pc = pc + q.f[k] * ROW(sPV, r.vs[k]);
      sPC[x] = pc;
    }
    __syncthreads();

    // phase 3: v', gradPVt', gradPVn', pv_edge' with both APVM terms (:319-329, :364-393,
    // :425-445), h_edge' (:117-126), and the edge's thickness flux (u h_edge)' and PV flux
    // (u h_edge pv_edge)', which the normal-velocity tendency sums over edgesOnEdge
    for (int x = tid; x < nEm * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const ERec r = load_erec(t.erec + 16 * (size_t)i);
      const Coef<12> q = load_coef<12>(t.eco + 12 * (size_t)i);  // weightsOnEdge, 1/dv, 1/dc
      F4 vt = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int j = 0; j < 10; j++) vt = vt + q.f[j] * ROW(U, r.eoe[j]);
      const F4 p1 = ROW(sPV, r.v1), p2 = ROW(sPV, r.v2);
      const F4 gptt = (p2 - p1) * q.f[10];
      const F4 gpnt = (ROW(sPC, r.c2) - ROW(sPC, r.c1)) * q.f[11];
      const F4 uet = ROW(U, i);
      const float ub = sUB[i], hb = sHB[i], pb = sPB[i];
      const F4 pet = 0.5f * p1 + 0.5f * p2 - (a * sGT[i]) * vt - (a * sVB[i]) * gptt - (a * sGN[i]) * uet -
                     (a * ub) * gpnt;
      const F4 het = 0.5f * (ROW(H, r.c1) + ROW(H, r.c2));
      sFA[x] = uet * hb + ub * het;
      sFB[x] = (hb * pb) * uet + (ub * hb) * pet + (ub * pb) * het;
      if (i < nEo) sPE[x] = pet;
    }
    __syncthreads();

    // phase 4: normal-velocity tendency (:564-768) and its RK update on owned edges:
    // q' = 0.5 pv_edge sum w (u h_edge)'_j + 0.5 sum w (u h_edge pv_edge)'_j
    //      + 0.5 pv_edge' sum w u_j h_edge_j, minus the gradients of ke' and g h'
    for (int x = tid; x < nEo * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const ERec r = load_erec(t.erec + 16 * (size_t)i);
      const Coef<12> q = load_coef<12>(t.eco + 12 * (size_t)i);
      F4 f1 = mv_fill<float, 4>(0.f), f2 = mv_fill<float, 4>(0.f);
      float sb = 0.f;
#pragma unroll
      for (int j = 0; j < 10; j++) {
        const int k = r.eoe[j];
        f1 = f1 + q.f[j] * ROW(sFA, k);
        f2 = f2 + q.f[j] * ROW(sFB, k);
        sb = sb + (q.f[j] * sUB[k]) * sHB[k];
      }
      const F4 qt = (0.5f * sPB[i]) * f1 + 0.5f * f2 + (0.5f * sb) * sPE[x];
      const F4 grad = (ROW(sKE, r.c2) - ROW(sKE, r.c1)) + float(GRAVITY) * (ROW(H, r.c2) - ROW(H, r.c1));
      const F4 tut = qt - grad * q.f[11];
#pragma unroll
      for (int m = 0; m < 4; m++) flag_nonfinite(bad, tut.x[m]);
      rk_members<float, double, 4>(rku, (size_t)t.ge[i] * B + b0 + 4 * s, tut);
    }
    __syncthreads();  // this chunk's rows are free for the prefetch of the chunk after next
  }
}

// ----------------------------------------------------------------------------------------
// Adjoint stage: sw_compute_tend_adj followed by sw_compute_solve_diagnostics_adj
// (src/mpas_sw_dyncore_adj.f90) at one linearisation point, as gathers over the tile, and the
// adjoint RK bookkeeping (ad_emit).
// ----------------------------------------------------------------------------------------
template <int M, int NT>
__global__ void __launch_bounds__(NT, 1) k_ad_fused(TileSetDev ts, int B, int cpb, Base<float> bs, float a,
                                                     AdIn<float> in, AdOut<float, double> out, int *bad,
                                                     int early) {
  constexpr int T = M / 4;
  const TileSmem t = stage_tile(ts, (B / M) / cpb, true);
  const int nEo = t.n[E_OWN], nEm = t.n[E_MID], nEa = t.n[E_ALL], nCo = t.n[C_OWN], nCk = t.n[C_KE],
            nCm = t.n[C_MID], nCa = t.n[C_ALL], nVa = t.n[V_ALL];
  const int tid = threadIdx.x, nt = NT;
  float *sUB = reinterpret_cast<float *>(t.rest), *sHB = sUB + nEa, *sPB = sHB + nEa, *sVB = sPB + nEa;
  float *sGT = sVB + nEm, *sGN = sGT + nEm, *sHVB = sGN + nEm, *sVOB = sHVB + nVa;
  F4 *rows = reinterpret_cast<F4 *>(t.rest + 4 * (size_t)base_floats(t.n, true));
  const size_t in_rows = (size_t)(nEa + nCa) * T;  // one buffer of member inputs: tu rows, then th
  F4 *sPA = rows + 2 * (size_t)(nEa + nCa) * T, *sHA = sPA + (size_t)nEm * T, *sVT = sHA + (size_t)nEm * T;
  F4 *sUD = sVT + (size_t)nEm * T, *sPC = sUD + (size_t)nEo * T, *sKE = sPC + (size_t)nCm * T;
  F4 *sVO = sKE + (size_t)nCk * T, *sHV = sVO + (size_t)nVa * T;
  auto load_base = [&]() {
    for (int i = tid; i < nEa; i += nt) {
      const int g = t.ge[i];
      sUB[i] = __ldg(bs.u + g);
      sHB[i] = __ldg(bs.he + g);
      sPB[i] = __ldg(bs.pe + g);
      if (i < nEm) {
        sVB[i] = __ldg(bs.v + g);
        sGT[i] = __ldg(bs.gpt + g);
        sGN[i] = __ldg(bs.gpn + g);
      }
    }
    for (int i = tid; i < nVa; i += nt) {
      const int g = t.gv[i];
      sHVB[i] = __ldg(bs.hv + g);
      sVOB[i] = __ldg(bs.vort + g);
    }
  };
  if (early) load_base();
  pdl_begin();
  if (!early) load_base();
  const int c0 = t.group * cpb;
  prefetch_rows<T>(t, in.tu, in.th, B, c0 * M, rows, rows + (size_t)nEa * T);
  for (int ci = 0; ci < cpb; ci++) {
    const int buf = ci & 1, b0 = (c0 + ci) * M;
    if (ci + 1 < cpb) {
      F4 *nx = rows + (buf ^ 1) * in_rows;
      prefetch_rows<T>(t, in.tu, in.th, B, b0 + M, nx, nx + (size_t)nEa * T);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const F4 *TU = rows + buf * in_rows, *TH = TU + (size_t)nEa * T;

    // phase 1, the edges whose adjoints the later phases gather: the q / workpv adjoint over
    // the transposed edgesOnEdge (:689-718) split into its thickness-flux part fa and PV-flux
    // part fb, the thickness-flux adjoint (:720-736), and from them pv_edge_ad, h_edge_ad, the
    // direct u_ad of the edge and the tangential-velocity adjoint of the APVM terms (:193-200,
    // :235-242)
    for (int x = tid; x < nEm * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const ERec r = load_erec(t.erec + 16 * (size_t)i);
      const Coef<24> q = load_coef<24>(t.eco + 24 * (size_t)i);  // w[10], wrev[10], dv, dc
      F4 fa = mv_fill<float, 4>(0.f), fb = mv_fill<float, 4>(0.f);
      float sb = 0.f;
#pragma unroll
      for (int j = 0; j < 10; j++) {
        const int k = r.eoe[j];
        const float wr = q.f[10 + j];
        const F4 tk = ROW(TU, k);
        fa = fa + (wr * sPB[k]) * tk;
        fb = fb + wr * tk;
        sb = sb + (q.f[j] * sUB[k]) * sHB[k];
      }
      fa = 0.5f * fa;
      fb = 0.5f * fb;
      const F4 dth = ROW(TH, r.c2) - ROW(TH, r.c1);
      const float ub = sUB[i], hb = sHB[i], pb = sPB[i], dv = q.f[20];
      const F4 pa = (0.5f * sb) * ROW(TU, i) + (ub * hb) * fb;
      sPA[x] = pa;
      sHA[x] = ub * fa + (ub * pb) * fb + (ub * dv) * dth;
      sVT[x] = -(a * sGT[i]) * pa;
      if (i < nEo) sUD[x] = (dv * hb) * dth + hb * fa + (hb * pb) * fb - (a * sGN[i]) * pa;
    }
    __syncthreads();

    // phase 2, cells: gradPVn adjoint onto pv_cell (:202-213); ke adjoint of the gradient
    // term (:696-699), kept over areaCell (the ke' it transposes was)
    for (int x = tid; x < nCm * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const CRec r = load_crec(t.crec + 24 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.c1 + 8 * (size_t)i);  // sign / dc x6, 1 / area, area
      F4 pc = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 6; k++) pc = pc + ((a * sUB[r.es[k]]) * q.f[k]) * ROW(sPA, r.es[k]);
      sPC[x] = pc;
      if (i < nCk) {
        F4 ke = mv_fill<float, 4>(0.f);
#pragma unroll
        for (int k = 0; k < 6; k++) ke = ke + q.f[k] * ROW(TU, r.es[k]);
        sKE[x] = ke * q.f[6];
      }
    }
    __syncthreads();

    // phase 3, vertices: pv_cell and pv_edge / gradPVt adjoints onto pv_vertex (:215-262),
    // then pv_vertex onto vorticity and h_vertex (:268-292); both kept over areaTriangle
    for (int x = tid; x < nVa * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const VRec r = load_vrec(t.vrec + 8 * (size_t)i);
      const Coef<8> q = load_coef<8>(t.vco + 8 * (size_t)i);  // kite / areaCell x3, sign / dv x3, 1 / area, f
      F4 pv = mv_fill<float, 4>(0.f);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        pv = pv + q.f[k] * ROW(sPC, r.cs[k]);
        pv = pv + (0.5f - (a * sVB[r.es[k]]) * q.f[3 + k]) * ROW(sPA, r.es[k]);
      }
      const float rh = 1.f / sHVB[i], ra = q.f[6];
      const float qq = ((q.f[7] + sVOB[i]) * rh) * rh;
      sVO[x] = (rh * ra) * pv;
      sHV[x] = -(qq * ra) * pv;
    }
    __syncthreads();

    // phase 4: u_ad of owned edges (direct terms, transposed tangential velocity :296-303, ke
    // :306-317, circulation :350-355) and h_ad of owned cells (gravity, h_edge :358-369,
    // h_vertex :286-289), with the stage's RK bookkeeping
    for (int x = tid; x < nEo * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const ERec r = load_erec(t.erec + 16 * (size_t)i);
      const Coef<24> q = load_coef<24>(t.eco + 24 * (size_t)i);
      F4 pu = sUD[x];
#pragma unroll
      for (int j = 0; j < 10; j++) pu = pu + q.f[10 + j] * ROW(sVT, r.eoe[j]);
      const float dc = q.f[21], kc = ((0.5f * dc) * q.f[20]) * sUB[i];
      pu = pu + kc * (ROW(sKE, r.c1) + ROW(sKE, r.c2)) + dc * (ROW(sVO, r.v2) - ROW(sVO, r.v1));
#pragma unroll
      for (int m = 0; m < 4; m++) flag_nonfinite(bad, pu.x[m]);
      ad_emit<float, double, 4>(out, 1, (size_t)t.ge[i] * B + b0 + 4 * s, pu, 1.f);
    }
    for (int x = tid; x < nCo * T; x += nt) {
      const int i = x / T, s = x - i * T;
      const CRec r = load_crec(t.crec + 24 * (size_t)i);
      const Coef<16> q = load_coef<16>(t.c2 + 16 * (size_t)i);  // h_edge halves x6, kites x6
      const float area = t.c1[8 * (size_t)i + 7];
      F4 ph = (float(GRAVITY) * area) * sKE[x];
#pragma unroll
      for (int k = 0; k < 6; k++) {
        ph = ph + q.f[k] * ROW(sHA, r.es[k]);
        ph = ph + q.f[6 + k] * ROW(sHV, r.vs[k]);
      }
      ad_emit<float, double, 4>(out, 0, (size_t)t.gc[i] * B + b0 + 4 * s, ph, area);
    }
    __syncthreads();  // this chunk's rows are free for the prefetch of the chunk after next
  }
}

#undef ROW

}  // namespace mpsw
