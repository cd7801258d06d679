// Definitions of the launchers declared in mpsw_launch.h (included by one translation unit
// per precision, which also instantiates them).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <initializer_list>
#include <stdexcept>
#include <utility>

#include "mpsw_kernels.cuh"
#include "mpsw_launch.h"
#include "mpsw_fused.cuh"
#include "mpsw_members.cuh"

namespace mpsw {

constexpr int kThreads = 128;
constexpr size_t kFusedSmemMax = 227 * 1024;   // shared memory a block may use

// Grid and block for `total` threads: 128-thread blocks (measured faster than 256 for the
// latency-bound gathers here), halved (down to 64) while that leaves fewer than two blocks per
// SM, so thin single-trajectory launches still spread over all SMs.
struct LaunchCfg {
  int grid, block;
  size_t smem = 0;  // dynamic shared memory bytes
};
// MPSW_BLOCK=64|128|256 overrides the starting block size.
inline int block_threads() {
  static const int b = [] {
    const char *e = std::getenv("MPSW_BLOCK");
    const int v = e ? std::atoi(e) : 0;
    return (v == 64 || v == 128 || v == 256) ? v : kThreads;
  }();
  return b;
}
inline LaunchCfg launch_cfg(long long total, int block0 = 0) {
  int block = block0 ? block0 : block_threads();
  while (block > 64 && total < 2LL * 148 * block) block >>= 1;
  long long g = (total + block - 1) / block;
  const long long cap = 148LL * 32 * 128 / block;  // grid-stride beyond 4096 threads per SM
  if (g < 1) g = 1;
  return {(int)(g < cap ? g : cap), block, 0};
}

// Programmatic dependent launch: every kernel is launched with programmatic stream
// serialisation, so the GPU may schedule it while its predecessor on the stream is still
// draining; each kernel begins with griddepcontrol.wait (pdl_begin, in MPSW_GRID_LOOP), which
// returns once the predecessor has completed and its writes are visible.  MPSW_PDL=0 launches
// with plain stream order instead.
inline bool pdl_enabled() {
  static const bool on = !(std::getenv("MPSW_PDL") && std::atoi(std::getenv("MPSW_PDL")) == 0);
  return on;
}

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), LaunchCfg c, cudaStream_t s, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)c.grid);
  cfg.blockDim = dim3((unsigned)c.block);
  cfg.dynamicSmemBytes = c.smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  // a failed launch is reported by the cudaGetLastError check that follows every launch sequence
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// every kernel launch of the engine goes through one of these launchers and is counted here
extern long long g_launches;

// Members per thread of a member kernel: 16 bytes of R per vector load (4 floats, 2 doubles),
// or `prefer` (a kernel measured faster at another width), reduced while B is not a multiple of
// it or a buffer is not aligned to V elements of the wider of R and A.  MPSW_VEC=1|2|4|8 overrides the starting width (8: FP32 only).
template <typename R, typename A>
inline int vec_width(int B, std::initializer_list<const void *> ptrs, int prefer = 0) {
  static const int forced = [] {
    const char *e = std::getenv("MPSW_VEC");
    const int v = e ? std::atoi(e) : 0;
    return (v == 1 || v == 2 || v == 4 || v == 8) ? v : 0;
  }();
  int v = forced ? forced : prefer ? prefer : (int)(16 / sizeof(R));
  if (sizeof(R) > 4 && v > 4) v = 4;  // 8 members per thread: FP32 only
  const size_t wide = sizeof(R) > sizeof(A) ? sizeof(R) : sizeof(A);
  for (; v > 1; v >>= 1) {
    if (B % v) continue;
    bool ok = true;
    for (const void *p : ptrs)
      if (p && ((uintptr_t)p % (v * wide))) ok = false;
    if (ok) break;
  }
  return v;
}

// run the statement with the compile-time member width VV equal to the runtime width v
// Staged edge kernels: blocks of epb = 256 / (B / V) edges (B / V threads each), used when the
// mesh has narrow bounds and a block holds at least two edges.  MPSW_STAGE=0 disables them.
inline bool stage_enabled() {
  static const bool on = !(std::getenv("MPSW_STAGE") && std::atoi(std::getenv("MPSW_STAGE")) == 0);
  return on;
}
// (and the block's stage fits the default 48 KB of dynamic shared memory)
template <typename R>
inline bool use_staged(const MeshDev<R> &m, int B, int v, size_t smem_per_edge_bytes, int block0 = 0) {
  const int tpe = B / v, bt = block0 ? block0 : block_threads();
  return stage_enabled() && m.max_eoe <= BoundsNarrow::e2 && m.max_eoc <= BoundsNarrow::c && tpe <= 128 &&
         tpe <= bt / 2 && smem_per_edge_bytes * (bt / tpe) <= 48 * 1024;
}

// the autotuned members-per-thread and block of a member kernel (0: default)
inline int tuned_v(KernelId k) { return g_tune ? g_tune->k[k].v : 0; }
inline int tuned_block(KernelId k) { return g_tune ? g_tune->k[k].block : 0; }
inline LaunchCfg staged_cfg(int n, int B, int v, size_t smem_per_edge_bytes, int block0 = 0) {
  const int tpe = B / v, epb = (block0 ? block0 : block_threads()) / tpe;
  return {(n + epb - 1) / epb, epb * tpe, smem_per_edge_bytes * epb};
}

// Width for the kernels measured faster at 8 FP32 members per thread (tl_edge_diag, ad_final):
// 0 (the default width) in FP64.
template <typename R>
constexpr int kWideV = sizeof(R) == 4 ? 8 : 0;

// run the statement with NB = BoundsNarrow when the mesh allows it, else BoundsAny
#define MPSW_BDISPATCH(m, ...)                                  \
  if ((m).max_eoe <= BoundsNarrow::e2 && (m).max_eoc <= BoundsNarrow::c) { \
    using NB = BoundsNarrow;                                    \
    __VA_ARGS__;                                                \
  } else {                                                      \
    using NB = BoundsAny;                                       \
    __VA_ARGS__;                                                \
  }

// run the statement once with NB = BoundsNarrow and once with NB = BoundsAny
#define MPSW_BDISPATCH_ALL(...)  \
  {                              \
    using NB = BoundsNarrow;     \
    __VA_ARGS__;                 \
  }                              \
  {                              \
    using NB = BoundsAny;        \
    __VA_ARGS__;                 \
  }

#define MPSW_VDISPATCH(v, ...)                            \
  switch (v) {                                            \
    case 8: { constexpr int VV = 8; if constexpr (sizeof(R) == 4) { __VA_ARGS__; } } break; \
    case 4: { constexpr int VV = 4; __VA_ARGS__; } break;  \
    case 2: { constexpr int VV = 2; __VA_ARGS__; } break;  \
    default: { constexpr int VV = 1; __VA_ARGS__; } break; \
  }

template <typename R, typename A>
void Launch<R, A>::fwd_vertex(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                              cudaStream_t s) {
  g_launches++;
  launch_k(k_fwd_vertex<R>, launch_cfg(m.nV), s, m, u, h, off, d);
}
template <typename R, typename A>
void Launch<R, A>::fwd_cell(const MeshDev<R> &m, const int *c_nb, const R *u, const R *h, R off,
                            const Diag<R> &d, const RK<R, A> &rk, R *tend_h, cudaStream_t s) {
  g_launches++;
  MPSW_BDISPATCH(m, launch_k(k_fwd_cell<R, A, NB::c>, launch_cfg(m.nC), s, m, c_nb, u, h, off, d, rk, tend_h));
}
template <typename R, typename A>
void Launch<R, A>::fwd_edge_diag(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                                 const Phys<R> &ph, cudaStream_t s) {
  g_launches++;
  if (sizeof(R) == 4 && !d.v) throw std::invalid_argument("FP32 fwd_edge_diag needs rows for the PV flux in d.v");
  Diag<R> dd = d;
  if (!(ph.visc4 > R(0))) dd.dsq_u = nullptr;  // delsq_u only feeds the del4 term
  MPSW_BDISPATCH(m, launch_k(k_fwd_edge_diag<R, NB::e2>, launch_cfg(m.nE), s, m, u, h, off, dd, ph));
}
template <typename R, typename A>
void Launch<R, A>::del4_vc(const MeshDev<R> &m, int B, const R *dsq_u, R *dsq_vort, R *dsq_div,
                           cudaStream_t s) {
  g_launches++;
  const int v = vec_width<R, A>(B, {dsq_u, dsq_vort, dsq_div});
  MPSW_VDISPATCH(v, MPSW_BDISPATCH(m, launch_k(k_del4_vc<R, VV, NB>, launch_cfg((long long)(m.nV + m.nC) * ((B) / (VV))), s, m, B, dsq_u, dsq_vort, dsq_div)));
}
template <typename R, typename A>
void Launch<R, A>::fwd_edge_tend(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                                 const Phys<R> &ph, const RK<R, A> &rk, R *tend_u, cudaStream_t s) {
  g_launches++;
  if (sizeof(R) == 4 && !d.v) throw std::invalid_argument("FP32 fwd_edge_tend needs the PV-flux rows in d.v");
  MPSW_BDISPATCH(m, launch_k(k_fwd_edge_tend<R, A, NB::e2>, launch_cfg(m.nE), s, m, u, h, off, d, ph, rk, tend_u));
}
template <typename R, typename A>
void Launch<R, A>::tracer_stage(const MeshDev<R> &m, const int *c_nb, int nT, const R *u, const R *he,
                                const R *tr_in, R *tr0, const R *h0, const R *h_next, R *tend, R *acc, R *tr_next,
                                R c, R w, int first, int last, cudaStream_t s) {
  g_launches++;
  MPSW_BDISPATCH(m, launch_k(k_tracer_stage<R, NB::c>, launch_cfg((long long)nT * m.nC), s, m, c_nb, nT, u, he, tr_in,
                             tr0, h0, h_next, tend, acc, tr_next, c, w, first, last));
}
template <typename R, typename A>
cudaError_t Launch<R, A>::preload_forward() {
  cudaFuncAttributes fa;
  cudaError_t err = cudaSuccess;
  auto load = [&](const void *k) {
    const cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (err == cudaSuccess) err = e;
  };
  load((const void *)k_fwd_vertex<R>);
  MPSW_BDISPATCH_ALL(load((const void *)k_fwd_cell<R, A, NB::c>); load((const void *)k_fwd_edge_diag<R, NB::e2>);
                     load((const void *)k_fwd_edge_tend<R, A, NB::e2>); load((const void *)k_del4_vc<R, 1, NB>));
  return err;
}
template <typename R, typename A>
void Launch<R, A>::tend_h(const MeshDev<R> &m, const R *u, const R *he, R *out, cudaStream_t s) {
  g_launches++;
  launch_k(k_tend_h<R>, launch_cfg(m.nC), s, m, u, he, out);
}
template <typename R, typename A>
void Launch<R, A>::recon(const MeshDev<R> &m, int B, int sphere, const R *u, R *X, R *Y, R *Z, R *Zon,
                         R *Mer, cudaStream_t s) {
  g_launches++;
  launch_k(k_recon<R>, launch_cfg((long long)m.nC * B), s, m, B, sphere, u, X, Y, Z, Zon, Mer);
}
template <typename R, typename A>
void Launch<R, A>::tl_vertex(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                             const Diag<R> &d, cudaStream_t s) {
  g_launches++;
  const int v = vec_width<R, A>(B, {ut, ht, d.circ, d.vort, d.hv, d.pvv}, tuned_v(K_TL_VERTEX));
  const int bk = tuned_block(K_TL_VERTEX);
  if (use_staged(m, B, v, vertex_stage_bytes<R>(), bk)) {
    MPSW_VDISPATCH(v, launch_k(tl_vertex_st_kernel<R, VV>(), staged_cfg(m.nV, B, VV, vertex_stage_bytes<R>(), bk), s, m, B,
                               bs, ut, ht, d));
    return;
  }
  MPSW_VDISPATCH(v, (launch_k(k_tl_vertex<R, VV>, launch_cfg((long long)(m.nV) * ((B) / (VV)), bk), s, m, B, bs, ut, ht, d)));
}
template <typename R, typename A>
void Launch<R, A>::tl_cell(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                           const Diag<R> &d, const RK<R, A> &rk, R *tend_h, cudaStream_t s) {
  g_launches++;
  const int v = vec_width<R, A>(B, {ut, ht, d.div, d.ke, d.pc, d.vc, d.pvv, d.vort, tend_h, rk.x0, rk.acc_in,
                                    rk.acc_out, rk.next, rk.t_out, rk.t_in[0], rk.t_in[1], rk.t_in[2], rk.x0r},
                                tuned_v(K_TL_CELL));
  const int bk = tuned_block(K_TL_CELL);
  if (use_staged(m, B, v, cell_stage_bytes<R>(), bk)) {
    MPSW_VDISPATCH(v, launch_k(tl_cell_st_kernel<R, A, VV>(), staged_cfg(m.nC, B, VV, cell_stage_bytes<R>(), bk), s, m, B,
                               bs, ut, ht, d, rk, tend_h, (int)g_stable_base));
    return;
  }
  MPSW_VDISPATCH(v, MPSW_BDISPATCH(m, launch_k(k_tl_cell<R, A, VV, NB>, launch_cfg((long long)(m.nC) * ((B) / (VV)), bk), s, m, B, bs, ut, ht, d, rk, tend_h)));
}
template <typename R, typename A>
void Launch<R, A>::tl_edge_diag(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                                const Diag<R> &d, const Phys<R> &ph, cudaStream_t s) {
  g_launches++;
  if (sizeof(R) == 4 && !d.v) throw std::invalid_argument("FP32 tl_edge_diag needs rows for the PV flux in d.v");
  Diag<R> dd = d;
  if (!(ph.visc4 > R(0))) dd.dsq_u = nullptr;  // delsq_u only feeds the del4 term
  const int v = vec_width<R, A>(B, {ut, ht, dd.pvv, dd.pc, dd.div, dd.vort, dd.pe, dd.he, dd.v, dd.gpt, dd.gpn, dd.dsq_u},
                                tuned_v(K_TL_EDGE_DIAG) ? tuned_v(K_TL_EDGE_DIAG) : kWideV<R>);
  const int bk = tuned_block(K_TL_EDGE_DIAG);
  constexpr int J = BoundsNarrow::e2;
  constexpr size_t eb = eoe_stage_bytes<R, J, 1, 0>();
  if (use_staged(m, B, v, eb, bk)) {
    MPSW_VDISPATCH(v, launch_k(tl_edge_diag_st_kernel<R, VV, J>(), staged_cfg(m.nE, B, VV, eb, bk), s, m, B, bs, ut, ht, dd, ph, (int)g_stable_base));
    return;
  }
  MPSW_VDISPATCH(v, MPSW_BDISPATCH(m, launch_k(k_tl_edge_diag<R, VV, NB>, launch_cfg((long long)(m.nE) * ((B) / (VV)), bk), s, m, B, bs, ut, ht, dd, ph)));
}
template <typename R, typename A>
void Launch<R, A>::tl_edge_tend(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                                const Diag<R> &d, const Phys<R> &ph, const RK<R, A> &rk, R *tend_u,
                                cudaStream_t s) {
  g_launches++;
  if (sizeof(R) == 4 && !d.v) throw std::invalid_argument("FP32 tl_edge_tend needs the PV-flux rows in d.v");
  const int v = vec_width<R, A>(B, {ut, ht, d.pe, d.he, d.v, d.ke, d.div, d.vort, d.dsq_div, d.dsq_vort, tend_u,
                                    rk.x0, rk.acc_in, rk.acc_out, rk.next, rk.t_out, rk.t_in[0], rk.t_in[1],
                                    rk.t_in[2], rk.x0r},
                                tuned_v(K_TL_EDGE_TEND));
  const int bk = tuned_block(K_TL_EDGE_TEND);
  constexpr int J = BoundsNarrow::e2;
  constexpr size_t eb = eoe_stage_bytes<R, J, 1, 3>();
  if (use_staged(m, B, v, eb, bk)) {
    MPSW_VDISPATCH(v, launch_k(tl_edge_tend_st_kernel<R, A, VV, J>(), staged_cfg(m.nE, B, VV, eb, bk),
                               s, m, B, bs, ut, ht, d, ph, rk, tend_u, (int)g_stable_base));
    return;
  }
  MPSW_VDISPATCH(v, MPSW_BDISPATCH(m, launch_k(k_tl_edge_tend<R, A, VV, NB>, launch_cfg((long long)(m.nE) * ((B) / (VV)), bk), s, m, B, bs, ut, ht, d, ph, rk, tend_u)));
}
// members per thread of one adjoint stage: every buffer the five kernels touch
template <typename R, typename A>
static int ad_width(int B, const AdIn<R> &in, const AdWork<R> &w, const AdOut<R, A> &out, int prefer = 0) {
  return vec_width<R, A>(B, {in.tu, in.th, w.pe_ad, w.he_ad, w.ud, w.gpn_ad, w.gpt_ad, w.v_ad, w.du_ad, w.pc_ad,
                             w.ke_ad, w.div_ad, w.hd, w.dd_ad, w.hv_ad, w.circ_ad, w.dc_ad, out.acc_u, out.acc_h,
                             out.x2u, out.x2h, out.dst_u, out.dst_h, out.tu_next, out.th_next, out.pad_out_u,
                             out.pad_out_h, out.pad_in_u[0], out.pad_in_u[1], out.pad_in_u[2], out.pad_in_h[0],
                             out.pad_in_h[1], out.pad_in_h[2], out.x2r_u, out.x2r_h},
                         prefer);
}

// preferred members per thread of adjoint kernel `which` (0 edge, 1 cell, 2 vertex, 3 final,
// 4-5 del4): the autotuned width, else 8 for ad_final in FP32, else the default
template <typename R>
inline int ad_prefer(int which) {
  static const KernelId ids[4] = {K_AD_EDGE, K_AD_CELL, K_AD_VERTEX, K_AD_FINAL};
  if (which < 4 && tuned_v(ids[which])) return tuned_v(ids[which]);
  return which == 3 ? kWideV<R> : 0;
}

template <typename R, typename A, int V, class NB>
static void ad_launch(int which, const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                      const AdIn<R> &in, const AdSeeds<R> &sd, const AdWork<R> &w, const AdOut<R, A> &out,
                      cudaStream_t s) {
  g_launches++;
  switch (which) {
    case 0: {
      constexpr int J = BoundsNarrow::e2;
      constexpr size_t eb = eoe_stage_bytes<R, J, 2, 3>();
      const int bk = tuned_block(K_AD_EDGE);
      if (use_staged(m, B, V, eb, bk))
        launch_k(ad_edge_st_kernel<R, A, V, J>(), staged_cfg(m.nE, B, V, eb, bk), s, m, B, bs, ph, in, sd, w, (int)g_stable_base);
      else
        launch_k(k_ad_edge<R, A, V, NB>, launch_cfg((long long)(m.nE) * ((B) / (V)), bk), s, m, B, bs, ph, in, sd, w);
      break;
    }
    case 1: {
      const int bk = tuned_block(K_AD_CELL);
      if (use_staged(m, B, V, ad_cell_stage_bytes<R>(), bk))
        launch_k(ad_cell_st_kernel<R, A, V>(), staged_cfg(m.nC, B, V, ad_cell_stage_bytes<R>(), bk), s, m, B, bs, ph, in, sd,
                 w, (int)g_stable_base);
      else
        launch_k(k_ad_cell<R, A, V, NB>, launch_cfg((long long)(m.nC) * ((B) / (V)), bk), s, m, B, bs, ph, in, sd, w);
      break;
    }
    case 2: {
      const int bk = tuned_block(K_AD_VERTEX);
      if (use_staged(m, B, V, ad_vertex_stage_bytes<R>(), bk))
        launch_k(ad_vertex_st_kernel<R, A, V>(), staged_cfg(m.nV, B, V, ad_vertex_stage_bytes<R>(), bk), s, m, B, bs, ph, in,
                 sd, w);
      else
        launch_k(k_ad_vertex<R, A, V>, launch_cfg((long long)(m.nV) * ((B) / (V)), bk), s, m, B, bs, ph, in, sd, w);
      break;
    }
    case 3: {
      constexpr int J = BoundsNarrow::e2;
      constexpr size_t eb = eoe_stage_bytes<R, J, 2, 1>();
      const int bk = tuned_block(K_AD_FINAL);
      if (use_staged(m, B, V, eb, bk)) {
        LaunchCfg c = staged_cfg(m.nE, B, V, eb, bk);
        const long long cthreads = (long long)m.nC * (B / V);
        const int cell_blocks = (int)((cthreads + c.block - 1) / c.block);
        c.grid += cell_blocks;
        launch_k(ad_final_st_kernel<R, A, V, J>(), c, s, m, B, bs, ph, w, out, cell_blocks, (int)g_stable_base);
      } else {
        launch_k(k_ad_final<R, A, V, NB>, launch_cfg((long long)(m.nC + m.nE) * ((B) / (V)), bk), s, m, B, bs, ph, w, out);
      }
      break;
    }
    case 4: launch_k(k_ad_del4_vc<R, V, NB>, launch_cfg((long long)(m.nV + m.nC) * ((B) / (V))), s, m, B, ph, in, w); break;
    default: launch_k(k_ad_del4_e<R, V>, launch_cfg((long long)(m.nE) * ((B) / (V))), s, m, B, w); break;
  }
}

template <typename R, typename A>
void Launch<R, A>::ad_stage(const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                            const AdIn<R> &in, const AdSeeds<R> &sd, const AdWork<R> &w,
                            const AdOut<R, A> &out, cudaStream_t s) {
  // each kernel at its own width (autotuned, else the default; ad_final defaults wider)
  auto one = [&](int which) {
    const int vk = ad_width<R, A>(B, in, w, out, ad_prefer<R>(which));
    MPSW_VDISPATCH(vk, MPSW_BDISPATCH(m, ad_launch<R, A, VV, NB>(which, m, B, bs, ph, in, sd, w, out, s)));
  };
  one(0);
  if (ph.visc4 > R(0)) {
    one(4);
    one(5);
  }
  one(1);
  one(2);
  one(3);
}
template <typename R, typename A>
void Launch<R, A>::ad_part(int which, const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                           const AdIn<R> &in, const AdWork<R> &w, const AdOut<R, A> &out,
                           cudaStream_t s) {
  const AdSeeds<R> sd{};
  const int k = which < 0 || which > 3 ? 3 : which;
  const int vk = ad_width<R, A>(B, in, w, out, ad_prefer<R>(k));
  MPSW_VDISPATCH(vk, MPSW_BDISPATCH(m, ad_launch<R, A, VV, NB>(k, m, B, bs, ph, in, sd, w, out, s)));
}
// Chunks of M members one fused-stage block walks (all B / M of its tile by default; fewer
// blocks per tile take more chunks each, so the tile's blob is staged fewer times).
// MPSW_FUSED_CPB overrides it when it divides B / M.
inline int fused_smem_index(int M) { return M == 32 ? 3 : M == 16 ? 2 : M == 8 ? 1 : 0; }
inline int fused_cpb(int B, int M) {
  const int chunks = B / M;
  const char *e = std::getenv("MPSW_FUSED_CPB");
  const int v = e ? std::atoi(e) : 0;
  return v > 0 && chunks % v == 0 ? v : chunks;
}
template <typename R, typename A>
bool Launch<R, A>::fused_ok(const FusedDev &f, int B, const Phys<R> &ph, int M) {
  constexpr bool f32 = std::is_same<R, float>::value && std::is_same<A, double>::value;
  if (!f32 || !f.ok || (M != 4 && M != 8 && M != 16 && M != 32) || B % M) return false;
  if (ph.visc2 > R(0) || ph.visc4 > R(0) || ph.wind || ph.drag) return false;
  if (M == 32 && f.nt == 256) return false;  // 32 members per chunk: 512- or 1024-thread blocks
  const int i = fused_smem_index(M);
  return f.tl.smem[i] <= kFusedSmemMax && f.ad.smem[i] <= kFusedSmemMax;
}

// run the statement with compile-time MM (members per chunk) and NN (threads per block)
#define MPSW_FUSED_DISPATCH(M, NT, ...)                                                       \
  switch ((M) * 10000 + (NT)) {                                                               \
    case 40256: { constexpr int MM = 4, NN = 256; __VA_ARGS__; } break;                       \
    case 40512: { constexpr int MM = 4, NN = 512; __VA_ARGS__; } break;                       \
    case 41024: { constexpr int MM = 4, NN = 1024; __VA_ARGS__; } break;                      \
    case 80256: { constexpr int MM = 8, NN = 256; __VA_ARGS__; } break;                       \
    case 80512: { constexpr int MM = 8, NN = 512; __VA_ARGS__; } break;                       \
    case 81024: { constexpr int MM = 8, NN = 1024; __VA_ARGS__; } break;                      \
    case 160256: { constexpr int MM = 16, NN = 256; __VA_ARGS__; } break;                     \
    case 160512: { constexpr int MM = 16, NN = 512; __VA_ARGS__; } break;                     \
    case 161024: { constexpr int MM = 16, NN = 1024; __VA_ARGS__; } break;                    \
    case 320512: { constexpr int MM = 32, NN = 512; __VA_ARGS__; } break;                     \
    case 321024: { constexpr int MM = 32, NN = 1024; __VA_ARGS__; } break;                    \
    default: throw std::invalid_argument("fused stage: unsupported members per chunk or block size"); \
  }

template <typename R, typename A>
cudaError_t Launch<R, A>::fused_prepare(const FusedDev &f) {
  if constexpr (std::is_same<R, float>::value && std::is_same<A, double>::value) {
    cudaError_t err = cudaSuccess;
    auto raise = [&](const void *k, size_t bytes) {
      if (bytes > kFusedSmemMax) return;
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (err == cudaSuccess) err = e;
    };
    for (int M : {4, 8, 16, 32}) {
      if (M == 32 && f.nt == 256) continue;
      const int i = fused_smem_index(M);
      MPSW_FUSED_DISPATCH(M, f.nt, raise((const void *)k_tl_fused<MM, NN>, f.tl.smem[i]);
                          raise((const void *)k_ad_fused<MM, NN>, f.ad.smem[i]));
    }
    return err;
  } else {
    (void)f;
    return cudaSuccess;
  }
}
template <typename R, typename A>
void Launch<R, A>::tl_fused(const FusedDev &f, int M, const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut,
                            const R *ht, const Phys<R> &ph, const RK<R, A> &rku, const RK<R, A> &rkh,
                            cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value && std::is_same<A, double>::value) {
    (void)m;
    if (!fused_ok(f, B, ph, M)) throw std::invalid_argument("fused tangent-linear stage not available here");
    g_launches++;
    const float a = ph.apvm * ph.dt;
    const int cpb = fused_cpb(B, M), i = fused_smem_index(M);
    const LaunchCfg c{f.tl.ntiles * ((B / M) / cpb), f.nt, f.tl.smem[i]};
    MPSW_FUSED_DISPATCH(M, f.nt, launch_k(k_tl_fused<MM, NN>, c, s, f.tl, B, cpb, bs, ut, ht, a, rku, rkh, ph.bad,
                                          (int)g_stable_base));
  } else {
    throw std::invalid_argument("fused stages run FP32 members only");
  }
}
template <typename R, typename A>
void Launch<R, A>::ad_fused(const FusedDev &f, int M, const MeshDev<R> &m, int B, const Base<R> &bs,
                            const Phys<R> &ph, const AdIn<R> &in, const AdOut<R, A> &out, cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value && std::is_same<A, double>::value) {
    (void)m;
    if (!fused_ok(f, B, ph, M)) throw std::invalid_argument("fused adjoint stage not available here");
    g_launches++;
    const float a = ph.apvm * ph.dt;
    const int cpb = fused_cpb(B, M), i = fused_smem_index(M);
    const LaunchCfg c{f.ad.ntiles * ((B / M) / cpb), f.nt, f.ad.smem[i]};
    MPSW_FUSED_DISPATCH(M, f.nt, launch_k(k_ad_fused<MM, NN>, c, s, f.ad, B, cpb, bs, a, in, out, ph.bad,
                                          (int)g_stable_base));
  } else {
    throw std::invalid_argument("fused stages run FP32 members only");
  }
}
template <typename R, typename A>
void Launch<R, A>::ad_tinit(const MeshDev<R> &m, int B, const A *x2u, const A *x2h, const R *seed_tu,
                            const R *seed_th, A wu, A wh, R *tu, R *th, cudaStream_t s) {
  g_launches++;
  const int v = vec_width<R, A>(B, {x2u, x2h, tu, th});
  MPSW_VDISPATCH(v, (launch_k(k_ad_tinit<R, A, VV>, launch_cfg((long long)(m.nE + m.nC) * ((B) / (VV))), s, m, B, x2u, x2h, seed_tu, seed_th,
                                                                                wu, wh, tu, th)));
}
template <typename R, typename A>
void Launch<R, A>::recon_adj(const MeshDev<R> &m, int sphere, R *Xa, R *Ya, R *Za, R *Zoa, R *Mea,
                             A *u_ad, cudaStream_t s) {
  g_launches++;
  launch_k(k_recon_adj_cell<R>, launch_cfg(m.nC), s, m, sphere, Xa, Ya, Za, Zoa, Mea);
  g_launches++;
  launch_k(k_recon_adj_edge<R, A>, launch_cfg(m.nE), s, m, Xa, Ya, Za, u_ad);
}
template <typename R, typename A>
void Launch<R, A>::to_internal(int n, int B, const int *perm, const double *src, R *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_to_internal<double, R>, launch_cfg((long long)n * B), s, n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_reference(int n, int B, const int *perm, const R *src, double *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_to_reference<R, double>, launch_cfg((long long)n * B), s, n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_internal_acc(int n, int B, const int *perm, const double *src, A *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_to_internal<double, A>, launch_cfg((long long)n * B), s, n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_reference_acc(int n, int B, const int *perm, const A *src, double *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_to_reference<A, double>, launch_cfg((long long)n * B), s, n, B, perm, src, dst);
}

}  // namespace mpsw
