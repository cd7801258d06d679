// Host-side launchers of the stencil kernels, one instantiation per precision.  The FP64
// instantiation lives in a translation unit compiled with --fmad=false (bit-identical to the
// reference arithmetic), the FP32 one in a unit compiled with contraction allowed.
#pragma once

#include <cuda_runtime.h>

#include "mpsw_internal.h"

namespace mpsw {

extern long long g_launches;

// Launch choices of the member kernels, picked per (precision, B) by the window's autotuner:
// members per thread and threads per block (0: the default choice).
enum KernelId {
  K_TL_VERTEX, K_TL_CELL, K_TL_EDGE_DIAG, K_TL_EDGE_TEND, K_AD_EDGE, K_AD_CELL, K_AD_VERTEX, K_AD_FINAL,
  K_TUNED
};
struct TuneCfg {
  int v = 0, block = 0;
};
struct TuneTable {
  TuneCfg k[K_TUNED];
};
// The table the launchers of the calling thread follow (null: defaults); set for the duration
// of a sweep by TuneScope.
extern thread_local const TuneTable *g_tune;
struct TuneScope {
  const TuneTable *prev;
  explicit TuneScope(const TuneTable *t) : prev(g_tune) { g_tune = t; }
  ~TuneScope() { g_tune = prev; }
};

// Set while launching a sweep in which no kernel writes the mesh or the linearisation points
// (sweeps over stored stages): the staged kernels then copy their neighbour lists into shared
// memory before waiting for the previous kernel, overlapping that copy with its tail.
extern thread_local bool g_stable_base;
struct StableBaseScope {
  bool prev;
  explicit StableBaseScope(bool on) : prev(g_stable_base) { g_stable_base = on; }
  ~StableBaseScope() { g_stable_base = prev; }
};

template <typename R, typename A>
struct Launch {
  // forward stage pieces (single trajectory)
  static void fwd_vertex(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d, cudaStream_t s);
  static void fwd_cell(const MeshDev<R> &m, const int *c_nb, const R *u, const R *h, R off, const Diag<R> &d,
                       const RK<R, A> &rk, R *tend_h, cudaStream_t s);
  static void fwd_edge_diag(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                            const Phys<R> &ph, cudaStream_t s);
  static void del4_vc(const MeshDev<R> &m, int B, const R *dsq_u, R *dsq_vort, R *dsq_div, cudaStream_t s);
  static void fwd_edge_tend(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                            const Phys<R> &ph, const RK<R, A> &rk, R *tend_u, cudaStream_t s);
  static void tend_h(const MeshDev<R> &m, const R *u, const R *he, R *out, cudaStream_t s);
  static void tracer_stage(const MeshDev<R> &m, const int *c_nb, int nT, const R *u, const R *he, const R *tr_in,
                           R *tr0, const R *h0, const R *h_next, R *tend, R *acc, R *tr_next, R c, R w, int first,
                           int last, cudaStream_t s);
  static void recon(const MeshDev<R> &m, int B, int sphere, const R *u, R *X, R *Y, R *Z, R *Zon,
                    R *Mer, cudaStream_t s);
  // load the single-trajectory stage kernels (fwd_vertex .. fwd_edge_tend, del4_vc) onto the
  // current device now, instead of at their first launch (lazy module loading)
  static cudaError_t preload_forward();
  // tangent linear, B members
  static void tl_vertex(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                        const Diag<R> &d, cudaStream_t s);
  static void tl_cell(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                      const Diag<R> &d, const RK<R, A> &rk, R *tend_h, cudaStream_t s);
  static void tl_edge_diag(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                           const Diag<R> &d, const Phys<R> &ph, cudaStream_t s);
  static void tl_edge_tend(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                           const Diag<R> &d, const Phys<R> &ph, const RK<R, A> &rk, R *tend_u,
                           cudaStream_t s);
  // adjoint of one stage, B members
  static void ad_stage(const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                       const AdIn<R> &in, const AdSeeds<R> &sd, const AdWork<R> &w,
                       const AdOut<R, A> &out, cudaStream_t s);
  // one kernel of ad_stage (0 edge, 1 cell, 2 vertex, 3 final), for timing
  static void ad_part(int which, const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                      const AdIn<R> &in, const AdWork<R> &w, const AdOut<R, A> &out, cudaStream_t s);
  // Fused member stages (FP32 members only; mpsw_fused.cuh): one kernel for a whole
  // tangent-linear or adjoint stage, M = 4 or 8 members per block.  The physics must be the
  // default (no viscosity, drag or wind) and the seeds empty; fused_ok() tells.
  static bool fused_ok(const FusedDev &f, int B, const Phys<R> &ph, int M);
  static void tl_fused(const FusedDev &f, int M, const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut,
                       const R *ht, const Phys<R> &ph, const RK<R, A> &rku, const RK<R, A> &rkh, cudaStream_t s);
  static void ad_fused(const FusedDev &f, int M, const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                       const AdIn<R> &in, const AdOut<R, A> &out, cudaStream_t s);
  // raise the fused kernels' dynamic shared-memory limit to what the tiles need
  static cudaError_t fused_prepare(const FusedDev &f);
  static void ad_tinit(const MeshDev<R> &m, int B, const A *x2u, const A *x2h, const R *seed_tu,
                       const R *seed_th, A wu, A wh, R *tu, R *th, cudaStream_t s);
  static void recon_adj(const MeshDev<R> &m, int sphere, R *Xa, R *Ya, R *Za, R *Zoa, R *Mea, A *u_ad,
                        cudaStream_t s);
  // boundary
  static void to_internal(int n, int B, const int *perm, const double *src, R *dst, cudaStream_t s);
  static void to_reference(int n, int B, const int *perm, const R *src, double *dst, cudaStream_t s);
  static void to_internal_acc(int n, int B, const int *perm, const double *src, A *dst, cudaStream_t s);
  static void to_reference_acc(int n, int B, const int *perm, const A *src, double *dst, cudaStream_t s);
};

void convert_d2f(long long n, const double *src, float *dst, cudaStream_t s);
void convert_d2f_off(long long n, const double *src, double off, float *dst, cudaStream_t s);
void convert_list(const ConvList &L, long long max_n, cudaStream_t s);
void convert_f2d(long long n, const float *src, double *dst, cudaStream_t s);

}  // namespace mpsw
