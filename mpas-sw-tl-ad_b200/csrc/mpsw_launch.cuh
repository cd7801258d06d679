// Definitions of the launchers declared in mpsw_launch.h (included by one translation unit
// per precision, which also instantiates them).
#pragma once

#include "mpsw_kernels.cuh"
#include "mpsw_launch.h"

namespace mpsw {

constexpr int kThreads = 256;

// Grid and block for `total` threads: 256-thread blocks, halved (down to 64) while that leaves
// fewer than two blocks per SM, so thin single-trajectory launches still spread over all SMs.
struct LaunchCfg {
  int grid, block;
};
inline LaunchCfg launch_cfg(long long total) {
  int block = kThreads;
  while (block > 64 && total < 2LL * 148 * block) block >>= 1;
  long long g = (total + block - 1) / block;
  const long long cap = 148LL * 16 * (kThreads / block);
  if (g < 1) g = 1;
  return {(int)(g < cap ? g : cap), block};
}
#define LCFG(total) launch_cfg(total).grid, launch_cfg(total).block

// every kernel launch of the engine goes through one of these launchers and is counted here
extern long long g_launches;

template <typename R, typename A>
void Launch<R, A>::fwd_vertex(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                              cudaStream_t s) {
  g_launches++;
  k_fwd_vertex<R><<<LCFG(m.nV), 0, s>>>(m, u, h, off, d);
}
template <typename R, typename A>
void Launch<R, A>::fwd_cell(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                            const RK<R, A> &rk, R *tend_h, cudaStream_t s) {
  g_launches++;
  k_fwd_cell<R, A><<<LCFG(m.nC), 0, s>>>(m, u, h, off, d, rk, tend_h);
}
template <typename R, typename A>
void Launch<R, A>::fwd_edge_diag(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                                 const Phys<R> &ph, cudaStream_t s) {
  g_launches++;
  k_fwd_edge_diag<R><<<LCFG(m.nE), 0, s>>>(m, u, h, off, d, ph);
}
template <typename R, typename A>
void Launch<R, A>::del4_vc(const MeshDev<R> &m, int B, const R *dsq_u, R *dsq_vort, R *dsq_div,
                           cudaStream_t s) {
  g_launches++;
  k_del4_vc<R><<<LCFG((long long)(m.nV + m.nC) * B), 0, s>>>(m, B, dsq_u, dsq_vort, dsq_div);
}
template <typename R, typename A>
void Launch<R, A>::fwd_edge_tend(const MeshDev<R> &m, const R *u, const R *h, R off, const Diag<R> &d,
                                 const Phys<R> &ph, const RK<R, A> &rk, R *tend_u, cudaStream_t s) {
  g_launches++;
  k_fwd_edge_tend<R, A><<<LCFG(m.nE), 0, s>>>(m, u, h, off, d, ph, rk, tend_u);
}
template <typename R, typename A>
void Launch<R, A>::tend_h(const MeshDev<R> &m, const R *u, const R *he, R *out, cudaStream_t s) {
  g_launches++;
  k_tend_h<R><<<LCFG(m.nC), 0, s>>>(m, u, he, out);
}
template <typename R, typename A>
void Launch<R, A>::recon(const MeshDev<R> &m, int B, int sphere, const R *u, R *X, R *Y, R *Z, R *Zon,
                         R *Mer, cudaStream_t s) {
  g_launches++;
  k_recon<R><<<LCFG((long long)m.nC * B), 0, s>>>(m, B, sphere, u, X, Y, Z, Zon, Mer);
}
template <typename R, typename A>
void Launch<R, A>::tl_vertex(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                             const Diag<R> &d, cudaStream_t s) {
  g_launches++;
  k_tl_vertex<R><<<LCFG((long long)m.nV * B), 0, s>>>(m, B, bs, ut, ht, d);
}
template <typename R, typename A>
void Launch<R, A>::tl_cell(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                           const Diag<R> &d, const RK<R, A> &rk, R *tend_h, cudaStream_t s) {
  g_launches++;
  k_tl_cell<R, A><<<LCFG((long long)m.nC * B), 0, s>>>(m, B, bs, ut, ht, d, rk, tend_h);
}
template <typename R, typename A>
void Launch<R, A>::tl_edge_diag(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                                const Diag<R> &d, const Phys<R> &ph, cudaStream_t s) {
  g_launches++;
  k_tl_edge_diag<R><<<LCFG((long long)m.nE * B), 0, s>>>(m, B, bs, ut, ht, d, ph);
}
template <typename R, typename A>
void Launch<R, A>::tl_edge_tend(const MeshDev<R> &m, int B, const Base<R> &bs, const R *ut, const R *ht,
                                const Diag<R> &d, const Phys<R> &ph, const RK<R, A> &rk, R *tend_u,
                                cudaStream_t s) {
  g_launches++;
  k_tl_edge_tend<R, A><<<LCFG((long long)m.nE * B), 0, s>>>(m, B, bs, ut, ht, d, ph, rk, tend_u);
}
template <typename R, typename A>
void Launch<R, A>::ad_stage(const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                            const AdIn<R> &in, const AdSeeds<R> &sd, const AdWork<R> &w,
                            const AdOut<R, A> &out, cudaStream_t s) {
  g_launches++;
  k_ad_edge<R, A><<<LCFG((long long)m.nE * B), 0, s>>>(m, B, bs, ph, in, sd, w);
  if (ph.visc4 > R(0)) {
    g_launches++;
    k_ad_del4_vc<R, A><<<LCFG((long long)(m.nV + m.nC) * B), 0, s>>>(m, B, ph, in, w);
    g_launches++;
    k_ad_del4_e<R><<<LCFG((long long)m.nE * B), 0, s>>>(m, B, w);
  }
  g_launches++;
  k_ad_cell<R, A><<<LCFG((long long)m.nC * B), 0, s>>>(m, B, bs, ph, in, sd, w);
  g_launches++;
  k_ad_vertex<R, A><<<LCFG((long long)m.nV * B), 0, s>>>(m, B, bs, ph, in, sd, w);
  g_launches++;
  k_ad_final<R, A><<<LCFG((long long)(m.nC + m.nE) * B), 0, s>>>(m, B, bs, w, out);
}
template <typename R, typename A>
void Launch<R, A>::ad_part(int which, const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                           const AdIn<R> &in, const AdWork<R> &w, const AdOut<R, A> &out,
                           cudaStream_t s) {
  const AdSeeds<R> sd{};
  g_launches++;
  switch (which) {
    case 0: k_ad_edge<R, A><<<LCFG((long long)m.nE * B), 0, s>>>(m, B, bs, ph, in, sd, w); break;
    case 1: k_ad_cell<R, A><<<LCFG((long long)m.nC * B), 0, s>>>(m, B, bs, ph, in, sd, w); break;
    case 2: k_ad_vertex<R, A><<<LCFG((long long)m.nV * B), 0, s>>>(m, B, bs, ph, in, sd, w); break;
    default: k_ad_final<R, A><<<LCFG((long long)(m.nC + m.nE) * B), 0, s>>>(m, B, bs, w, out); break;
  }
}
template <typename R, typename A>
void Launch<R, A>::ad_tinit(const MeshDev<R> &m, int B, const A *x2u, const A *x2h, const R *seed_tu,
                            const R *seed_th, A wu, A wh, R *tu, R *th, cudaStream_t s) {
  g_launches++;
  k_ad_tinit<R, A><<<LCFG((long long)(m.nE + m.nC) * B), 0, s>>>(m, B, x2u, x2h, seed_tu,
                                                                             seed_th, wu, wh, tu, th);
}
template <typename R, typename A>
void Launch<R, A>::recon_adj(const MeshDev<R> &m, int sphere, R *Xa, R *Ya, R *Za, R *Zoa, R *Mea,
                             A *u_ad, cudaStream_t s) {
  g_launches++;
  k_recon_adj_cell<R><<<LCFG(m.nC), 0, s>>>(m, sphere, Xa, Ya, Za, Zoa, Mea);
  g_launches++;
  k_recon_adj_edge<R, A><<<LCFG(m.nE), 0, s>>>(m, Xa, Ya, Za, u_ad);
}
template <typename R, typename A>
void Launch<R, A>::to_internal(int n, int B, const int *perm, const double *src, R *dst, cudaStream_t s) {
  g_launches++;
  k_to_internal<double, R><<<LCFG((long long)n * B), 0, s>>>(n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_reference(int n, int B, const int *perm, const R *src, double *dst, cudaStream_t s) {
  g_launches++;
  k_to_reference<R, double><<<LCFG((long long)n * B), 0, s>>>(n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_internal_acc(int n, int B, const int *perm, const double *src, A *dst, cudaStream_t s) {
  g_launches++;
  k_to_internal<double, A><<<LCFG((long long)n * B), 0, s>>>(n, B, perm, src, dst);
}
template <typename R, typename A>
void Launch<R, A>::to_reference_acc(int n, int B, const int *perm, const A *src, double *dst, cudaStream_t s) {
  g_launches++;
  k_to_reference<A, double><<<LCFG((long long)n * B), 0, s>>>(n, B, perm, src, dst);
}

}  // namespace mpsw
