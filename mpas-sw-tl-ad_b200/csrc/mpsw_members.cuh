// Member kernels: tangent linear and adjoint of the RK4 stages for B members about one stored
// linearisation point, and the del4 intermediates.
//
// Member arrays are [n][B]; each thread holds V consecutive members of one entity (Mv<R,V>)
// and moves them with vector loads, so the connectivity, weights and linearisation-point
// values of a neighbour are loaded once for V independent accumulation chains.  Every
// member's arithmetic is the scalar expression of the reference, element by element, so V
// does not change a single rounding (V = 1 is the single-member module path).
#pragma once

#include <cstdlib>

#include "mpsw_kernels.cuh"

namespace mpsw {

// Register caps of the staged member kernels at 8 FP32 members per thread (the form the
// autotuner picks on large meshes): each kernel X has a second form k_X_rc held to
// MPSW_REGS_X registers, which X_kernel() selects for R = float, V = 8; 0 keeps the compiler's
// own choice.  The values are the measured optimum on the level-7 mesh (occupancy against
// in-flight loads per thread).
// MPSW_REGCAP=0 launches the compiler's register choice instead (to measure the caps on other
// meshes without a rebuild).
inline bool regcap_on() {
  static const bool on = !(std::getenv("MPSW_REGCAP") && std::atoi(std::getenv("MPSW_REGCAP")) == 0);
  return on;
}
#ifndef MPSW_REGS_TL_VERTEX
#define MPSW_REGS_TL_VERTEX 32
#endif
#ifndef MPSW_REGS_TL_CELL
#define MPSW_REGS_TL_CELL 72
#endif
#ifndef MPSW_REGS_TL_EDGE_DIAG
#define MPSW_REGS_TL_EDGE_DIAG 64
#endif
#ifndef MPSW_REGS_TL_EDGE_TEND
#define MPSW_REGS_TL_EDGE_TEND 64
#endif
#ifndef MPSW_REGS_AD_EDGE
#define MPSW_REGS_AD_EDGE 56
#endif
#ifndef MPSW_REGS_AD_CELL
#define MPSW_REGS_AD_CELL 72
#endif
#ifndef MPSW_REGS_AD_VERTEX
#define MPSW_REGS_AD_VERTEX 0
#endif
#ifndef MPSW_REGS_AD_FINAL
#define MPSW_REGS_AD_FINAL 40
#endif

// ---- V members of one entity -------------------------------------------------------------
template <typename R, int V>
struct alignas(sizeof(R) * V) Mv {
  R x[V];
};

#define MPSW_MV_OP(op)                                                                            \
  template <typename R, int V>                                                                  \
  __device__ __forceinline__ Mv<R, V> operator op(const Mv<R, V> &a, const Mv<R, V> &b) {       \
    Mv<R, V> r;                                                                                 \
    _Pragma("unroll") for (int i = 0; i < V; i++) r.x[i] = a.x[i] op b.x[i];                    \
    return r;                                                                                   \
  }                                                                                             \
  template <typename R, int V>                                                                  \
  __device__ __forceinline__ Mv<R, V> operator op(R a, const Mv<R, V> &b) {                     \
    Mv<R, V> r;                                                                                 \
    _Pragma("unroll") for (int i = 0; i < V; i++) r.x[i] = a op b.x[i];                         \
    return r;                                                                                   \
  }                                                                                             \
  template <typename R, int V>                                                                  \
  __device__ __forceinline__ Mv<R, V> operator op(const Mv<R, V> &a, R b) {                     \
    Mv<R, V> r;                                                                                 \
    _Pragma("unroll") for (int i = 0; i < V; i++) r.x[i] = a.x[i] op b;                         \
    return r;                                                                                   \
  }
MPSW_MV_OP(+)
MPSW_MV_OP(-)
MPSW_MV_OP(*)
MPSW_MV_OP(/)
#undef MPSW_MV_OP

template <typename R, int V>
__device__ __forceinline__ Mv<R, V> operator-(const Mv<R, V> &a) {
  Mv<R, V> r;
#pragma unroll
  for (int i = 0; i < V; i++) r.x[i] = -a.x[i];
  return r;
}

template <typename R, int V>
__device__ __forceinline__ Mv<R, V> mv_fill(R a) {
  Mv<R, V> r;
#pragma unroll
  for (int i = 0; i < V; i++) r.x[i] = a;
  return r;
}

// vector load / store of V consecutive members (the offset is a multiple of V)
template <int V, typename R>
__device__ __forceinline__ Mv<R, V> ldv(const R *p) {
  return *reinterpret_cast<const Mv<R, V> *>(p);
}
template <int V, typename R>
__device__ __forceinline__ void stv(R *p, const Mv<R, V> &v) {
  *reinterpret_cast<Mv<R, V> *>(p) = v;
}

template <int V, typename D, typename S>
__device__ __forceinline__ Mv<D, V> mv_cast(const Mv<S, V> &a) {
  Mv<D, V> r;
#pragma unroll
  for (int i = 0; i < V; i++) r.x[i] = D(a.x[i]);
  return r;
}

// thread t -> (entity, first member)
#define MPSW_MEMBER_LOOP(t, n, B, V)                                      \
  MPSW_GRID_LOOP(t, (long long)(n) * ((B) / (V)))

struct EntMember {
  int ent, b;
};
__device__ __forceinline__ EntMember ent_member(long long t, int B, int V) {
  const int bv = B / V;
  const int ent = (int)(t / bv);
  return {ent, (int)(t - (long long)ent * bv) * V};
}

// RK4 bookkeeping of V members (src/mpas_sw_module.f90:590-611)
template <typename R, typename A, int V>
__device__ __forceinline__ void rk_members(const RK<R, A> &rk, size_t o, const Mv<R, V> &t) {
  const bool last = rk.t_in[0] != nullptr;  // the stage that sums the stored tendencies
  if (rk.next && !last) {
    Mv<R, V> n;
    if (rk.x0r) {
      const Mv<R, V> x = ldv<V>(rk.x0r + o);
      const R c = R(rk.c);
#pragma unroll
      for (int i = 0; i < V; i++) n.x[i] = x.x[i] + c * t.x[i];
    } else {
      const Mv<A, V> x0 = ldv<V>(rk.x0 + o);
#pragma unroll
      for (int i = 0; i < V; i++) n.x[i] = rk.frozen ? R(x0.x[i]) : R(x0.x[i] + rk.c * A(t.x[i]));
    }
    stv<V>(rk.next + o, n);
  }
  if (rk.frozen) return;
  if (rk.t_out) {
    stv<V>(rk.t_out + o, t);
  } else if (rk.t_in[0]) {
    Mv<A, V> a = ldv<V>(rk.x0 + o);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const Mv<R, V> tj = ldv<V>(rk.t_in[j] + o);
#pragma unroll
      for (int i = 0; i < V; i++) a.x[i] = a.x[i] + rk.wt[j] * A(tj.x[i]);
    }
#pragma unroll
    for (int i = 0; i < V; i++) a.x[i] = a.x[i] + rk.w * A(t.x[i]);
    stv<V>(rk.acc_out + o, a);
    if (rk.next) stv<V>(rk.next + o, mv_cast<V, R>(a));  // the next step's rounded stage-1 input
  } else if (rk.acc_out) {
    Mv<A, V> a = ldv<V>(rk.acc_in + o);
#pragma unroll
    for (int i = 0; i < V; i++) a.x[i] = a.x[i] + rk.w * A(t.x[i]);
    stv<V>(rk.acc_out + o, a);
  }
}

// del4 intermediates (src/mpas_sw_dyncore.f90:554-589): delsq_vorticity on vertices and
// delsq_divergence on cells.  One grid covers the vertex threads followed by the cell threads.
template <typename R, int V, class NB>
__global__ void k_del4_vc(MeshDev<R> m, int B, const R *__restrict__ dsq_u, R *dsq_vort, R *dsq_div) {
  using M = Mv<R, V>;
  const int nV = m.nV, nC = m.nC;
  const long long tv = (long long)nV * (B / V);
  MPSW_GRID_LOOP(t, tv + (long long)nC * (B / V)) {
    if (t < tv) {
      const EntMember q = ent_member(t, B, V);
      const int v = q.ent;
      M dcirc = mv_fill<R, V>(R(0));
#pragma unroll
      for (int k = 0; k < VDEG; k++) {
        const int e = ld(m.v_es, (size_t)k * nV + v);
        const R s = R(m.v_esg[(size_t)k * nV + v]);
        dcirc = dcirc + s * (ld(m.e_dc, e) * ldv<V>(dsq_u + (size_t)e * B + q.b));
      }
      stv<V>(dsq_vort + (size_t)v * B + q.b, dcirc * (R(1) / ld(m.v_area, v)));
    } else {
      const EntMember q = ent_member(t - tv, B, V);
      const int c = q.ent;
      const int n = ld(m.c_n, c);
      M dd = mv_fill<R, V>(R(0));
      MPSW_SLOTS(k, NB::c, n) {
        const int e = ld(m.c_es, (size_t)k * nC + c);
        const R s = R(m.c_esg[(size_t)k * nC + c]);
        dd = dd + s * (ldv<V>(dsq_u + (size_t)e * B + q.b) * ld(m.e_dv, e));
      }
      stv<V>(dsq_div + (size_t)c * B + q.b, dd * (R(1) / ld(m.c_area, c)));
    }
  }
}

// ---- edgesOnEdge lists ------------------------------------------------------------------
// The edge kernels read the edgesOnEdge list of their edge through an accessor: slot j gives the
// neighbour edge nb(j), weightsOnEdge w(j), its transpose wr(j) and linearisation-point fields at
// the neighbour f(k, j).  EoeGlobal reads them from global memory; EoeShared from a block's
// shared-memory copy (stage_eoe), so the member loads of every slot take their addresses from
// shared memory instead of waiting on an index load from global memory.  Both give the same
// values, so a kernel body computes the same numbers with either.
template <typename R>
struct EoeGlobal {
  const int *eoe;
  const R *wv, *wrv;
  const R *fld[3];
  int nE, e;
  __device__ int nb(int j) const { return ld(eoe, (size_t)j * nE + e); }
  __device__ R w(int j) const { return ld(wv, (size_t)j * nE + e); }
  __device__ R wr(int j) const { return ld(wrv, (size_t)j * nE + e); }
  __device__ R f(int k, int j) const { return ld(fld[k], nb(j)); }
  static constexpr bool kPadded = false;  // slots at or past nEdgesOnEdge must not be read
};
template <typename R>
__device__ __forceinline__ EoeGlobal<R> eoe_global(const MeshDev<R> &m, int e, const R *f0 = nullptr,
                                                   const R *f1 = nullptr, const R *f2 = nullptr) {
  EoeGlobal<R> g;
  g.eoe = m.e_eoe;
  g.wv = m.e_w;
  g.wrv = m.e_wrev;
  g.fld[0] = f0;
  g.fld[1] = f1;
  g.fld[2] = f2;
  g.nE = m.nE;
  g.e = e;
  return g;
}

template <typename R>
struct EoeShared {
  const int *snb;
  const R *sw, *swr, *sf;
  int le, epb, J;
  __device__ int at(int j) const { return j * epb + le; }
  __device__ int nb(int j) const { return snb[at(j)]; }
  __device__ R w(int j) const { return sw[at(j)]; }
  __device__ R wr(int j) const { return swr[at(j)]; }
  __device__ R f(int k, int j) const { return sf[(size_t)k * J * epb + at(j)]; }
  // Slots at or past nEdgesOnEdge hold neighbour 0 with zero weights and fields: every term of
  // such a slot is an exact zero, so a body may run all J slots without a bound check.
  static constexpr bool kPadded = true;
};

// Shared-memory bytes per edge of a stage with HW weights arrays (0-2) and NF fields.
template <typename R, int J, int HW, int NF>
constexpr size_t eoe_stage_bytes() {
  return (size_t)J * (sizeof(int) + (HW + NF) * sizeof(R));
}

// Copy the lists of edges e0 .. e0 + epb - 1 into shared memory (weights: e_w if HW >= 1, e_wrev
// if HW == 2; fields[k] at the neighbours) with coalesced slot-major loads spread over the block,
// then __syncthreads.  Every thread of the block must call it; le selects the caller's edge.
template <typename R, int J, int HW, int NF>
__device__ EoeShared<R> stage_eoe(const MeshDev<R> &m, int e0, int epb, int le, const R *const *fields) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sw = reinterpret_cast<R *>(smem_raw);
  R *swr = sw + (HW >= 1 ? (size_t)J * epb : 0);
  R *sf = swr + (HW >= 2 ? (size_t)J * epb : 0);
  int *snb = reinterpret_cast<int *>(sf + (size_t)NF * J * epb);
  const int nE = m.nE;
  for (int i = threadIdx.x; i < J * epb; i += blockDim.x) {
    const int j = i / epb, l = i - j * epb, e = e0 + l;
    int nb = 0;
    R w = R(0), wr = R(0);
    R f[NF > 0 ? NF : 1];
#pragma unroll
    for (int k = 0; k < NF; k++) f[k] = R(0);
    if (e < nE && j < ld(m.e_n, e)) {
      nb = ld(m.e_eoe, (size_t)j * nE + e);
      if (HW >= 1) w = ld(m.e_w, (size_t)j * nE + e);
      if (HW >= 2) wr = ld(m.e_wrev, (size_t)j * nE + e);
#pragma unroll
      for (int k = 0; k < NF; k++) f[k] = ld(fields[k], nb);
    }
    snb[i] = nb;
    if (HW >= 1) sw[i] = w;
    if (HW >= 2) swr[i] = wr;
#pragma unroll
    for (int k = 0; k < NF; k++) sf[(size_t)k * J * epb + i] = f[k];
  }
  __syncthreads();
  EoeShared<R> st;
  st.snb = snb;
  st.sw = sw;
  st.swr = swr;
  st.sf = sf;
  st.le = le;
  st.epb = epb;
  st.J = J;
  return st;
}

// The thread's edge and first member in a staged edge kernel (blocks of epb edges with B / V
// threads each); false for threads past the last edge.
__device__ __forceinline__ bool staged_edge(int nE, int B, int V, int *le, int *e, int *b) {
  const int tpe = B / V;
  *le = threadIdx.x / tpe;
  *e = blockIdx.x * (blockDim.x / tpe) + *le;
  *b = (threadIdx.x - *le * tpe) * V;
  return *le < (int)(blockDim.x / tpe) && *e < nE;
}

// ----------------------------------------------------------------------------------------
// Tangent linear (src/mpas_sw_dyncore_tlm.f90)
// ----------------------------------------------------------------------------------------

// :255-271 and :344-360
template <typename R, int V>
__global__ void k_tl_vertex(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                            const R *__restrict__ ht, Diag<R> d) {
  using M = Mv<R, V>;
  const int nV = m.nV;
  MPSW_MEMBER_LOOP(t, nV, B, V) {
    const EntMember q = ent_member(t, B, V);
    const int v = q.ent;
    M circ = mv_fill<R, V>(R(0));
#pragma unroll
    for (int k = 0; k < VDEG; k++) {
      const int e = ld(m.v_es, (size_t)k * nV + v);
      const R s = R(m.v_esg[(size_t)k * nV + v]);
      circ = circ + s * (ld(m.e_dc, e) * ldv<V>(ut + (size_t)e * B + q.b));
    }
    const R area = ld(m.v_area, v);
    const M vort = circ / area;
    M hvt = mv_fill<R, V>(R(0));
#pragma unroll
    for (int k = 0; k < VDEG; k++)
      hvt = hvt + ldv<V>(ht + (size_t)ld(m.v_c, (size_t)k * nV + v) * B + q.b) * ld(m.v_k, (size_t)k * nV + v);
    hvt = hvt / area;
    const R hv = ld(bs.hv, v);
    const M pvt = vort / hv - (hvt * (ld(m.v_f, v) + ld(bs.vort, v))) / (hv * hv);
    const size_t o = (size_t)v * B + q.b;
    if (d.circ) stv<V>(d.circ + o, circ);
    if (d.vort) stv<V>(d.vort + o, vort);
    if (d.hv) stv<V>(d.hv + o, hvt);
    stv<V>(d.pvv + o, pvt);
  }
}

// Shared-memory bytes per vertex of k_tl_vertex_st's stage: 3 slots of 2 indices and 3 values.
template <typename R>
__host__ __device__ constexpr size_t vertex_stage_bytes() {
  return (size_t)VDEG * (2 * sizeof(int) + 3 * sizeof(R));
}

// k_tl_vertex with each block's vertex lists (edge, sign and dcEdge in the reference's scatter
// order; cell and kite) copied into shared memory before waiting for the previous kernel: they
// are mesh data, which no kernel writes.  Same operations as k_tl_vertex.
template <typename R, int V>
__device__ __forceinline__ void tl_vertex_st_run(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d) {
  using M = Mv<R, V>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nV = m.nV, tpe = B / V, vpb = blockDim.x / tpe;
  const int v0 = blockIdx.x * vpb;
  const size_t SV = (size_t)VDEG * vpb;
  R *ssg = reinterpret_cast<R *>(smem_raw), *sdc = ssg + SV, *skt = sdc + SV;  // [VDEG][vpb] each
  int *se = reinterpret_cast<int *>(skt + SV), *sc = se + SV;
  for (int i = threadIdx.x; i < VDEG * vpb; i += blockDim.x) {
    const int k = i / vpb, v = v0 + (i - k * vpb);
    int e = 0, c = 0;
    R sg = R(0), dc = R(0), kt = R(0);
    if (v < nV) {
      e = ld(m.v_es, (size_t)k * nV + v);
      sg = R(m.v_esg[(size_t)k * nV + v]);
      dc = ld(m.e_dc, e);
      c = ld(m.v_c, (size_t)k * nV + v);
      kt = ld(m.v_k, (size_t)k * nV + v);
    }
    ssg[i] = sg; sdc[i] = dc; skt[i] = kt; se[i] = e; sc[i] = c;
  }
  __syncthreads();
  pdl_begin();
  const int lv = threadIdx.x / tpe, v = v0 + lv;
  if (lv >= vpb || v >= nV) return;
  const int b = (threadIdx.x - lv * tpe) * V;
  M circ = mv_fill<R, V>(R(0));
#pragma unroll
  for (int k = 0; k < VDEG; k++) {
    const int i = k * vpb + lv;
    circ = circ + ssg[i] * (sdc[i] * ldv<V>(ut + (size_t)se[i] * B + b));
  }
  const R area = ld(m.v_area, v);
  M hvt = mv_fill<R, V>(R(0));
#pragma unroll
  for (int k = 0; k < VDEG; k++) {
    const int i = k * vpb + lv;
    hvt = hvt + ldv<V>(ht + (size_t)sc[i] * B + b) * skt[i];
  }
  const R hv = ld(bs.hv, v);
  M vort, pvt;
  if constexpr (sizeof(R) == 4) {
    // FP32 members: reciprocals of areaTriangle and h_vertex formed once per vertex
    const R ra = R(1) / area, rh = R(1) / hv;
    vort = circ * ra;
    hvt = hvt * ra;
    pvt = vort * rh - hvt * (((ld(m.v_f, v) + ld(bs.vort, v)) * rh) * rh);
  } else {
    vort = circ / area;
    hvt = hvt / area;
    pvt = vort / hv - (hvt * (ld(m.v_f, v) + ld(bs.vort, v))) / (hv * hv);
  }
  const size_t o = (size_t)v * B + b;
  if (d.circ) stv<V>(d.circ + o, circ);
  if (d.vort) stv<V>(d.vort + o, vort);
  if (d.hv) stv<V>(d.hv + o, hvt);
  stv<V>(d.pvv + o, pvt);
}
template <typename R, int V>
__global__ void k_tl_vertex_st(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d) {
  tl_vertex_st_run<R, V>(m, B, bs, ut, ht, d);
}
#if MPSW_REGS_TL_VERTEX > 0
template <int V>
__global__ void __maxnreg__(MPSW_REGS_TL_VERTEX) k_tl_vertex_st_rc(MeshDev<float> m, int B, Base<float> bs, const float *__restrict__ ut,
                               const float *__restrict__ ht, Diag<float> d) {
  tl_vertex_st_run<float, V>(m, B, bs, ut, ht, d);
}
#endif
template <typename R, int V>
inline auto tl_vertex_st_kernel() {
#if MPSW_REGS_TL_VERTEX > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_tl_vertex_st_rc<V> : &k_tl_vertex_st<R, V>;
  else return &k_tl_vertex_st<R, V>;
#else
  return &k_tl_vertex_st<R, V>;
#endif
}

// :274-316, :397-421, thickness tendency :541-561 and the RK update.  In FP32 the kernel is held
// to 48 registers (5 blocks of 256 threads per SM), which measured faster than the 56 it takes
// otherwise.
template <typename R, typename A, int V, class NB>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1) k_tl_cell(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                          const R *__restrict__ ht, Diag<R> d, RK<R, A> rk, R *tend_h) {
  using M = Mv<R, V>;
  const int nC = m.nC;
  MPSW_MEMBER_LOOP(t, nC, B, V) {
    const EntMember q = ent_member(t, B, V);
    const int c = q.ent;
    const int n = ld(m.c_n, c);
    M div = mv_fill<R, V>(R(0)), th = mv_fill<R, V>(R(0));
    MPSW_SLOTS(k, NB::c, n) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R s = R(m.c_esg[(size_t)k * nC + c]);
      const M ue = ldv<V>(ut + (size_t)e * B + q.b);
      const R dve = ld(m.e_dv, e);
      div = div + s * (ue * dve);
      const M het = R(0.5) * (ldv<V>(ht + (size_t)ld(m.e_c1, e) * B + q.b) +
                              ldv<V>(ht + (size_t)ld(m.e_c2, e) * B + q.b));
      const M flux = (ue * dve) * ld(bs.he, e) + (ld(bs.u, e) * dve) * het;
      th = th + (-s) * flux;
    }
    const R area = ld(m.c_area, c);
    div = div * (R(1) / area);
    M ke = mv_fill<R, V>(R(0));
    MPSW_SLOTS(i, NB::c, n) {
      const int e = ld(m.c_eoc, (size_t)i * nC + c);
      ke = ke + ((R(0.25) * ld(m.e_dc, e)) * ld(m.e_dv, e)) * ((R(2) * ld(bs.u, e)) * ldv<V>(ut + (size_t)e * B + q.b));
    }
    ke = ke / area;
    M pc = mv_fill<R, V>(R(0)), vc = mv_fill<R, V>(R(0));
    MPSW_SLOTS(k, NB::c, n) {
      const int v = ld(m.c_vs, (size_t)k * nC + c);
      const R kt = ld(m.c_vk, (size_t)k * nC + c);
      pc = pc + (kt * ldv<V>(d.pvv + (size_t)v * B + q.b)) / area;
      if (d.vc) vc = vc + (kt * ldv<V>(d.vort + (size_t)v * B + q.b)) / area;
    }
    th = th / area;
    const size_t o = (size_t)c * B + q.b;
    if (d.div) stv<V>(d.div + o, div);
    stv<V>(d.ke + o, ke);
    stv<V>(d.pc + o, pc);
    if (d.vc) stv<V>(d.vc + o, vc);
    if (tend_h) stv<V>(tend_h + o, th);
    rk_members<R, A, V>(rk, o, th);
  }
}

// Shared-memory bytes per cell of tl_cell_st's stage: 6 slots of 4 indices and 7 coefficients.
template <typename R>
__host__ __device__ constexpr size_t cell_stage_bytes() {
  return (size_t)BoundsNarrow::c * (4 * sizeof(int) + 7 * sizeof(R));
}

// k_tl_cell with each block's cell lists staged in shared memory (meshes with at most 6
// edgesOnCell): per slot the edge (reference scatter order) and its sign, the cell across it,
// dvEdge, the linearisation point's h_edge and u there, the edgesOnCell edge with its two ke
// coefficients, and the vertex with its kite.  The member loads then take their addresses from
// shared memory, and h at the cell itself is loaded once (h_edge is the same sum in either
// order).  Slots past the cell's edge count hold index 0 with zero coefficients, so every term
// there is an exact zero and all 6 slots run without a bound check.  early: copy the lists
// before waiting for the previous kernel.
template <typename R, typename A, int V>
__device__ __forceinline__ void tl_cell_st_run(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                                               const R *__restrict__ ht, Diag<R> d, RK<R, A> rk, R *tend_h,
                                               int early) {
  using M = Mv<R, V>;
  constexpr int S = BoundsNarrow::c;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (!early) pdl_begin();
  const int nC = m.nC, tpe = B / V, cpb = blockDim.x / tpe;
  const int c0 = blockIdx.x * cpb;
  R *sr = reinterpret_cast<R *>(smem_raw);  // [7][S][cpb]
  int *si = reinterpret_cast<int *>(sr + (size_t)7 * S * cpb);  // [4][S][cpb]
  const size_t SC = (size_t)S * cpb;
  for (int i = threadIdx.x; i < S * cpb; i += blockDim.x) {
    const int k = i / cpb, lc = i - k * cpb, c = c0 + lc;
    int e = 0, nb = 0, eo = 0, v = 0;
    R sg = R(0), dve = R(0), heb = R(0), ub = R(0), k1 = R(0), k2 = R(0), kt = R(0);
    if (c < nC && k < ld(m.c_n, c)) {
      e = ld(m.c_es, (size_t)k * nC + c);
      sg = R(m.c_esg[(size_t)k * nC + c]);
      const int c1 = ld(m.e_c1, e);
      nb = c1 == c ? ld(m.e_c2, e) : c1;
      dve = ld(m.e_dv, e);
      heb = ld(bs.he, e);
      ub = ld(bs.u, e);
      // FP32 members take ke's terms in the scatter order, from the same edge loads
      eo = sizeof(R) == 4 ? e : ld(m.c_eoc, (size_t)k * nC + c);
      k1 = (R(0.25) * ld(m.e_dc, eo)) * ld(m.e_dv, eo);
      k2 = R(2) * ld(bs.u, eo);
      v = ld(m.c_vs, (size_t)k * nC + c);
      kt = ld(m.c_vk, (size_t)k * nC + c);
    }
    sr[0 * SC + i] = sg; sr[1 * SC + i] = dve; sr[2 * SC + i] = heb; sr[3 * SC + i] = ub;
    sr[4 * SC + i] = k1; sr[5 * SC + i] = k2; sr[6 * SC + i] = kt;
    si[0 * SC + i] = e; si[1 * SC + i] = nb; si[2 * SC + i] = eo; si[3 * SC + i] = v;
  }
  __syncthreads();
  if (early) pdl_begin();
  const int lc = threadIdx.x / tpe, c = c0 + lc;
  if (lc >= cpb || c >= nC) return;
  const int b = (threadIdx.x - lc * tpe) * V;
  const M htc = ldv<V>(ht + (size_t)c * B + b);
  M div = mv_fill<R, V>(R(0)), th = mv_fill<R, V>(R(0)), ke = mv_fill<R, V>(R(0));
  MPSW_SLOTS(k, S, S) {
    const int i = k * cpb + lc;
    const R s = sr[0 * SC + i], dve = sr[1 * SC + i];
    const M ue = ldv<V>(ut + (size_t)si[0 * SC + i] * B + b);
    div = div + s * (ue * dve);
    const M het = R(0.5) * (htc + ldv<V>(ht + (size_t)si[1 * SC + i] * B + b));
    const M flux = (ue * dve) * sr[2 * SC + i] + (sr[3 * SC + i] * dve) * het;
    th = th + (-s) * flux;
    if constexpr (sizeof(R) == 4) ke = ke + sr[4 * SC + i] * (sr[5 * SC + i] * ue);
  }
  const R area = ld(m.c_area, c);
  div = div * (R(1) / area);
  if constexpr (sizeof(R) != 4) {
    MPSW_SLOTS(k, S, S) {
      const int i = k * cpb + lc;
      ke = ke + sr[4 * SC + i] * (sr[5 * SC + i] * ldv<V>(ut + (size_t)si[2 * SC + i] * B + b));
    }
  }
  M pc = mv_fill<R, V>(R(0)), vc = mv_fill<R, V>(R(0));
  if constexpr (sizeof(R) == 4) {
    // FP32 members: 1 / areaCell formed once, no division per member
    const R ra = R(1) / area;
    ke = ke * ra;
    MPSW_SLOTS(k, S, S) {
      const int i = k * cpb + lc;
      const int v = si[3 * SC + i];
      const R kr = sr[6 * SC + i] * ra;
      pc = pc + kr * ldv<V>(d.pvv + (size_t)v * B + b);
      if (d.vc) vc = vc + kr * ldv<V>(d.vort + (size_t)v * B + b);
    }
    th = th * ra;
  } else {
    ke = ke / area;
    MPSW_SLOTS(k, S, S) {
      const int i = k * cpb + lc;
      const int v = si[3 * SC + i];
      const R kt = sr[6 * SC + i];
      pc = pc + (kt * ldv<V>(d.pvv + (size_t)v * B + b)) / area;
      if (d.vc) vc = vc + (kt * ldv<V>(d.vort + (size_t)v * B + b)) / area;
    }
    th = th / area;
  }
  const size_t o = (size_t)c * B + b;
  if (d.div) stv<V>(d.div + o, div);
  stv<V>(d.ke + o, ke);
  stv<V>(d.pc + o, pc);
  if (d.vc) stv<V>(d.vc + o, vc);
  if (tend_h) stv<V>(tend_h + o, th);
  rk_members<R, A, V>(rk, o, th);
}
template <typename R, typename A, int V>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1)
    k_tl_cell_st(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut, const R *__restrict__ ht, Diag<R> d,
                 RK<R, A> rk, R *tend_h, int early) {
  tl_cell_st_run<R, A, V>(m, B, bs, ut, ht, d, rk, tend_h, early);
}
#if MPSW_REGS_TL_CELL > 0
// (without the 48-register bound of the other forms)
template <typename A, int V>
__global__ void __maxnreg__(MPSW_REGS_TL_CELL) k_tl_cell_st_rc(MeshDev<float> m, int B, Base<float> bs,
                                                              const float *__restrict__ ut,
                                                              const float *__restrict__ ht, Diag<float> d,
                                                              RK<float, A> rk, float *tend_h, int early) {
  tl_cell_st_run<float, A, V>(m, B, bs, ut, ht, d, rk, tend_h, early);
}
#endif
template <typename R, typename A, int V>
inline auto tl_cell_st_kernel() {
#if MPSW_REGS_TL_CELL > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_tl_cell_st_rc<A, V> : &k_tl_cell_st<R, A, V>;
  else return &k_tl_cell_st<R, A, V>;
#else
  return &k_tl_cell_st<R, A, V>;
#endif
}

// :319-329, :364-393, :425-445, h_edge_tl :117-126, delsq_u_tl :638-652.  Body for edge e,
// members b .. b+V-1; l is the edge's edgesOnEdge list.
template <typename R, int V, int NMAX, class L>
__device__ __forceinline__ void tl_edge_diag_body(const MeshDev<R> &m, int B, const Base<R> &bs,
                                                  const R *__restrict__ ut, const R *__restrict__ ht,
                                                  const Diag<R> &d, const Phys<R> &ph, int e, int b, const L &l) {
  using M = Mv<R, V>;
  const int n = ld(m.e_n, e);
  M vt = mv_fill<R, V>(R(0));
  MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n)
    vt = vt + l.w(j) * ldv<V>(ut + (size_t)l.nb(j) * B + b);
  const int v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e), c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
  const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
  const M pv1 = ldv<V>(d.pvv + (size_t)v1 * B + b), pv2 = ldv<V>(d.pvv + (size_t)v2 * B + b);
  // FP32 members: multiply by 1 / dvEdge, 1 / dcEdge instead of dividing each member
  const M gptt = sizeof(R) == 4 ? (pv2 - pv1) * (R(1) / dv) : (pv2 - pv1) / dv;
  // pv_edge's two vertex terms: the reference adds them over edgesOnVertex, which lists the same
  // two endpoints; a sum of two terms is the same in either order, so the loaded rows serve
  M pet = mv_fill<R, V>(R(0));
  pet = pet + R(0.5) * pv1;
  pet = pet + R(0.5) * pv2;
  pet = pet - ((ph.apvm * vt) * ph.dt) * ld(bs.gpt, e) - ((ph.apvm * ld(bs.v, e)) * ph.dt) * gptt;
  const M dpc = ldv<V>(d.pc + (size_t)c2 * B + b) - ldv<V>(d.pc + (size_t)c1 * B + b);
  const M gpnt = sizeof(R) == 4 ? dpc * (R(1) / dc) : dpc / dc;
  const M uet = ldv<V>(ut + (size_t)e * B + b);
  pet = pet - ((ph.apvm * uet) * ph.dt) * ld(bs.gpn, e) - ((ph.apvm * ld(bs.u, e)) * ph.dt) * gpnt;
  const size_t o = (size_t)e * B + b;
  stv<V>(d.pe + o, pet);
  const M het = R(0.5) * (ldv<V>(ht + (size_t)c1 * B + b) + ldv<V>(ht + (size_t)c2 * B + b));
  if constexpr (sizeof(R) == 4) {
    // FP32 members: the edge's tangent thickness flux (u h_edge)' in d.he and tangent PV flux
    // (u h_edge pv_edge)' in d.v, the two rows tl_edge_tend gathers at the neighbours
    const R ub = ld(bs.u, e), hb = ld(bs.he, e), pb = ld(bs.pe, e);
    stv<V>(d.he + o, uet * hb + ub * het);
    stv<V>(d.v + o, (uet * hb) * pb + (ub * hb) * pet + (ub * pb) * het);
  } else {
    stv<V>(d.he + o, het);
    if (d.v) stv<V>(d.v + o, vt);
  }
  if (d.gpt) stv<V>(d.gpt + o, gptt);
  if (d.gpn) stv<V>(d.gpn + o, gpnt);
  if (d.dsq_u)
    stv<V>(d.dsq_u + o, (ldv<V>(d.div + (size_t)c2 * B + b) - ldv<V>(d.div + (size_t)c1 * B + b)) / dc -
                            (ldv<V>(d.vort + (size_t)v2 * B + b) - ldv<V>(d.vort + (size_t)v1 * B + b)) / dv);
}

template <typename R, int V, class NB>
__global__ void k_tl_edge_diag(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d, Phys<R> ph) {
  MPSW_MEMBER_LOOP(t, m.nE, B, V) {
    const EntMember q = ent_member(t, B, V);
    tl_edge_diag_body<R, V, NB::e2>(m, B, bs, ut, ht, d, ph, q.ent, q.b, eoe_global(m, q.ent));
  }
}

template <typename R, int V, int J>
__device__ __forceinline__ void tl_edge_diag_st_run(const MeshDev<R> &m, int B, const Base<R> &bs,
                                                    const R *__restrict__ ut, const R *__restrict__ ht,
                                                    const Diag<R> &d, const Phys<R> &ph, int early) {
  if (!early) pdl_begin();
  int le, e, b;
  const bool mine = staged_edge(m.nE, B, V, &le, &e, &b);
  const int epb = blockDim.x / (B / V);
  const EoeShared<R> st = stage_eoe<R, J, 1, 0>(m, blockIdx.x * epb, epb, le, nullptr);
  if (early) pdl_begin();
  if (mine) tl_edge_diag_body<R, V, J>(m, B, bs, ut, ht, d, ph, e, b, st);
}
template <typename R, int V, int J>
__global__ void k_tl_edge_diag_st(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                                  const R *__restrict__ ht, Diag<R> d, Phys<R> ph, int early) {
  tl_edge_diag_st_run<R, V, J>(m, B, bs, ut, ht, d, ph, early);
}
#if MPSW_REGS_TL_EDGE_DIAG > 0
template <int V, int J>
__global__ void __maxnreg__(MPSW_REGS_TL_EDGE_DIAG) k_tl_edge_diag_st_rc(MeshDev<float> m, int B, Base<float> bs,
                                                                        const float *__restrict__ ut,
                                                                        const float *__restrict__ ht, Diag<float> d,
                                                                        Phys<float> ph, int early) {
  tl_edge_diag_st_run<float, V, J>(m, B, bs, ut, ht, d, ph, early);
}
#endif
template <typename R, int V, int J>
inline auto tl_edge_diag_st_kernel() {
#if MPSW_REGS_TL_EDGE_DIAG > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_tl_edge_diag_st_rc<V, J> : &k_tl_edge_diag_st<R, V, J>;
  else return &k_tl_edge_diag_st<R, V, J>;
#else
  return &k_tl_edge_diag_st<R, V, J>;
#endif
}

// sw_compute_tend_tlm normal-velocity part :564-768 and the RK update.  Body for edge e,
// members b .. b+V-1; l is the edge's edgesOnEdge list with fields pv_edge, u, h_edge.
template <typename R, typename A, int V, int NMAX, class L>
__device__ __forceinline__ void tl_edge_tend_body(const MeshDev<R> &m, int B, const Base<R> &bs,
                                                  const R *__restrict__ ut, const R *__restrict__ ht,
                                                  const Diag<R> &d, const Phys<R> &ph, const RK<R, A> &rk,
                                                  R *tend_u, int e, int b, const L &l) {
  using M = Mv<R, V>;
  const int n = ld(m.e_n, e);
  const M pet_e = ldv<V>(d.pe + (size_t)e * B + b);
  const R pe_e = ld(bs.pe, e);
  M qt = mv_fill<R, V>(R(0));
  if constexpr (sizeof(R) == 4) {
    // FP32 members: q' = 0.5 pv_edge(e) sum w (u h_edge)'_j + 0.5 sum w (u h_edge pv_edge)'_j
    //                  + 0.5 pv_edge'(e) sum w u_j h_edge_j, the same sum regrouped by the
    // neighbour fluxes tl_edge_diag leaves in d.he and d.v: two member rows per neighbour
    M f1 = mv_fill<R, V>(R(0)), f2 = mv_fill<R, V>(R(0));
    R sb = R(0);
    MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n) {
      const size_t on = (size_t)l.nb(j) * B + b;
      const R w = l.w(j);
      f1 = f1 + w * ldv<V>(d.he + on);
      f2 = f2 + w * ldv<V>(d.v + on);
      sb = sb + (w * l.f(1, j)) * l.f(2, j);
    }
    qt = (R(0.5) * pe_e) * f1 + R(0.5) * f2 + (R(0.5) * sb) * pet_e;
  } else {
    MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n) {
      const int eoe = l.nb(j);
      const R w = l.w(j);
      const M wpvt = R(0.5) * (pet_e + ldv<V>(d.pe + (size_t)eoe * B + b));
      const R wpv = R(0.5) * (pe_e + l.f(0, j));
      const R ub = l.f(1, j), heb = l.f(2, j);
      qt = qt + ((w * ldv<V>(ut + (size_t)eoe * B + b)) * wpv) * heb + ((w * ub) * wpvt) * heb +
           ((w * ub) * wpv) * ldv<V>(d.he + (size_t)eoe * B + b);
    }
  }
  const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e), v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e);
  const R dc = ld(m.e_dc, e), dv = ld(m.e_dv, e);
  const M grad = (ldv<V>(d.ke + (size_t)c2 * B + b) - ldv<V>(d.ke + (size_t)c1 * B + b)) +
                 R(GRAVITY) * (ldv<V>(ht + (size_t)c2 * B + b) - ldv<V>(ht + (size_t)c1 * B + b));
  // FP32 members: multiply by 1 / dcEdge instead of dividing each member
  M tut = sizeof(R) == 4 ? qt - grad * (R(1) / dc) : qt - grad / dc;
  if (ph.visc2 > R(0)) {
    M ud = (ldv<V>(d.div + (size_t)c2 * B + b) - ldv<V>(d.div + (size_t)c1 * B + b)) / dc -
           (ldv<V>(d.vort + (size_t)v2 * B + b) - ldv<V>(d.vort + (size_t)v1 * B + b)) / dv;
    ud = (ld(m.e_sc2, e) * ph.visc2) * ud;
    tut = tut + ud;
  }
  if (ph.visc4 > R(0)) {
    M ud = (ldv<V>(d.dsq_div + (size_t)c2 * B + b) - ldv<V>(d.dsq_div + (size_t)c1 * B + b)) / dc -
           (ldv<V>(d.dsq_vort + (size_t)v2 * B + b) - ldv<V>(d.dsq_vort + (size_t)v1 * B + b)) / dv;
    ud = (ld(m.e_sc4, e) * ph.visc4) * ud;
    tut = tut - ud;
  }
  const R hh = ld(bs.he, e);
  // h_edge' of the edge itself (d.he holds the thickness flux for FP32 members)
  const M het = R(0.5) * (ldv<V>(ht + (size_t)c1 * B + b) + ldv<V>(ht + (size_t)c2 * B + b));
  if (ph.wind) tut = tut - ((het * ld(m.e_usrc, e)) / R(RHO_REF)) / (hh * hh);
  if (ph.drag) {
    const M ket_e = R(0.5) * (ldv<V>(d.ke + (size_t)c1 * B + b) + ldv<V>(d.ke + (size_t)c2 * B + b));
    const R ke_e = R(0.5) * (ld(bs.ke, c1) + ld(bs.ke, c2));
    const R uu = ld(bs.u, e), sq = sqrt(R(2) * ke_e);
    tut = tut - ((R(1.0e-3) * ldv<V>(ut + (size_t)e * B + b)) * sq) / hh -
          ((((R(0.5) * R(1.0e-3)) * uu) * (R(2) * ket_e)) / sq) / hh +
          (((R(1.0e-3) * uu) * sq) * het) / (hh * hh);
  }
  const size_t o = (size_t)e * B + b;
  if (ph.bad) {
#pragma unroll
    for (int i = 0; i < V; i++) flag_nonfinite(ph.bad, tut.x[i]);
  }
  if (tend_u) stv<V>(tend_u + o, tut);
  rk_members<R, A, V>(rk, o, tut);
}

template <typename R, typename A, int V, class NB>
__global__ void k_tl_edge_tend(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d, Phys<R> ph, RK<R, A> rk,
                               R *tend_u) {
  MPSW_MEMBER_LOOP(t, m.nE, B, V) {
    const EntMember q = ent_member(t, B, V);
    tl_edge_tend_body<R, A, V, NB::e2>(m, B, bs, ut, ht, d, ph, rk, tend_u, q.ent, q.b,
                                       eoe_global(m, q.ent, bs.pe, bs.u, bs.he));
  }
}

// k_tl_edge_tend with the edgesOnEdge lists staged in shared memory: one block per epb edges.
// early: copy the lists before waiting for the previous kernel (g_stable_base).
template <typename R, typename A, int V, int J>
__device__ __forceinline__ void tl_edge_tend_st_run(const MeshDev<R> &m, int B, const Base<R> &bs,
                                                    const R *__restrict__ ut, const R *__restrict__ ht,
                                                    const Diag<R> &d, const Phys<R> &ph, const RK<R, A> &rk,
                                                    R *tend_u, int early) {
  if (!early) pdl_begin();
  int le, e, b;
  const bool mine = staged_edge(m.nE, B, V, &le, &e, &b);
  const int epb = blockDim.x / (B / V);
  const R *const fields[3] = {bs.pe, bs.u, bs.he};
  const EoeShared<R> st = stage_eoe<R, J, 1, 3>(m, blockIdx.x * epb, epb, le, fields);
  if (early) pdl_begin();
  if (mine) tl_edge_tend_body<R, A, V, J>(m, B, bs, ut, ht, d, ph, rk, tend_u, e, b, st);
}
template <typename R, typename A, int V, int J>
__global__ void k_tl_edge_tend_st(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                                  const R *__restrict__ ht, Diag<R> d, Phys<R> ph, RK<R, A> rk,
                                  R *tend_u, int early) {
  tl_edge_tend_st_run<R, A, V, J>(m, B, bs, ut, ht, d, ph, rk, tend_u, early);
}
#if MPSW_REGS_TL_EDGE_TEND > 0
template <typename A, int V, int J>
__global__ void __maxnreg__(MPSW_REGS_TL_EDGE_TEND) k_tl_edge_tend_st_rc(MeshDev<float> m, int B, Base<float> bs,
                                                                        const float *__restrict__ ut,
                                                                        const float *__restrict__ ht, Diag<float> d,
                                                                        Phys<float> ph, RK<float, A> rk,
                                                                        float *tend_u, int early) {
  tl_edge_tend_st_run<float, A, V, J>(m, B, bs, ut, ht, d, ph, rk, tend_u, early);
}
#endif
template <typename R, typename A, int V, int J>
inline auto tl_edge_tend_st_kernel() {
#if MPSW_REGS_TL_EDGE_TEND > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_tl_edge_tend_st_rc<A, V, J> : &k_tl_edge_tend_st<R, A, V, J>;
  else return &k_tl_edge_tend_st<R, A, V, J>;
#else
  return &k_tl_edge_tend_st<R, A, V, J>;
#endif
}

// ----------------------------------------------------------------------------------------
// Adjoint of one RK stage (src/mpas_sw_dyncore_adj.f90): sw_compute_tend_adj (:455-738)
// followed by sw_compute_solve_diagnostics_adj (:1-453) at the same linearisation point,
// as gathers over transposed connectivity; no atomics.
// ----------------------------------------------------------------------------------------

// Tendency adjoint of the last stage of a step (src/mpas_sw_module.f90:912-914 at rk=4):
// tu = wu * x2u + seed_tu, th = (wh * x2h + seed_th) / areaCell.  Edge threads then cell threads.
template <typename R, typename A, int V>
__global__ void k_ad_tinit(MeshDev<R> m, int B, const A *x2u, const A *x2h, const R *seed_tu,
                           const R *seed_th, A wu, A wh, R *tu, R *th) {
  const long long te = (long long)m.nE * (B / V);
  MPSW_GRID_LOOP(t, te + (long long)m.nC * (B / V)) {
    if (t < te) {
      const EntMember q = ent_member(t, B, V);
      const size_t o = (size_t)q.ent * B + q.b;
      Mv<R, V> r;
#pragma unroll
      for (int i = 0; i < V; i++) {
        A x = x2u ? wu * x2u[o + i] : A(0);
        if (seed_tu) x = x + A(seed_tu[q.ent]);
        r.x[i] = R(x);
      }
      stv<V>(tu + o, r);
    } else {
      const EntMember q = ent_member(t - te, B, V);
      const size_t o = (size_t)q.ent * B + q.b;
      const A area = A(ld(m.c_area, q.ent));
      Mv<R, V> r;
#pragma unroll
      for (int i = 0; i < V; i++) {
        A x = x2h ? wh * x2h[o + i] : A(0);
        if (seed_th) x = x + A(seed_th[q.ent]);
        r.x[i] = R(x / area);
      }
      stv<V>(th + o, r);
    }
  }
}

// Edge stage: workpv/q adjoint (:689-718) as a gather over the transposed edgesOnEdge,
// thickness-flux adjoint (:720-736), drag (:549-565), wind (:567-572), then the APVM adjoints
// of the diagnostics (:193-200, :235-242).
template <typename R, typename A, int V, int NMAX, class L>
__device__ __forceinline__ void ad_edge_body(const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                                             const AdIn<R> &in, const AdSeeds<R> &sd, const AdWork<R> &w, int e,
                                             int b, const L &l) {
  using M = Mv<R, V>;
  const int n = ld(m.e_n, e);
  const M Te = ldv<V>(in.tu + (size_t)e * B + b);
  const R ue = ld(bs.u, e), hee = ld(bs.he, e), pee = ld(bs.pe, e);
  M pe_ad = mv_fill<R, V>(R(0)), he_ad = mv_fill<R, V>(R(0)), ud = mv_fill<R, V>(R(0));
  if constexpr (sizeof(R) == 4) {
    // FP32 members: the same terms with the per-slot coefficients formed once per thread and
    // the edge's own tendency adjoint factored out of its sum
    R sq = R(0);
    MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n) {
      const R wr = l.wr(j), wru = wr * ue;
      const R wpv = R(0.5) * (l.f(2, j) + pee);
      const M Tn = ldv<V>(in.tu + (size_t)l.nb(j) * B + b);
      sq = sq + (l.w(j) * l.f(0, j)) * l.f(1, j);
      he_ad = he_ad + (wru * wpv) * Tn;
      pe_ad = pe_ad + (R(0.5) * (wru * hee)) * Tn;
      ud = ud + ((wr * wpv) * hee) * Tn;
    }
    pe_ad = pe_ad + (R(0.5) * sq) * Te;
  } else {
    MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n) {
      const int nb = l.nb(j);
      const R wj = l.w(j);
      const R wr = l.wr(j);
      pe_ad = pe_ad + R(0.5) * (((wj * l.f(0, j)) * l.f(1, j)) * Te);
      const M Tn = ldv<V>(in.tu + (size_t)nb * B + b);
      const R wpv = R(0.5) * (l.f(2, j) + pee);
      he_ad = he_ad + ((wr * ue) * wpv) * Tn;
      pe_ad = pe_ad + R(0.5) * (((wr * ue) * hee) * Tn);
      ud = ud + ((wr * wpv) * hee) * Tn;
    }
  }
  const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
  const R dv = ld(m.e_dv, e);
  const M fa = ldv<V>(in.th + (size_t)c2 * B + b) - ldv<V>(in.th + (size_t)c1 * B + b);
  he_ad = he_ad + (ue * dv) * fa;
  ud = ud + (dv * hee) * fa;
  if (ph.drag) {
    const R sq = sqrt(R(2) * (R(0.5) * (ld(bs.ke, c1) + ld(bs.ke, c2))));
    he_ad = he_ad + (((R(1.0e-3) * ue) * sq) / (hee * hee)) * Te;
    ud = ud - ((R(1.0e-3) * sq) / hee) * Te;
  }
  if (ph.wind) he_ad = he_ad - ((ld(m.e_usrc, e) / R(RHO_REF)) / (hee * hee)) * Te;
  M gpn_ad = mv_fill<R, V>(R(0)), gpt_ad = mv_fill<R, V>(R(0)), v_ad = mv_fill<R, V>(R(0));
  if (sd.pe) pe_ad = pe_ad + sd.pe[e];
  if (sd.he) he_ad = he_ad + sd.he[e];
  if (sd.gpn) gpn_ad = mv_fill<R, V>(sd.gpn[e]);
  if (sd.gpt) gpt_ad = mv_fill<R, V>(sd.gpt[e]);
  if (sd.v) v_ad = mv_fill<R, V>(sd.v[e]);
  gpn_ad = gpn_ad - ((ph.apvm * ue) * ph.dt) * pe_ad;
  ud = ud - ((ph.apvm * ph.dt) * ld(bs.gpn, e)) * pe_ad;
  gpt_ad = gpt_ad - ((ph.apvm * ld(bs.v, e)) * ph.dt) * pe_ad;
  v_ad = v_ad - ((ph.apvm * ph.dt) * ld(bs.gpt, e)) * pe_ad;
  const size_t o = (size_t)e * B + b;
  stv<V>(w.pe_ad + o, pe_ad);
  stv<V>(w.he_ad + o, he_ad);
  stv<V>(w.ud + o, ud);
  // without seeds the window sweeps leave these null: gradPVn_ad, gradPVt_ad and v_ad are then
  // re-formed from pv_edge_ad by their readers with these same expressions
  if (w.gpn_ad) stv<V>(w.gpn_ad + o, gpn_ad);
  if (w.gpt_ad) stv<V>(w.gpt_ad + o, gpt_ad);
  if (w.v_ad) stv<V>(w.v_ad + o, v_ad);
}

template <typename R, typename A, int V, class NB>
__global__ void k_ad_edge(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                          AdWork<R> w) {
  MPSW_MEMBER_LOOP(t, m.nE, B, V) {
    const EntMember q = ent_member(t, B, V);
    ad_edge_body<R, A, V, NB::e2>(m, B, bs, ph, in, sd, w, q.ent, q.b, eoe_global(m, q.ent, bs.u, bs.he, bs.pe));
  }
}

// k_ad_edge with the edgesOnEdge lists (both weights; u, h_edge, pv_edge at the neighbours)
// staged in shared memory: one block per epb edges.
template <typename R, typename A, int V, int J>
__device__ __forceinline__ void ad_edge_st_run(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                             AdWork<R> w, int early) {
  if (!early) pdl_begin();
  int le, e, b;
  const bool mine = staged_edge(m.nE, B, V, &le, &e, &b);
  const int epb = blockDim.x / (B / V);
  const R *const fields[3] = {bs.u, bs.he, bs.pe};
  const EoeShared<R> st = stage_eoe<R, J, 2, 3>(m, blockIdx.x * epb, epb, le, fields);
  if (early) pdl_begin();
  if (mine) ad_edge_body<R, A, V, J>(m, B, bs, ph, in, sd, w, e, b, st);
}
template <typename R, typename A, int V, int J>
__global__ void k_ad_edge_st(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                             AdWork<R> w, int early) {
  ad_edge_st_run<R, A, V, J>(m, B, bs, ph, in, sd, w, early);
}
#if MPSW_REGS_AD_EDGE > 0
template <typename A, int V, int J>
__global__ void __maxnreg__(MPSW_REGS_AD_EDGE) k_ad_edge_st_rc(MeshDev<float> m, int B, Base<float> bs, Phys<float> ph, AdIn<float> in, AdSeeds<float> sd,
                             AdWork<float> w, int early) {
  ad_edge_st_run<float, A, V, J>(m, B, bs, ph, in, sd, w, early);
}
#endif
template <typename R, typename A, int V, int J>
inline auto ad_edge_st_kernel() {
#if MPSW_REGS_AD_EDGE > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_ad_edge_st_rc<A, V, J> : &k_ad_edge_st<R, A, V, J>;
  else return &k_ad_edge_st<R, A, V, J>;
#else
  return &k_ad_edge_st<R, A, V, J>;
#endif
}

// del4 adjoint, first half (:588-634): delsq_vorticity/delsq_circulation adjoint on vertices
// and delsq_divergence adjoint on cells.
template <typename R, int V, class NB>
__global__ void k_ad_del4_vc(MeshDev<R> m, int B, Phys<R> ph, AdIn<R> in, AdWork<R> w) {
  using M = Mv<R, V>;
  const int nV = m.nV, nC = m.nC;
  const long long tv = (long long)nV * (B / V);
  MPSW_GRID_LOOP(t, tv + (long long)nC * (B / V)) {
    if (t < tv) {
      const EntMember q = ent_member(t, B, V);
      const int v = q.ent;
      M acc = mv_fill<R, V>(R(0));
#pragma unroll
      for (int k = 0; k < VDEG; k++) {
        const int e = ld(m.v_es, (size_t)k * nV + v);
        const R sg = R(m.v_esg[(size_t)k * nV + v]);
        const M ud4 = (ld(m.e_sc4, e) * ph.visc4) * (-ldv<V>(in.tu + (size_t)e * B + q.b));
        acc = acc + (-sg) * (ud4 / ld(m.e_dv, e));
      }
      stv<V>(w.dc_ad + (size_t)v * B + q.b, acc * (R(1) / ld(m.v_area, v)));
    } else {
      const EntMember q = ent_member(t - tv, B, V);
      const int c = q.ent;
      const int n = ld(m.c_n, c);
      M acc = mv_fill<R, V>(R(0));
      MPSW_SLOTS(k, NB::c, n) {
        const int e = ld(m.c_es, (size_t)k * nC + c);
        const R sg = R(m.c_esg[(size_t)k * nC + c]);
        const M ud4 = (ld(m.e_sc4, e) * ph.visc4) * (-ldv<V>(in.tu + (size_t)e * B + q.b));
        acc = acc + (-sg) * (ud4 / ld(m.e_dc, e));
      }
      stv<V>(w.dd_ad + (size_t)c * B + q.b, acc * (R(1) / ld(m.c_area, c)));
    }
  }
}

// del4 adjoint, second half (:617-643): delsq_u adjoint on edges.
template <typename R, int V>
__global__ void k_ad_del4_e(MeshDev<R> m, int B, AdWork<R> w) {
  using M = Mv<R, V>;
  const int nE = m.nE;
  MPSW_MEMBER_LOOP(t, nE, B, V) {
    const EntMember q = ent_member(t, B, V);
    const int e = q.ent;
    const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
    M du = mv_fill<R, V>(R(0));
    du = du - dv * ldv<V>(w.dd_ad + (size_t)ld(m.e_c2, e) * B + q.b);
    du = du + dv * ldv<V>(w.dd_ad + (size_t)ld(m.e_c1, e) * B + q.b);
    du = du + dc * ldv<V>(w.dc_ad + (size_t)ld(m.e_v2, e) * B + q.b);
    du = du - dc * ldv<V>(w.dc_ad + (size_t)ld(m.e_v1, e) * B + q.b);
    stv<V>(w.du_ad + (size_t)e * B + q.b, du);
  }
}

// Cell stage: gradPVn adjoint onto pv_cell (:202-213), gravity/ke terms of the tendency
// adjoint (:696-699), drag ke terms, del2/del4 divergence adjoints, h_edge adjoint (:358-369),
// then the 1/areaCell scalings of ke_ad and divergence_ad (:306-326).
template <typename R, typename A, int V, class NB>
__global__ void k_ad_cell(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                          AdWork<R> w) {
  using M = Mv<R, V>;
  const int nC = m.nC;
  MPSW_MEMBER_LOOP(t, nC, B, V) {
    const EntMember q = ent_member(t, B, V);
    const int c = q.ent;
    const int n = ld(m.c_n, c);
    M pc_ad = mv_fill<R, V>(sd.pc ? sd.pc[c] : R(0));
    M ke_ad = mv_fill<R, V>(sd.ke ? sd.ke[c] : R(0));
    M div_ad = mv_fill<R, V>(sd.div ? sd.div[c] : R(0));
    M hd = mv_fill<R, V>(R(0));
    MPSW_SLOTS(k, NB::c, n) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R sg = R(m.c_esg[(size_t)k * nC + c]);
      const size_t oe = (size_t)e * B + q.b;
      const M Te = ldv<V>(in.tu + oe);
      const R dce = ld(m.e_dc, e);
      const M gpn_ad = w.gpn_ad ? ldv<V>(w.gpn_ad + oe)
                                : mv_fill<R, V>(R(0)) - ((ph.apvm * ld(bs.u, e)) * ph.dt) * ldv<V>(w.pe_ad + oe);
      pc_ad = pc_ad + (-sg) * (gpn_ad / dce);
      ke_ad = ke_ad + sg * (Te / dce);
      hd = hd + sg * ((R(GRAVITY) / dce) * Te);
      if (ph.drag) {
        const R sq = sqrt(R(2) * (R(0.5) * (ld(bs.ke, ld(m.e_c1, e)) + ld(bs.ke, ld(m.e_c2, e)))));
        const M kea = -(((((R(0.5) * R(1.0e-3)) * ld(bs.u, e)) * R(2)) / sq) / ld(bs.he, e)) * Te;
        ke_ad = ke_ad + R(0.5) * kea;
      }
      if (ph.visc2 > R(0)) {
        const M ud2 = (ld(m.e_sc2, e) * ph.visc2) * Te;
        div_ad = div_ad + (-sg) * (ud2 / dce);
      }
      if (ph.visc4 > R(0)) div_ad = div_ad + (-sg) * (ldv<V>(w.du_ad + oe) / dce);
      hd = hd + R(0.5) * ldv<V>(w.he_ad + oe);
    }
    const R area = ld(m.c_area, c);
    const size_t o = (size_t)c * B + q.b;
    stv<V>(w.pc_ad + o, pc_ad);
    stv<V>(w.ke_ad + o, ke_ad / area);
    if (w.div_ad) stv<V>(w.div_ad + o, div_ad * (R(1) / area));
    stv<V>(w.hd + o, hd);
  }
}

// Shared-memory bytes per cell of ad_cell_st's stage: 6 slots of an edge index and 6 coefficients.
template <typename R>
__host__ __device__ constexpr size_t ad_cell_stage_bytes() {
  return (size_t)BoundsNarrow::c * (sizeof(int) + 6 * sizeof(R));
}

// k_ad_cell with each block's cell lists staged in shared memory (meshes with at most 6
// edgesOnCell): per slot the edge (reference scatter order), its sign, dcEdge and the scalar
// coefficients of the slot's terms (gradPVn, gravity, drag, del2), computed with the same
// operations as k_ad_cell.  Slots past the cell's edge count hold edge 0 with sign 0, dcEdge 1
// and zero coefficients, so every term there is an exact zero and all 6 slots run without a
// bound check.  early: copy the lists before waiting for the previous kernel.
template <typename R, typename A, int V>
__device__ __forceinline__ void ad_cell_st_run(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd, AdWork<R> w,
                             int early) {
  using M = Mv<R, V>;
  constexpr int S = BoundsNarrow::c;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (!early) pdl_begin();
  const int nC = m.nC, tpe = B / V, cpb = blockDim.x / tpe;
  const int c0 = blockIdx.x * cpb;
  R *sr = reinterpret_cast<R *>(smem_raw);                      // [6][S][cpb]
  int *se = reinterpret_cast<int *>(sr + (size_t)6 * S * cpb);  // [S][cpb]
  const size_t SC = (size_t)S * cpb;
  for (int i = threadIdx.x; i < S * cpb; i += blockDim.x) {
    const int k = i / cpb, lc = i - k * cpb, c = c0 + lc;
    int e = 0;
    R sg = R(0), dce = R(1), gq = R(0), gg = R(0), kd = R(0), k2 = R(0);
    if (c < nC && k < ld(m.c_n, c)) {
      e = ld(m.c_es, (size_t)k * nC + c);
      sg = R(m.c_esg[(size_t)k * nC + c]);
      dce = ld(m.e_dc, e);
      gq = (ph.apvm * ld(bs.u, e)) * ph.dt;
      gg = R(GRAVITY) / dce;
      if (ph.drag) {
        const R sq = sqrt(R(2) * (R(0.5) * (ld(bs.ke, ld(m.e_c1, e)) + ld(bs.ke, ld(m.e_c2, e)))));
        kd = -(((((R(0.5) * R(1.0e-3)) * ld(bs.u, e)) * R(2)) / sq) / ld(bs.he, e));
      }
      if (ph.visc2 > R(0)) k2 = ld(m.e_sc2, e) * ph.visc2;
    }
    sr[0 * SC + i] = sg; sr[1 * SC + i] = dce; sr[2 * SC + i] = gq; sr[3 * SC + i] = gg;
    sr[4 * SC + i] = kd; sr[5 * SC + i] = k2;
    se[i] = e;
  }
  __syncthreads();
  if (early) pdl_begin();
  const int lc = threadIdx.x / tpe, c = c0 + lc;
  if (lc >= cpb || c >= nC) return;
  const int b = (threadIdx.x - lc * tpe) * V;
  M pc_ad = mv_fill<R, V>(sd.pc ? sd.pc[c] : R(0));
  M ke_ad = mv_fill<R, V>(sd.ke ? sd.ke[c] : R(0));
  M div_ad = mv_fill<R, V>(sd.div ? sd.div[c] : R(0));
  M hd = mv_fill<R, V>(R(0));
  MPSW_SLOTS(k, S, S) {
    const int i = k * cpb + lc;
    const size_t oe = (size_t)se[i] * B + b;
    const R sg = sr[0 * SC + i], dce = sr[1 * SC + i];
    const R half = R(0.5) * (sg * sg);  // 0.5 (sg is +-1), or 0 in a padded slot
    const M Te = ldv<V>(in.tu + oe);
    const M gpn_ad = w.gpn_ad ? ldv<V>(w.gpn_ad + oe) : mv_fill<R, V>(R(0)) - sr[2 * SC + i] * ldv<V>(w.pe_ad + oe);
    if constexpr (sizeof(R) == 4) {
      // FP32 members: the slot's sign over dcEdge formed once, no division per member
      const R rs = sg / dce;
      pc_ad = pc_ad - rs * gpn_ad;
      ke_ad = ke_ad + rs * Te;
      hd = hd + sg * (sr[3 * SC + i] * Te);
      if (ph.drag) ke_ad = ke_ad + R(0.5) * (sr[4 * SC + i] * Te);
      if (ph.visc2 > R(0)) div_ad = div_ad - (rs * sr[5 * SC + i]) * Te;
      if (ph.visc4 > R(0)) div_ad = div_ad - rs * ldv<V>(w.du_ad + oe);
    } else {
      pc_ad = pc_ad + (-sg) * (gpn_ad / dce);
      ke_ad = ke_ad + sg * (Te / dce);
      hd = hd + sg * (sr[3 * SC + i] * Te);
      if (ph.drag) ke_ad = ke_ad + R(0.5) * (sr[4 * SC + i] * Te);
      if (ph.visc2 > R(0)) div_ad = div_ad + (-sg) * ((sr[5 * SC + i] * Te) / dce);
      if (ph.visc4 > R(0)) div_ad = div_ad + (-sg) * (ldv<V>(w.du_ad + oe) / dce);
    }
    hd = hd + half * ldv<V>(w.he_ad + oe);
  }
  const R area = ld(m.c_area, c);
  const size_t o = (size_t)c * B + b;
  stv<V>(w.pc_ad + o, pc_ad);
  stv<V>(w.ke_ad + o, ke_ad / area);
  if (w.div_ad) stv<V>(w.div_ad + o, div_ad * (R(1) / area));
  stv<V>(w.hd + o, hd);
}
template <typename R, typename A, int V>
__global__ void k_ad_cell_st(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd, AdWork<R> w,
                             int early) {
  ad_cell_st_run<R, A, V>(m, B, bs, ph, in, sd, w, early);
}
#if MPSW_REGS_AD_CELL > 0
template <typename A, int V>
__global__ void __maxnreg__(MPSW_REGS_AD_CELL) k_ad_cell_st_rc(MeshDev<float> m, int B, Base<float> bs, Phys<float> ph, AdIn<float> in, AdSeeds<float> sd, AdWork<float> w,
                             int early) {
  ad_cell_st_run<float, A, V>(m, B, bs, ph, in, sd, w, early);
}
#endif
template <typename R, typename A, int V>
inline auto ad_cell_st_kernel() {
#if MPSW_REGS_AD_CELL > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_ad_cell_st_rc<A, V> : &k_ad_cell_st<R, A, V>;
  else return &k_ad_cell_st<R, A, V>;
#else
  return &k_ad_cell_st<R, A, V>;
#endif
}

// Vertex stage: pv_cell -> pv_vertex (:215-229), pv_edge -> pv_vertex (:244-252),
// gradPVt -> pv_vertex (:254-262), del2/del4 vorticity adjoints, pv_vertex -> h_vertex and
// vorticity (:268-284), vorticity -> circulation (:343-349).
template <typename R, typename A, int V>
__global__ void k_ad_vertex(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in,
                            AdSeeds<R> sd, AdWork<R> w) {
  using M = Mv<R, V>;
  const int nV = m.nV;
  MPSW_MEMBER_LOOP(t, nV, B, V) {
    const EntMember q = ent_member(t, B, V);
    const int v = q.ent;
    M pvv_ad = mv_fill<R, V>(sd.pvv ? sd.pvv[v] : R(0));
    M vort_ad = mv_fill<R, V>(sd.vort ? sd.vort[v] : R(0));
#pragma unroll
    for (int i = 0; i < VDEG; i++) {
      const int c = ld(m.v_c, (size_t)i * nV + v);
      const R ka = ld(m.v_k, (size_t)i * nV + v) / ld(m.c_area, c);
      if (sd.vc) vort_ad = vort_ad + ka * sd.vc[c];
      pvv_ad = pvv_ad + ka * ldv<V>(w.pc_ad + (size_t)c * B + q.b);
    }
#pragma unroll
    for (int i = 0; i < VDEG; i++)
      pvv_ad = pvv_ad + R(0.5) * ldv<V>(w.pe_ad + (size_t)ld(m.v_e, (size_t)i * nV + v) * B + q.b);
#pragma unroll
    for (int k = 0; k < VDEG; k++) {
      const int e = ld(m.v_es, (size_t)k * nV + v);
      const R sg = R(m.v_esg[(size_t)k * nV + v]);
      const R dve = ld(m.e_dv, e);
      const size_t oe = (size_t)e * B + q.b;
      const M gpt_ad = w.gpt_ad ? ldv<V>(w.gpt_ad + oe)
                                : mv_fill<R, V>(R(0)) - ((ph.apvm * ld(bs.v, e)) * ph.dt) * ldv<V>(w.pe_ad + oe);
      pvv_ad = pvv_ad + sg * (gpt_ad / dve);
      if (ph.visc2 > R(0)) {
        const M ud2 = (ld(m.e_sc2, e) * ph.visc2) * ldv<V>(in.tu + oe);
        vort_ad = vort_ad + (-sg) * (ud2 / dve);
      }
      if (ph.visc4 > R(0)) vort_ad = vort_ad + (-sg) * (ldv<V>(w.du_ad + oe) / dve);
    }
    const R hv = ld(bs.hv, v), area = ld(m.v_area, v);
    M hv_ad = mv_fill<R, V>(sd.hv ? sd.hv[v] : R(0));
    hv_ad = hv_ad - ((ld(m.v_f, v) + ld(bs.vort, v)) / (hv * hv)) * pvv_ad;
    vort_ad = vort_ad + pvv_ad / hv;
    hv_ad = hv_ad / area;
    const M circ_ad = mv_fill<R, V>(sd.circ ? sd.circ[v] : R(0)) + vort_ad / area;
    const size_t o = (size_t)v * B + q.b;
    stv<V>(w.hv_ad + o, hv_ad);
    stv<V>(w.circ_ad + o, circ_ad);
  }
}

// Shared-memory bytes per vertex of k_ad_vertex_st's stage: 3 slots of 3 indices and 4 values.
template <typename R>
__host__ __device__ constexpr size_t ad_vertex_stage_bytes() {
  return (size_t)VDEG * (3 * sizeof(int) + 4 * sizeof(R));
}

// k_ad_vertex with each block's vertex lists (cell with kite / areaCell; edgesOnVertex edge;
// edge in the reference's scatter order with its sign, dvEdge and del2 coefficient) copied into
// shared memory before waiting for the previous kernel: they are mesh data, which no kernel
// writes.  Same operations as k_ad_vertex.
template <typename R, typename A, int V>
__device__ __forceinline__ void ad_vertex_st_run(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                               AdWork<R> w) {
  using M = Mv<R, V>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nV = m.nV, tpe = B / V, vpb = blockDim.x / tpe;
  const int v0 = blockIdx.x * vpb;
  const size_t SV = (size_t)VDEG * vpb;
  R *ska = reinterpret_cast<R *>(smem_raw), *ssg = ska + SV, *sdv = ssg + SV, *sk2 = sdv + SV;  // [VDEG][vpb]
  int *sc = reinterpret_cast<int *>(sk2 + SV), *sve = sc + SV, *ses = sve + SV;
  for (int i = threadIdx.x; i < VDEG * vpb; i += blockDim.x) {
    const int k = i / vpb, v = v0 + (i - k * vpb);
    int c = 0, ve = 0, e = 0;
    R ka = R(0), sg = R(0), dve = R(1), k2 = R(0);
    if (v < nV) {
      c = ld(m.v_c, (size_t)k * nV + v);
      ka = ld(m.v_k, (size_t)k * nV + v) / ld(m.c_area, c);
      ve = ld(m.v_e, (size_t)k * nV + v);
      e = ld(m.v_es, (size_t)k * nV + v);
      sg = R(m.v_esg[(size_t)k * nV + v]);
      dve = ld(m.e_dv, e);
      if (ph.visc2 > R(0)) k2 = ld(m.e_sc2, e) * ph.visc2;
    }
    ska[i] = ka; ssg[i] = sg; sdv[i] = dve; sk2[i] = k2; sc[i] = c; sve[i] = ve; ses[i] = e;
  }
  __syncthreads();
  pdl_begin();
  const int lv = threadIdx.x / tpe, v = v0 + lv;
  if (lv >= vpb || v >= nV) return;
  const int b = (threadIdx.x - lv * tpe) * V;
  M pvv_ad = mv_fill<R, V>(sd.pvv ? sd.pvv[v] : R(0));
  M vort_ad = mv_fill<R, V>(sd.vort ? sd.vort[v] : R(0));
#pragma unroll
  for (int k = 0; k < VDEG; k++) {
    const int i = k * vpb + lv;
    const R ka = ska[i];
    if (sd.vc) vort_ad = vort_ad + ka * sd.vc[sc[i]];
    pvv_ad = pvv_ad + ka * ldv<V>(w.pc_ad + (size_t)sc[i] * B + b);
  }
#pragma unroll
  for (int k = 0; k < VDEG; k++)
    pvv_ad = pvv_ad + R(0.5) * ldv<V>(w.pe_ad + (size_t)sve[k * vpb + lv] * B + b);
#pragma unroll
  for (int k = 0; k < VDEG; k++) {
    const int i = k * vpb + lv;
    const int e = ses[i];
    const R sg = ssg[i], dve = sdv[i];
    const size_t oe = (size_t)e * B + b;
    const M gpt_ad = w.gpt_ad ? ldv<V>(w.gpt_ad + oe)
                              : mv_fill<R, V>(R(0)) - ((ph.apvm * ld(bs.v, e)) * ph.dt) * ldv<V>(w.pe_ad + oe);
    if constexpr (sizeof(R) == 4) {
      // FP32 members: the slot's sign over dvEdge formed once, no division per member
      const R rs = sg / dve;
      pvv_ad = pvv_ad + rs * gpt_ad;
      if (ph.visc2 > R(0)) vort_ad = vort_ad - (rs * sk2[i]) * ldv<V>(in.tu + oe);
      if (ph.visc4 > R(0)) vort_ad = vort_ad - rs * ldv<V>(w.du_ad + oe);
    } else {
      pvv_ad = pvv_ad + sg * (gpt_ad / dve);
      if (ph.visc2 > R(0)) {
        const M ud2 = sk2[i] * ldv<V>(in.tu + oe);
        vort_ad = vort_ad + (-sg) * (ud2 / dve);
      }
      if (ph.visc4 > R(0)) vort_ad = vort_ad + (-sg) * (ldv<V>(w.du_ad + oe) / dve);
    }
  }
  const R hv = ld(bs.hv, v), area = ld(m.v_area, v);
  M hv_ad = mv_fill<R, V>(sd.hv ? sd.hv[v] : R(0));
  hv_ad = hv_ad - ((ld(m.v_f, v) + ld(bs.vort, v)) / (hv * hv)) * pvv_ad;
  vort_ad = vort_ad + pvv_ad / hv;
  hv_ad = hv_ad / area;
  const M circ_ad = mv_fill<R, V>(sd.circ ? sd.circ[v] : R(0)) + vort_ad / area;
  const size_t o = (size_t)v * B + b;
  stv<V>(w.hv_ad + o, hv_ad);
  stv<V>(w.circ_ad + o, circ_ad);
}
template <typename R, typename A, int V>
__global__ void k_ad_vertex_st(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                               AdWork<R> w) {
  ad_vertex_st_run<R, A, V>(m, B, bs, ph, in, sd, w);
}
#if MPSW_REGS_AD_VERTEX > 0
template <typename A, int V>
__global__ void __maxnreg__(MPSW_REGS_AD_VERTEX) k_ad_vertex_st_rc(MeshDev<float> m, int B, Base<float> bs, Phys<float> ph, AdIn<float> in, AdSeeds<float> sd,
                               AdWork<float> w) {
  ad_vertex_st_run<float, A, V>(m, B, bs, ph, in, sd, w);
}
#endif
template <typename R, typename A, int V>
inline auto ad_vertex_st_kernel() {
#if MPSW_REGS_AD_VERTEX > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_ad_vertex_st_rc<A, V> : &k_ad_vertex_st<R, A, V>;
  else return &k_ad_vertex_st<R, A, V>;
#else
  return &k_ad_vertex_st<R, A, V>;
#endif
}

template <typename R, typename A, int V>
__device__ __forceinline__ void ad_emit(const AdOut<R, A> &out, int is_edge, size_t o, const Mv<R, V> &pad,
                                        R area) {
  A *acc = is_edge ? out.acc_u : out.acc_h;
  const A *x2 = is_edge ? out.x2u : out.x2h;
  R *tn = is_edge ? out.tu_next : out.th_next;
  const A wn = is_edge ? out.wu : out.wh, cn = is_edge ? out.cu : out.ch;
  Mv<A, V> next;
  const R *const *pin = is_edge ? out.pad_in_u : out.pad_in_h;
  R *pout = is_edge ? out.pad_out_u : out.pad_out_h;
  if (out.mode == AD_FINAL) {
    A *dst = is_edge ? out.dst_u : out.dst_h;
    Mv<A, V> a;
    if (pin[0]) {  // the stored contributions of the three later stages, in stage order
      a = mv_cast<V, A>(ldv<V>(pin[0] + o));
#pragma unroll
      for (int j = 1; j < 3; j++) {
        const Mv<R, V> pj = ldv<V>(pin[j] + o);
#pragma unroll
        for (int i = 0; i < V; i++) a.x[i] = a.x[i] + A(pj.x[i]);
      }
    } else {
      a = ldv<V>(acc + o);
    }
    const Mv<A, V> x = ldv<V>(x2 + o);
    Mv<A, V> d;
#pragma unroll
    for (int i = 0; i < V; i++) {
      d.x[i] = (a.x[i] + x.x[i]) + A(pad.x[i]);
      next.x[i] = wn * d.x[i];
    }
    stv<V>(dst + o, d);
    if (R *xr = is_edge ? out.x2r_u : out.x2r_h) stv<V>(xr + o, mv_cast<V, R>(d));
  } else {
    if (pout) {
      stv<V>(pout + o, pad);
    } else {
      Mv<A, V> a;
      if (out.mode == AD_SET) {
        a = mv_cast<V, A>(pad);
      } else {
        a = ldv<V>(acc + o);
#pragma unroll
        for (int i = 0; i < V; i++) a.x[i] = a.x[i] + A(pad.x[i]);
      }
      stv<V>(acc + o, a);
    }
    if (tn) {
      const R *xr = is_edge ? out.x2r_u : out.x2r_h;
      if (xr) {
        const Mv<R, V> x = ldv<V>(xr + o);
#pragma unroll
        for (int i = 0; i < V; i++) next.x[i] = wn * A(x.x[i]) + cn * A(pad.x[i]);
      } else {
        const Mv<A, V> x = x2 ? ldv<V>(x2 + o) : mv_fill<A, V>(A(0));
#pragma unroll
        for (int i = 0; i < V; i++) next.x[i] = (x2 ? wn * x.x[i] : A(0)) + cn * A(pad.x[i]);
      }
    }
  }
  if (tn) {
    Mv<R, V> r;
#pragma unroll
    for (int i = 0; i < V; i++) {
      if constexpr (sizeof(R) == 4)  // FP32 members: one reciprocal of areaCell per cell
        r.x[i] = is_edge ? R(next.x[i]) : R(next.x[i] * (A(1) / A(area)));
      else
        r.x[i] = is_edge ? R(next.x[i]) : R(next.x[i] / A(area));
    }
    stv<V>(tn + o, r);
  }
}

// Final stage of the adjoint: h_vertex -> h (:286-289) on cells, and on edges the transposed
// tangential velocity (:296-303), ke (:306-317), divergence (:327-340) and circulation
// (:350-355) adjoints.  Cell threads then edge threads.
template <typename R, typename A, int V, int NMAX>
__device__ __forceinline__ void ad_final_cell(const MeshDev<R> &m, int B, const AdWork<R> &w,
                                              const AdOut<R, A> &out, int c, int b) {
  using M = Mv<R, V>;
  const int nC = m.nC;
  const int n = ld(m.c_n, c);
  M ph_ = ldv<V>(w.hd + (size_t)c * B + b);
  MPSW_PADDED(k, NMAX, n)
    ph_ = ph_ + ld(m.c_vk, (size_t)k * nC + c) * ldv<V>(w.hv_ad + (size_t)ld(m.c_vs, (size_t)k * nC + c) * B + b);
  ad_emit<R, A, V>(out, 0, (size_t)c * B + b, ph_, ld(m.c_area, c));
}

// l's field 0 is gradPVt of the linearisation point at the neighbours (to re-form v_ad).
template <typename R, typename A, int V, int NMAX, class L>
__device__ __forceinline__ void ad_final_edge(const MeshDev<R> &m, int B, const Base<R> &bs, const Phys<R> &ph,
                                              const AdWork<R> &w, const AdOut<R, A> &out, int e, int b,
                                              const L &l) {
  using M = Mv<R, V>;
  const int n = ld(m.e_n, e);
  M pu = ldv<V>(w.ud + (size_t)e * B + b);
  MPSW_SLOTS(j, NMAX, L::kPadded ? NMAX : n) {
    const size_t on = (size_t)l.nb(j) * B + b;
    const M v_ad = w.v_ad ? ldv<V>(w.v_ad + on)
                          : mv_fill<R, V>(R(0)) - ((ph.apvm * ph.dt) * l.f(0, j)) * ldv<V>(w.pe_ad + on);
    pu = pu + l.wr(j) * v_ad;
  }
  const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e), v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e);
  const R dc = ld(m.e_dc, e), dv = ld(m.e_dv, e);
  const R kc = (((R(0.25) * dc) * dv) * R(2)) * ld(bs.u, e);
  pu = pu + kc * ldv<V>(w.ke_ad + (size_t)c1 * B + b);
  pu = pu + kc * ldv<V>(w.ke_ad + (size_t)c2 * B + b);
  if (w.div_ad) {  // null where it would be zero (window sweeps without viscosity)
    pu = pu - dv * ldv<V>(w.div_ad + (size_t)c2 * B + b);
    pu = pu + dv * ldv<V>(w.div_ad + (size_t)c1 * B + b);
  }
  pu = pu + dc * ldv<V>(w.circ_ad + (size_t)v2 * B + b);
  pu = pu - dc * ldv<V>(w.circ_ad + (size_t)v1 * B + b);
  if (ph.bad) {
#pragma unroll
    for (int i = 0; i < V; i++) flag_nonfinite(ph.bad, pu.x[i]);
  }
  ad_emit<R, A, V>(out, 1, (size_t)e * B + b, pu, R(1));
}

template <typename R, typename A, int V, class NB>
__global__ void k_ad_final(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdWork<R> w, AdOut<R, A> out) {
  const long long tc = (long long)m.nC * (B / V);
  MPSW_GRID_LOOP(t, tc + (long long)m.nE * (B / V)) {
    if (t < tc) {
      const EntMember q = ent_member(t, B, V);
      ad_final_cell<R, A, V, NB::c>(m, B, w, out, q.ent, q.b);
    } else {
      const EntMember q = ent_member(t - tc, B, V);
      ad_final_edge<R, A, V, NB::e2>(m, B, bs, ph, w, out, q.ent, q.b, eoe_global(m, q.ent, bs.gpt));
    }
  }
}

// k_ad_final with staged edge lists: the first cell_blocks blocks take the cells (one member
// group per thread), the others epb edges each with their lists in shared memory.
template <typename R, typename A, int V, int J>
__device__ __forceinline__ void ad_final_st_run(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdWork<R> w, AdOut<R, A> out,
                              int cell_blocks, int early) {
  if ((int)blockIdx.x < cell_blocks) {
    pdl_begin();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (long long)m.nC * (B / V)) {
      const EntMember q = ent_member(t, B, V);
      ad_final_cell<R, A, V, BoundsNarrow::c>(m, B, w, out, q.ent, q.b);
    }
    return;
  }
  const int tpe = B / V, epb = blockDim.x / tpe;
  const int le = threadIdx.x / tpe;
  const int e = ((int)blockIdx.x - cell_blocks) * epb + le;
  const int b = (threadIdx.x - le * tpe) * V;
  if (!early) pdl_begin();
  const R *const fields[1] = {bs.gpt};
  const EoeShared<R> st = stage_eoe<R, J, 2, 1>(m, ((int)blockIdx.x - cell_blocks) * epb, epb, le, fields);
  if (early) pdl_begin();
  if (le < epb && e < m.nE) ad_final_edge<R, A, V, J>(m, B, bs, ph, w, out, e, b, st);
}
template <typename R, typename A, int V, int J>
__global__ void k_ad_final_st(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdWork<R> w, AdOut<R, A> out,
                              int cell_blocks, int early) {
  ad_final_st_run<R, A, V, J>(m, B, bs, ph, w, out, cell_blocks, early);
}
#if MPSW_REGS_AD_FINAL > 0
template <typename A, int V, int J>
__global__ void __maxnreg__(MPSW_REGS_AD_FINAL) k_ad_final_st_rc(MeshDev<float> m, int B, Base<float> bs, Phys<float> ph, AdWork<float> w, AdOut<float, A> out,
                              int cell_blocks, int early) {
  ad_final_st_run<float, A, V, J>(m, B, bs, ph, w, out, cell_blocks, early);
}
#endif
template <typename R, typename A, int V, int J>
inline auto ad_final_st_kernel() {
#if MPSW_REGS_AD_FINAL > 0
  if constexpr (std::is_same<R, float>::value && V == 8) return regcap_on() ? &k_ad_final_st_rc<A, V, J> : &k_ad_final_st<R, A, V, J>;
  else return &k_ad_final_st<R, A, V, J>;
#else
  return &k_ad_final_st<R, A, V, J>;
#endif
}

}  // namespace mpsw
