// Stencil kernels of the shallow-water RK4 dycore, its tangent linear and its adjoint.
//
// Every reference loop that scatters (x(cell(e)) += ...) is rewritten as a gather over the
// transposed connectivity built by the host set-up, in the order the reference visits the
// scattering entities, so the FP64 instantiation (compiled without FMA contraction) reproduces
// the reference arithmetic operation for operation.  The adjoint kernels turn the reference's
// reverse-order scatters into deterministic gathers: no atomics anywhere.
//
// Kernels are templated on R (stencil arithmetic and storage of provisional states,
// diagnostics and members) and A (RK4 accumulation); B is the number of members riding the
// trailing dimension of member arrays ([n][B]).  One thread handles one (entity, member) pair.
#pragma once

#include <type_traits>

#include "mpsw_internal.h"

namespace mpsw {

// Kernels launched with programmatic stream serialisation start while the previous kernel on
// the stream may still run: wait for it (and its memory writes) before touching any buffer,
// then let the next kernel be scheduled.  Both are no-ops for a kernel launched without it.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Grid-stride loop over `total` work items, preceded by pdl_begin(): every kernel body starts
// with it.
#define MPSW_GRID_LOOP(t, total)                                                               \
  pdl_begin();                                                                                 \
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)(total); \
       t += (long long)gridDim.x * blockDim.x)

// Raise the non-finite flag (Phys::bad) when x is NaN or infinite.
template <typename R>
__device__ __forceinline__ void flag_nonfinite(int *bad, R x) {
  if (bad && !isfinite(x)) *bad = 1;
}

template <typename R>
__device__ __forceinline__ R ld(const R *p, size_t i) {
  return __ldg(p + i);
}

// Bounds of the neighbour loops.  BoundsNarrow serves meshes with at most 10 edgesOnEdge and 6
// edgesOnCell (every quasi-uniform hexagon/pentagon mesh): the loops get compile-time trip
// counts and are unrolled with `slot < n` as a predicate, so the connectivity, weight and member
// loads of all slots can be in flight together instead of one slot after another.  BoundsAny
// keeps runtime trip counts for any mesh within MAXE2 / MAXE.
struct BoundsNarrow {
  static constexpr int e2 = 10, c = 6;
};
struct BoundsAny {
  static constexpr int e2 = 0, c = 0;
};

// j over the first n slots of a list whose length is at most NMAX (NMAX 0: no static bound)
#define MPSW_SLOTS(j, NMAX, n)                                                \
  _Pragma("unroll") for (int j = 0; j < ((NMAX) > 0 ? (NMAX) : (n)); j++) \
    if ((NMAX) == 0 || j < (n))

// The device mesh pads every list past its entity's count with index 0 and zero weights, signs
// and kites (MAXE2 slots for edgesOnEdge, MAXE for the cell lists).  A term whose coefficient
// is one of those padded values is an exact zero there, so such a loop may run all NMAX slots of
// a narrow mesh without a bound check: MPSW_PADDED(j, NMAX, n).
#define MPSW_PADDED(j, NMAX, n) MPSW_SLOTS(j, NMAX, ((NMAX) > 0 ? (NMAX) : (n)))


// ----------------------------------------------------------------------------------------
// Forward: sw_compute_solve_diagnostics (src/mpas_sw_dyncore.f90:1-361) split by entity.
// h is stored relative to `off` (0 for FP64, a reference depth for reduced precision).
// ----------------------------------------------------------------------------------------

// circulation/vorticity (:208-219), h_vertex and pv_vertex (:282-292)
template <typename R>
__global__ void k_fwd_vertex(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                             Diag<R> d) {
  const int nV = m.nV;
  MPSW_GRID_LOOP(t, nV) {
    const int v = (int)t;
    R circ = R(0);
#pragma unroll
    for (int k = 0; k < VDEG; k++) {
      const int e = ld(m.v_es, (size_t)k * nV + v);
      const R s = R(m.v_esg[(size_t)k * nV + v]);
      circ = circ + s * (ld(m.e_dc, e) * ld(u, e));
    }
    const R area = ld(m.v_area, v);
    const R vort = circ / area;
    R hv = R(0);
#pragma unroll
    for (int k = 0; k < VDEG; k++)
      hv = hv + (ld(h, ld(m.v_c, (size_t)k * nV + v)) + off) * ld(m.v_k, (size_t)k * nV + v);
    hv = hv / area;
    const R pv = (ld(m.v_f, v) + vort) / hv;
    if (d.circ) d.circ[v] = circ;
    d.vort[v] = vort;
    d.hv[v] = hv;
    d.pvv[v] = pv;
  }
}

// divergence (:222-242), ke (:245-256), pv_cell/vorticity_cell (:324-340) and the thickness
// tendency (:468-482) with its RK update.
// c_nb[k][c] is the cell across edge k of the cell (its h_edge sums this cell's h and that
// cell's, in either order: the same value)
template <typename R, typename A, int NC>
__global__ void k_fwd_cell(MeshDev<R> m, const int *__restrict__ c_nb, const R *__restrict__ u,
                           const R *__restrict__ h, R off, Diag<R> d, RK<R, A> rk, R *tend_h) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, nC) {
    const int c = (int)t;
    const int n = ld(m.c_n, c);
    const R hc = ld(h, c) + off;
    R div = R(0), th = R(0);
    MPSW_PADDED(k, NC, n) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R s = R(m.c_esg[(size_t)k * nC + c]);
      const R ue = ld(u, e), dve = ld(m.e_dv, e);
      div = div + s * (ue * dve);
      const R he = R(0.5) * (hc + (ld(h, ld(c_nb, (size_t)k * nC + c)) + off));
      th = th + (-s) * ((ue * dve) * he);
    }
    const R area = ld(m.c_area, c);
    div = div * (R(1) / area);
    R ke = R(0);
    for (int i = 0; i < n; i++) {
      const int e = ld(m.c_eoc, (size_t)i * nC + c);
      const R ue = ld(u, e);
      ke = ke + ((R(0.25) * ld(m.e_dc, e)) * ld(m.e_dv, e)) * (ue * ue);
    }
    R pc = R(0), vc = R(0);
    if constexpr (sizeof(R) == 4) {
      // FP32 stencils: 1 / areaCell formed once instead of eight divisions
      const R ra = R(1) / area;
      ke = ke * ra;
      MPSW_PADDED(k, NC, n) {
        const int v = ld(m.c_vs, (size_t)k * nC + c);
        const R kr = ld(m.c_vk, (size_t)k * nC + c) * ra;
        pc = pc + kr * d.pvv[v];
        if (d.vc) vc = vc + kr * d.vort[v];
      }
      th = th * ra;
    } else {
      ke = ke / area;
      MPSW_PADDED(k, NC, n) {
        const int v = ld(m.c_vs, (size_t)k * nC + c);
        const R kt = ld(m.c_vk, (size_t)k * nC + c);
        pc = pc + (kt * d.pvv[v]) / area;
        if (d.vc) vc = vc + (kt * d.vort[v]) / area;
      }
      th = th / area;
    }
    d.div[c] = div;
    d.ke[c] = ke;
    d.pc[c] = pc;
    if (d.vc) d.vc[c] = vc;
    if (tend_h) tend_h[c] = th;
    if (rk.next) rk.next[c] = R((rk.x0[c] - A(rk.off)) + rk.c * A(th));
    if (rk.acc_out) rk.acc_out[c] = rk.acc_in[c] + rk.w * A(th);
  }
}

// tangential velocity (:259-267), gradPVt (:296-301), pv_edge with both APVM terms
// (:305-320, :344-359), h_edge (:95-105) and, for del4, delsq_u (:539-551).
template <typename R, int NE>
__global__ void k_fwd_edge_diag(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                                Diag<R> d, Phys<R> ph) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, nE) {
    const int e = (int)t;
    const int n = ld(m.e_n, e);
    R v = R(0);
    MPSW_PADDED(j, NE, n)
      v = v + ld(m.e_w, (size_t)j * nE + e) * ld(u, ld(m.e_eoe, (size_t)j * nE + e));
    const int v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e), c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
    const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
    const R pv1 = d.pvv[v1], pv2 = d.pvv[v2];
    const R gpt = (pv2 - pv1) / dv;
    // pv_edge's two vertex terms: the reference adds them over edgesOnVertex, which lists the
    // same two endpoints; a sum of two terms is the same in either order
    R pe = R(0);
    pe = pe + R(0.5) * pv1;
    pe = pe + R(0.5) * pv2;
    pe = pe - ((ph.apvm * v) * ph.dt) * gpt;
    const R gpn = (d.pc[c2] - d.pc[c1]) / dc;
    pe = pe - ((ph.apvm * ld(u, e)) * ph.dt) * gpn;
    d.pe[e] = pe;
    const R he = R(0.5) * ((ld(h, c1) + off) + (ld(h, c2) + off));
    if constexpr (sizeof(R) == 4) {
      // FP32 stencils: the edge's thickness flux u h_edge in d.he and PV flux u h_edge pv_edge
      // in d.v, the two values k_fwd_edge_tend gathers at the neighbours
      const R f = ld(u, e) * he;
      d.he[e] = f;
      d.v[e] = f * pe;
    } else {
      d.he[e] = he;
      if (d.v) d.v[e] = v;
    }
    if (d.gpt) d.gpt[e] = gpt;
    if (d.gpn) d.gpn[e] = gpn;
    if (d.dsq_u) d.dsq_u[e] = (d.div[c2] - d.div[c1]) / dc - (d.vort[v2] - d.vort[v1]) / dv;
  }
}

// Normal-velocity tendency (src/mpas_sw_dyncore.f90:485-637) and its RK update.
template <typename R, typename A, int NE>
__global__ void k_fwd_edge_tend(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                                Diag<R> d, Phys<R> ph, RK<R, A> rk, R *tend_u) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, nE) {
    const int e = (int)t;
    const int n = ld(m.e_n, e);
    const R pee = d.pe[e];
    R q = R(0);
    if constexpr (sizeof(R) == 4) {
      // FP32 stencils: q = 0.5 pv_edge(e) sum w (u h_edge)_j + 0.5 sum w (u h_edge pv_edge)_j,
      // the same sum regrouped by the neighbour fluxes k_fwd_edge_diag leaves in d.he and d.v
      R f1 = R(0), f2 = R(0);
      MPSW_PADDED(j, NE, n) {
        const int eoe = ld(m.e_eoe, (size_t)j * nE + e);
        const R w = ld(m.e_w, (size_t)j * nE + e);
        f1 = f1 + w * d.he[eoe];
        f2 = f2 + w * d.v[eoe];
      }
      q = (R(0.5) * pee) * f1 + R(0.5) * f2;
    } else {
      MPSW_PADDED(j, NE, n) {
        const int eoe = ld(m.e_eoe, (size_t)j * nE + e);
        const R wpv = R(0.5) * (pee + d.pe[eoe]);
        q = q + ((ld(m.e_w, (size_t)j * nE + e) * ld(u, eoe)) * wpv) * d.he[eoe];
      }
    }
    const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e), v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e);
    const R dc = ld(m.e_dc, e), dv = ld(m.e_dv, e);
    R grav;
    if constexpr (std::is_same<R, double>::value) {
      grav = R(GRAVITY) * ((((ld(h, c2) + off) + ld(m.c_hs, c2)) - (ld(h, c1) + off)) - ld(m.c_hs, c1));
    } else {  // reduced precision: difference the offset-free values first
      grav = R(GRAVITY) * ((ld(h, c2) - ld(h, c1)) + (ld(m.c_hs, c2) - ld(m.c_hs, c1)));
    }
    R tu = q - ((d.ke[c2] - d.ke[c1]) + grav) / dc;
    if (ph.visc2 > R(0)) {
      R ud = (d.div[c2] - d.div[c1]) / dc - (d.vort[v2] - d.vort[v1]) / dv;
      ud = (ld(m.e_sc2, e) * ph.visc2) * ud;
      tu = tu + ud;
    }
    if (ph.visc4 > R(0)) {
      R ud = (d.dsq_div[c2] - d.dsq_div[c1]) / dc - (d.dsq_vort[v2] - d.dsq_vort[v1]) / dv;
      ud = (ld(m.e_sc4, e) * ph.visc4) * ud;
      tu = tu - ud;
    }
    // h_edge of the edge itself (d.he holds the thickness flux with FP32 stencils)
    const R hee = sizeof(R) == 4 ? R(0.5) * ((ld(h, c1) + off) + (ld(h, c2) + off)) : d.he[e];
    if (ph.wind) tu = tu + (ld(m.e_usrc, e) / R(RHO_REF)) / hee;
    if (ph.drag) {
      const R kee = R(0.5) * (d.ke[c1] + d.ke[c2]);
      tu = tu - ((R(1.0e-3) * ld(u, e)) * sqrt(R(2) * kee)) / hee;
    }
    if (ph.bad && !isfinite(tu)) *ph.bad = 1;
    if (tend_u) tend_u[e] = tu;
    if (rk.next) rk.next[e] = rk.frozen ? R(rk.x0[e]) : R(rk.x0[e] + rk.c * A(tu));
    if (rk.acc_out && !rk.frozen) rk.acc_out[e] = rk.acc_in[e] + rk.w * A(tu);
  }
}

// Tracer transport in one RK4 stage, the call the reference leaves out of sw_rk4
// (src/mpas_sw_module.f90:587): MPAS's order-2 scalar tendency in the form of the thickness
// tendency (:468-482) -- the h_edge-weighted flux of the edge-mean tracer, gathered in the
// reference's scatter order and divided by areaCell -- then MPAS's mass-weighted RK4 update.
// One thread per (tracer, cell); tracers are [nT][nC].  The stage input tr_in is advected by the
// stage's u and h_edge (he).  first: acc = tr0 h0 + w tend; otherwise acc += w tend.  tr_next
// (stages 1-3): (h0 tr0 + c tend) / h_next.  last (stage 4): tr0 = acc / h_next, h_next being the
// new h.  tend (optional) receives the stage's tendency.
template <typename R, int NC>
__global__ void k_tracer_stage(MeshDev<R> m, const int *__restrict__ c_nb, int nT, const R *__restrict__ u,
                               const R *__restrict__ he, const R *__restrict__ tr_in, R *tr0, const R *h0,
                               const R *h_next, R *tend, R *acc, R *tr_next, R c, R w, int first, int last) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, (long long)nT * nC) {
    const int cc = (int)(t % nC);
    const R *tr = tr_in + (t - cc);
    const int n = ld(m.c_n, cc);
    const R tc = tr[cc];
    R sum = R(0);
    MPSW_PADDED(k, NC, n) {
      const int e = ld(m.c_es, (size_t)k * nC + cc);
      const R s = R(m.c_esg[(size_t)k * nC + cc]);
      const R flux = (ld(u, e) * ld(m.e_dv, e)) * ld(he, e);
      const R tre = R(0.5) * (tc + tr[ld(c_nb, (size_t)k * nC + cc)]);
      sum = sum + (-s) * (flux * tre);
    }
    const R td = sum / ld(m.c_area, cc);
    if (tend) tend[t] = td;
    const R a = first ? tr0[t] * h0[cc] + w * td : acc[t] + w * td;
    if (tr_next) tr_next[t] = (h0[cc] * tr0[t] + c * td) / h_next[cc];
    if (last) tr0[t] = a / h_next[cc];
    else acc[t] = a;
  }
}

// Stand-alone thickness tendency from a given h_edge (src/mpas_sw_dyncore.f90:468-482).
template <typename R>
__global__ void k_tend_h(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ he, R *tend_h) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, nC) {
    const int c = (int)t;
    const int n = ld(m.c_n, c);
    R th = R(0);
    for (int k = 0; k < n; k++) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R s = R(m.c_esg[(size_t)k * nC + c]);
      th = th + (-s) * ((ld(u, e) * ld(m.e_dv, e)) * he[e]);
    }
    tend_h[c] = th / ld(m.c_area, c);
  }
}

// mpas_reconstruct_2d (src/mpas_sw_operators.f90:283-370) for B members.
template <typename R>
__global__ void k_recon(MeshDev<R> m, int B, int sphere, const R *__restrict__ u, R *X, R *Y, R *Z,
                        R *Zon, R *Mer) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, (long long)nC * B) {
    const int c = (int)(t / B), b = (int)(t - (long long)c * B);
    const int n = ld(m.c_n, c);
    R x = R(0), y = R(0), z = R(0);
    for (int i = 0; i < n; i++) {
      const int e = ld(m.c_eoc, (size_t)i * nC + c);
      const R ue = u[(size_t)e * B + b];
      x = x + ld(m.c_coef, ((size_t)0 * MAXE + i) * nC + c) * ue;
      y = y + ld(m.c_coef, ((size_t)1 * MAXE + i) * nC + c) * ue;
      z = z + ld(m.c_coef, ((size_t)2 * MAXE + i) * nC + c) * ue;
    }
    const size_t o = (size_t)c * B + b;
    if (X) X[o] = x;
    if (Y) Y[o] = y;
    if (Z) Z[o] = z;
    if (sphere) {
      const R clat = ld(m.c_trig, c), slat = ld(m.c_trig, (size_t)nC + c);
      const R clon = ld(m.c_trig, (size_t)2 * nC + c), slon = ld(m.c_trig, (size_t)3 * nC + c);
      Zon[o] = -x * slon + y * clon;
      Mer[o] = -(x * clon + y * slon) * slat + z * clat;
    } else {
      Zon[o] = x;
      Mer[o] = y;
    }
  }
}

// mpas_reconstruct_2d_adj (src/mpas_sw_dyncore_adj.f90:740-831), single member: cell part
// folds the zonal/meridional seeds into X/Y/Z seeds, edge part gathers coeffs^T * seeds.
template <typename R>
__global__ void k_recon_adj_cell(MeshDev<R> m, int sphere, R *Xa, R *Ya, R *Za, R *Zoa, R *Mea) {
  MPSW_GRID_LOOP(t, m.nC) {
    const int c = (int)t, nC = m.nC;
    if (sphere) {
      const R clat = ld(m.c_trig, c), slat = ld(m.c_trig, (size_t)nC + c);
      const R clon = ld(m.c_trig, (size_t)2 * nC + c), slon = ld(m.c_trig, (size_t)3 * nC + c);
      Za[c] = Za[c] + clat * Mea[c];
      Ya[c] = Ya[c] - slon * slat * Mea[c];
      Xa[c] = Xa[c] - clon * slat * Mea[c];
      Mea[c] = R(0);
      Ya[c] = Ya[c] + clon * Zoa[c];
      Xa[c] = Xa[c] - slon * Zoa[c];
      Zoa[c] = R(0);
    } else {
      Ya[c] = Ya[c] + Mea[c];
      Mea[c] = R(0);
      Xa[c] = Xa[c] + Zoa[c];
      Zoa[c] = R(0);
    }
  }
}
template <typename R, typename A>
__global__ void k_recon_adj_edge(MeshDev<R> m, const R *Xa, const R *Ya, const R *Za, A *u_ad) {
  MPSW_GRID_LOOP(t, m.nE) {
    const int e = (int)t, nC = m.nC;
    A acc = u_ad[e];
    const int cs[2] = {ld(m.e_c2, e), ld(m.e_c1, e)};
    const int ss[2] = {ld(m.e_slot2, e), ld(m.e_slot1, e)};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = cs[q], i = ss[q];
      acc = acc + ld(m.c_coef, ((size_t)2 * MAXE + i) * nC + c) * Za[c];
      acc = acc + ld(m.c_coef, ((size_t)1 * MAXE + i) * nC + c) * Ya[c];
      acc = acc + ld(m.c_coef, ((size_t)0 * MAXE + i) * nC + c) * Xa[c];
    }
    u_ad[e] = acc;
  }
}

// ----------------------------------------------------------------------------------------
// Boundary kernels: reference order <-> internal order, precision conversion.
// ----------------------------------------------------------------------------------------
// dst[new(i)][b] = src[i][b]  (perm maps reference index -> internal index)
template <typename S, typename D>
__global__ void k_to_internal(int n, int B, const int *__restrict__ perm, const S *__restrict__ src,
                              D *dst) {
  MPSW_GRID_LOOP(t, (long long)n * B) {
    const int i = (int)(t / B), b = (int)(t - (long long)i * B);
    dst[(size_t)perm[i] * B + b] = D(src[t]);
  }
}
// dst[i][b] = src[new(i)][b]
template <typename S, typename D>
__global__ void k_to_reference(int n, int B, const int *__restrict__ perm, const S *__restrict__ src,
                               D *dst) {
  MPSW_GRID_LOOP(t, (long long)n * B) {
    const int i = (int)(t / B), b = (int)(t - (long long)i * B);
    dst[t] = D(src[(size_t)perm[i] * B + b]);
  }
}
template <typename S, typename D>
__global__ void k_convert(long long n, const S *__restrict__ src, D *dst) {
  MPSW_GRID_LOOP(t, n) dst[t] = D(src[t]);
}

// Rounds up to kConvMax double arrays to float in one launch (linearisation point of a stage).
// dst = float(src - off): reduced-precision h relative to a reference depth
static __global__ void k_convert_off(long long n, const double *src, double off, float *dst) {
  MPSW_GRID_LOOP(t, n) dst[t] = float(src[t] - off);
}

static __global__ void k_convert_list(ConvList L) {
  pdl_begin();  // also when the list is empty
  for (int i = 0; i < L.count; i++) {
    const double *__restrict__ s = L.src[i];
    float *__restrict__ d = L.dst[i];
    double *__restrict__ d64 = L.dst64[i];
    MPSW_GRID_LOOP(t, L.n[i]) {
      const double x = s[t];
      if (d) d[t] = float(x);
      if (d64) d64[t] = x;
    }
  }
}

}  // namespace mpsw
