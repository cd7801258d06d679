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

#define MPSW_GRID_LOOP(t, total)                                                         \
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)(total); \
       t += (long long)gridDim.x * blockDim.x)

template <typename R>
__device__ __forceinline__ R ld(const R *p, size_t i) {
  return __ldg(p + i);
}

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
template <typename R, typename A>
__global__ void k_fwd_cell(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                           Diag<R> d, RK<R, A> rk, R *tend_h) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, nC) {
    const int c = (int)t;
    const int n = ld(m.c_n, c);
    R div = R(0), th = R(0);
    for (int k = 0; k < n; k++) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R s = R(m.c_esg[(size_t)k * nC + c]);
      const R ue = ld(u, e), dve = ld(m.e_dv, e);
      div = div + s * (ue * dve);
      const R he = R(0.5) * ((ld(h, ld(m.e_c1, e)) + off) + (ld(h, ld(m.e_c2, e)) + off));
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
    ke = ke / area;
    R pc = R(0), vc = R(0);
    for (int k = 0; k < n; k++) {
      const int v = ld(m.c_vs, (size_t)k * nC + c);
      const R kt = ld(m.c_vk, (size_t)k * nC + c);
      pc = pc + (kt * d.pvv[v]) / area;
      if (d.vc) vc = vc + (kt * d.vort[v]) / area;
    }
    th = th / area;
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
template <typename R>
__global__ void k_fwd_edge_diag(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                                Diag<R> d, Phys<R> ph) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, nE) {
    const int e = (int)t;
    const int n = ld(m.e_n, e);
    R v = R(0);
    for (int j = 0; j < n; j++)
      v = v + ld(m.e_w, (size_t)j * nE + e) * ld(u, ld(m.e_eoe, (size_t)j * nE + e));
    const int v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e), c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
    const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
    const R gpt = (d.pvv[v2] - d.pvv[v1]) / dv;
    R pe = R(0);
    pe = pe + R(0.5) * d.pvv[ld(m.e_va, e)];
    pe = pe + R(0.5) * d.pvv[ld(m.e_vb, e)];
    pe = pe - ((ph.apvm * v) * ph.dt) * gpt;
    const R gpn = (d.pc[c2] - d.pc[c1]) / dc;
    pe = pe - ((ph.apvm * ld(u, e)) * ph.dt) * gpn;
    d.pe[e] = pe;
    d.he[e] = R(0.5) * ((ld(h, c1) + off) + (ld(h, c2) + off));
    if (d.v) d.v[e] = v;
    if (d.gpt) d.gpt[e] = gpt;
    if (d.gpn) d.gpn[e] = gpn;
    if (d.dsq_u) d.dsq_u[e] = (d.div[c2] - d.div[c1]) / dc - (d.vort[v2] - d.vort[v1]) / dv;
  }
}

// del4 intermediates (:554-589): delsq_vorticity on vertices, delsq_divergence on cells, for
// B members.  One grid covers the V*B vertex threads followed by the N*B cell threads.
template <typename R>
__global__ void k_del4_vc(MeshDev<R> m, int B, const R *__restrict__ dsq_u, R *dsq_vort,
                          R *dsq_div) {
  const int nV = m.nV, nC = m.nC;
  const long long tv = (long long)nV * B;
  MPSW_GRID_LOOP(t, tv + (long long)nC * B) {
    if (t < tv) {
      const int v = (int)(t / B), b = (int)(t - (long long)v * B);
      R dcirc = R(0);
#pragma unroll
      for (int k = 0; k < VDEG; k++) {
        const int e = ld(m.v_es, (size_t)k * nV + v);
        const R s = R(m.v_esg[(size_t)k * nV + v]);
        dcirc = dcirc + s * (ld(m.e_dc, e) * dsq_u[(size_t)e * B + b]);
      }
      dsq_vort[(size_t)v * B + b] = dcirc * (R(1) / ld(m.v_area, v));
    } else {
      const long long t2 = t - tv;
      const int c = (int)(t2 / B), b = (int)(t2 - (long long)c * B);
      const int n = ld(m.c_n, c);
      R dd = R(0);
      for (int k = 0; k < n; k++) {
        const int e = ld(m.c_es, (size_t)k * nC + c);
        const R s = R(m.c_esg[(size_t)k * nC + c]);
        dd = dd + s * (dsq_u[(size_t)e * B + b] * ld(m.e_dv, e));
      }
      dsq_div[(size_t)c * B + b] = dd * (R(1) / ld(m.c_area, c));
    }
  }
}

// Normal-velocity tendency (src/mpas_sw_dyncore.f90:485-637) and its RK update.
template <typename R, typename A>
__global__ void k_fwd_edge_tend(MeshDev<R> m, const R *__restrict__ u, const R *__restrict__ h, R off,
                                Diag<R> d, Phys<R> ph, RK<R, A> rk, R *tend_u) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, nE) {
    const int e = (int)t;
    const int n = ld(m.e_n, e);
    const R pee = d.pe[e];
    R q = R(0);
    for (int j = 0; j < n; j++) {
      const int eoe = ld(m.e_eoe, (size_t)j * nE + e);
      const R wpv = R(0.5) * (pee + d.pe[eoe]);
      q = q + ((ld(m.e_w, (size_t)j * nE + e) * ld(u, eoe)) * wpv) * d.he[eoe];
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
    if (ph.wind) tu = tu + (ld(m.e_usrc, e) / R(RHO_REF)) / d.he[e];
    if (ph.drag) {
      const R kee = R(0.5) * (d.ke[c1] + d.ke[c2]);
      tu = tu - ((R(1.0e-3) * ld(u, e)) * sqrt(R(2) * kee)) / d.he[e];
    }
    if (tend_u) tend_u[e] = tu;
    if (rk.next) rk.next[e] = rk.frozen ? R(rk.x0[e]) : R(rk.x0[e] + rk.c * A(tu));
    if (rk.acc_out && !rk.frozen) rk.acc_out[e] = rk.acc_in[e] + rk.w * A(tu);
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

// ----------------------------------------------------------------------------------------
// Tangent linear (src/mpas_sw_dyncore_tlm.f90), B members about one stored linearisation
// point.  Member arrays are [n][B]; base arrays are [n].
// ----------------------------------------------------------------------------------------

// :255-271 and :344-360
template <typename R>
__global__ void k_tl_vertex(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                            const R *__restrict__ ht, Diag<R> d) {
  const int nV = m.nV;
  MPSW_GRID_LOOP(t, (long long)nV * B) {
    const int v = (int)(t / B), b = (int)(t - (long long)v * B);
    R circ = R(0);
#pragma unroll
    for (int k = 0; k < VDEG; k++) {
      const int e = ld(m.v_es, (size_t)k * nV + v);
      const R s = R(m.v_esg[(size_t)k * nV + v]);
      circ = circ + s * (ld(m.e_dc, e) * ut[(size_t)e * B + b]);
    }
    const R area = ld(m.v_area, v);
    const R vort = circ / area;
    R hvt = R(0);
#pragma unroll
    for (int k = 0; k < VDEG; k++)
      hvt = hvt + ht[(size_t)ld(m.v_c, (size_t)k * nV + v) * B + b] * ld(m.v_k, (size_t)k * nV + v);
    hvt = hvt / area;
    const R hv = ld(bs.hv, v);
    const R pvt = vort / hv - (hvt * (ld(m.v_f, v) + ld(bs.vort, v))) / (hv * hv);
    const size_t o = (size_t)v * B + b;
    if (d.circ) d.circ[o] = circ;
    d.vort[o] = vort;
    if (d.hv) d.hv[o] = hvt;
    d.pvv[o] = pvt;
  }
}

// :274-316, :397-421, tendency :541-561 and the RK update
template <typename R, typename A>
__global__ void k_tl_cell(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                          const R *__restrict__ ht, Diag<R> d, RK<R, A> rk, R *tend_h) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, (long long)nC * B) {
    const int c = (int)(t / B), b = (int)(t - (long long)c * B);
    const int n = ld(m.c_n, c);
    R div = R(0), th = R(0);
    for (int k = 0; k < n; k++) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R s = R(m.c_esg[(size_t)k * nC + c]);
      const R ue = ut[(size_t)e * B + b], dve = ld(m.e_dv, e);
      div = div + s * (ue * dve);
      const R het = R(0.5) * (ht[(size_t)ld(m.e_c1, e) * B + b] + ht[(size_t)ld(m.e_c2, e) * B + b]);
      const R flux = (ue * dve) * ld(bs.he, e) + (ld(bs.u, e) * dve) * het;
      th = th + (-s) * flux;
    }
    const R area = ld(m.c_area, c);
    div = div * (R(1) / area);
    R ke = R(0);
    for (int i = 0; i < n; i++) {
      const int e = ld(m.c_eoc, (size_t)i * nC + c);
      ke = ke + ((R(0.25) * ld(m.e_dc, e)) * ld(m.e_dv, e)) * ((R(2) * ld(bs.u, e)) * ut[(size_t)e * B + b]);
    }
    ke = ke / area;
    R pc = R(0), vc = R(0);
    for (int k = 0; k < n; k++) {
      const int v = ld(m.c_vs, (size_t)k * nC + c);
      const R kt = ld(m.c_vk, (size_t)k * nC + c);
      pc = pc + (kt * d.pvv[(size_t)v * B + b]) / area;
      if (d.vc) vc = vc + (kt * d.vort[(size_t)v * B + b]) / area;
    }
    th = th / area;
    const size_t o = (size_t)c * B + b;
    d.div[o] = div;
    d.ke[o] = ke;
    d.pc[o] = pc;
    if (d.vc) d.vc[o] = vc;
    if (tend_h) tend_h[o] = th;
    if (rk.next) rk.next[o] = R(rk.x0[o] + rk.c * A(th));
    if (rk.acc_out) rk.acc_out[o] = rk.acc_in[o] + rk.w * A(th);
  }
}

// :319-329, :364-393, :425-445, h_edge_tl :117-126, delsq_u_tl :638-652
template <typename R>
__global__ void k_tl_edge_diag(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d, Phys<R> ph) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, (long long)nE * B) {
    const int e = (int)(t / B), b = (int)(t - (long long)e * B);
    const int n = ld(m.e_n, e);
    R vt = R(0);
    for (int j = 0; j < n; j++)
      vt = vt + ld(m.e_w, (size_t)j * nE + e) * ut[(size_t)ld(m.e_eoe, (size_t)j * nE + e) * B + b];
    const int v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e), c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
    const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
    const R gptt = (d.pvv[(size_t)v2 * B + b] - d.pvv[(size_t)v1 * B + b]) / dv;
    R pet = R(0);
    pet = pet + R(0.5) * d.pvv[(size_t)ld(m.e_va, e) * B + b];
    pet = pet + R(0.5) * d.pvv[(size_t)ld(m.e_vb, e) * B + b];
    pet = pet - ((ph.apvm * vt) * ph.dt) * ld(bs.gpt, e) - ((ph.apvm * ld(bs.v, e)) * ph.dt) * gptt;
    const R gpnt = (d.pc[(size_t)c2 * B + b] - d.pc[(size_t)c1 * B + b]) / dc;
    const R uet = ut[(size_t)e * B + b];
    pet = pet - ((ph.apvm * uet) * ph.dt) * ld(bs.gpn, e) - ((ph.apvm * ld(bs.u, e)) * ph.dt) * gpnt;
    const size_t o = (size_t)e * B + b;
    d.pe[o] = pet;
    d.he[o] = R(0.5) * (ht[(size_t)c1 * B + b] + ht[(size_t)c2 * B + b]);
    if (d.v) d.v[o] = vt;
    if (d.gpt) d.gpt[o] = gptt;
    if (d.gpn) d.gpn[o] = gpnt;
    if (d.dsq_u)
      d.dsq_u[o] = (d.div[(size_t)c2 * B + b] - d.div[(size_t)c1 * B + b]) / dc -
                   (d.vort[(size_t)v2 * B + b] - d.vort[(size_t)v1 * B + b]) / dv;
  }
}

// sw_compute_tend_tlm normal-velocity part :564-768 and the RK update
template <typename R, typename A>
__global__ void k_tl_edge_tend(MeshDev<R> m, int B, Base<R> bs, const R *__restrict__ ut,
                               const R *__restrict__ ht, Diag<R> d, Phys<R> ph, RK<R, A> rk,
                               R *tend_u) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, (long long)nE * B) {
    const int e = (int)(t / B), b = (int)(t - (long long)e * B);
    const int n = ld(m.e_n, e);
    const R pet_e = d.pe[(size_t)e * B + b], pe_e = ld(bs.pe, e);
    R qt = R(0);
    for (int j = 0; j < n; j++) {
      const int eoe = ld(m.e_eoe, (size_t)j * nE + e);
      const R w = ld(m.e_w, (size_t)j * nE + e);
      const R wpvt = R(0.5) * (pet_e + d.pe[(size_t)eoe * B + b]);
      const R wpv = R(0.5) * (pe_e + ld(bs.pe, eoe));
      const R ub = ld(bs.u, eoe), heb = ld(bs.he, eoe);
      qt = qt + ((w * ut[(size_t)eoe * B + b]) * wpv) * heb + ((w * ub) * wpvt) * heb +
           ((w * ub) * wpv) * d.he[(size_t)eoe * B + b];
    }
    const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e), v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e);
    const R dc = ld(m.e_dc, e), dv = ld(m.e_dv, e);
    R tut = qt - ((d.ke[(size_t)c2 * B + b] - d.ke[(size_t)c1 * B + b]) +
                  R(GRAVITY) * (ht[(size_t)c2 * B + b] - ht[(size_t)c1 * B + b])) / dc;
    if (ph.visc2 > R(0)) {
      R ud = (d.div[(size_t)c2 * B + b] - d.div[(size_t)c1 * B + b]) / dc -
             (d.vort[(size_t)v2 * B + b] - d.vort[(size_t)v1 * B + b]) / dv;
      ud = (ld(m.e_sc2, e) * ph.visc2) * ud;
      tut = tut + ud;
    }
    if (ph.visc4 > R(0)) {
      R ud = (d.dsq_div[(size_t)c2 * B + b] - d.dsq_div[(size_t)c1 * B + b]) / dc -
             (d.dsq_vort[(size_t)v2 * B + b] - d.dsq_vort[(size_t)v1 * B + b]) / dv;
      ud = (ld(m.e_sc4, e) * ph.visc4) * ud;
      tut = tut - ud;
    }
    const R hh = ld(bs.he, e);
    const R het = d.he[(size_t)e * B + b];
    if (ph.wind) tut = tut - ((het * ld(m.e_usrc, e)) / R(RHO_REF)) / (hh * hh);
    if (ph.drag) {
      const R ket_e = R(0.5) * (d.ke[(size_t)c1 * B + b] + d.ke[(size_t)c2 * B + b]);
      const R ke_e = R(0.5) * (ld(bs.ke, c1) + ld(bs.ke, c2));
      const R uu = ld(bs.u, e), sq = sqrt(R(2) * ke_e);
      tut = tut - ((R(1.0e-3) * ut[(size_t)e * B + b]) * sq) / hh -
            ((((R(0.5) * R(1.0e-3)) * uu) * (R(2) * ket_e)) / sq) / hh +
            (((R(1.0e-3) * uu) * sq) * het) / (hh * hh);
    }
    const size_t o = (size_t)e * B + b;
    if (tend_u) tend_u[o] = tut;
    if (rk.next) rk.next[o] = rk.frozen ? R(rk.x0[o]) : R(rk.x0[o] + rk.c * A(tut));
    if (rk.acc_out && !rk.frozen) rk.acc_out[o] = rk.acc_in[o] + rk.w * A(tut);
  }
}

// ----------------------------------------------------------------------------------------
// Adjoint of one RK stage (src/mpas_sw_dyncore_adj.f90): sw_compute_tend_adj (:455-738)
// followed by sw_compute_solve_diagnostics_adj (:1-453) at the same linearisation point,
// as gathers.  tend_ad is formed on the fly from the step-output adjoint and the next
// stage's provisional adjoint (src/mpas_sw_module.f90:912-942).
// ----------------------------------------------------------------------------------------
// Tendency adjoint of the last stage of a step (src/mpas_sw_module.f90:912-914 at rk=4):
// tu = wu * x2u + seed_tu, th = (wh * x2h + seed_th) / areaCell.  One grid covers E*B edge
// threads then N*B cell threads.
template <typename R, typename A>
__global__ void k_ad_tinit(MeshDev<R> m, int B, const A *x2u, const A *x2h, const R *seed_tu,
                           const R *seed_th, A wu, A wh, R *tu, R *th) {
  const int nE = m.nE;
  const long long te = (long long)nE * B;
  MPSW_GRID_LOOP(t, te + (long long)m.nC * B) {
    if (t < te) {
      const int e = (int)(t / B);
      A x = x2u ? wu * x2u[t] : A(0);
      if (seed_tu) x = x + A(seed_tu[e]);
      tu[t] = R(x);
    } else {
      const long long t2 = t - te;
      const int c = (int)(t2 / B);
      A x = x2h ? wh * x2h[t2] : A(0);
      if (seed_th) x = x + A(seed_th[c]);
      th[t2] = R(x / A(ld(m.c_area, c)));
    }
  }
}

// Edge stage: workpv/q adjoint (:689-718) as a gather over the transposed edgesOnEdge,
// thickness-flux adjoint (:720-736), drag (:549-565), wind (:567-572), then the APVM adjoints
// of the diagnostics (:193-200, :235-242).
template <typename R, typename A>
__global__ void k_ad_edge(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                          AdWork<R> w) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, (long long)nE * B) {
    const int e = (int)(t / B), b = (int)(t - (long long)e * B);
    const int n = ld(m.e_n, e);
    const R Te = in.tu[(size_t)e * B + b];
    const R ue = ld(bs.u, e), hee = ld(bs.he, e), pee = ld(bs.pe, e);
    R pe_ad = R(0), he_ad = R(0), ud = R(0);
    for (int j = 0; j < n; j++) {
      const int nb = ld(m.e_eoe, (size_t)j * nE + e);
      const R wj = ld(m.e_w, (size_t)j * nE + e);
      const R wr = ld(m.e_wrev, (size_t)j * nE + e);
      pe_ad = pe_ad + R(0.5) * (((wj * ld(bs.u, nb)) * ld(bs.he, nb)) * Te);
      const R Tn = in.tu[(size_t)nb * B + b];
      const R wpv = R(0.5) * (ld(bs.pe, nb) + pee);
      he_ad = he_ad + ((wr * ue) * wpv) * Tn;
      pe_ad = pe_ad + R(0.5) * (((wr * ue) * hee) * Tn);
      ud = ud + ((wr * wpv) * hee) * Tn;
    }
    const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e);
    const R dv = ld(m.e_dv, e);
    const R fa = in.th[(size_t)c2 * B + b] - in.th[(size_t)c1 * B + b];
    he_ad = he_ad + (ue * dv) * fa;
    ud = ud + (dv * hee) * fa;
    if (ph.drag) {
      const R sq = sqrt(R(2) * (R(0.5) * (ld(bs.ke, c1) + ld(bs.ke, c2))));
      he_ad = he_ad + (((R(1.0e-3) * ue) * sq) / (hee * hee)) * Te;
      ud = ud - ((R(1.0e-3) * sq) / hee) * Te;
    }
    if (ph.wind) he_ad = he_ad - ((ld(m.e_usrc, e) / R(RHO_REF)) / (hee * hee)) * Te;
    R gpn_ad = R(0), gpt_ad = R(0), v_ad = R(0);
    if (sd.pe) pe_ad = pe_ad + sd.pe[e];
    if (sd.he) he_ad = he_ad + sd.he[e];
    if (sd.gpn) gpn_ad = sd.gpn[e];
    if (sd.gpt) gpt_ad = sd.gpt[e];
    if (sd.v) v_ad = sd.v[e];
    gpn_ad = gpn_ad - ((ph.apvm * ue) * ph.dt) * pe_ad;
    ud = ud - ((ph.apvm * ph.dt) * ld(bs.gpn, e)) * pe_ad;
    gpt_ad = gpt_ad - ((ph.apvm * ld(bs.v, e)) * ph.dt) * pe_ad;
    v_ad = v_ad - ((ph.apvm * ph.dt) * ld(bs.gpt, e)) * pe_ad;
    const size_t o = (size_t)e * B + b;
    w.pe_ad[o] = pe_ad;
    w.he_ad[o] = he_ad;
    w.ud[o] = ud;
    w.gpn_ad[o] = gpn_ad;
    w.gpt_ad[o] = gpt_ad;
    w.v_ad[o] = v_ad;
  }
}

// del4 adjoint, first half (:588-634): delsq_vorticity/delsq_circulation adjoint on vertices
// and delsq_divergence adjoint on cells.
template <typename R, typename A>
__global__ void k_ad_del4_vc(MeshDev<R> m, int B, Phys<R> ph, AdIn<R> in, AdWork<R> w) {
  const int nV = m.nV, nC = m.nC;
  const long long tv = (long long)nV * B;
  MPSW_GRID_LOOP(t, tv + (long long)nC * B) {
    if (t < tv) {
      const int v = (int)(t / B), b = (int)(t - (long long)v * B);
      R acc = R(0);
#pragma unroll
      for (int k = 0; k < VDEG; k++) {
        const int e = ld(m.v_es, (size_t)k * nV + v);
        const R sg = R(m.v_esg[(size_t)k * nV + v]);
        const R ud4 = (ld(m.e_sc4, e) * ph.visc4) * (-in.tu[(size_t)e * B + b]);
        acc = acc + (-sg) * (ud4 / ld(m.e_dv, e));
      }
      w.dc_ad[(size_t)v * B + b] = acc * (R(1) / ld(m.v_area, v));
    } else {
      const long long t2 = t - tv;
      const int c = (int)(t2 / B), b = (int)(t2 - (long long)c * B);
      const int n = ld(m.c_n, c);
      R acc = R(0);
      for (int k = 0; k < n; k++) {
        const int e = ld(m.c_es, (size_t)k * nC + c);
        const R sg = R(m.c_esg[(size_t)k * nC + c]);
        const R ud4 = (ld(m.e_sc4, e) * ph.visc4) * (-in.tu[(size_t)e * B + b]);
        acc = acc + (-sg) * (ud4 / ld(m.e_dc, e));
      }
      w.dd_ad[(size_t)c * B + b] = acc * (R(1) / ld(m.c_area, c));
    }
  }
}

// del4 adjoint, second half (:617-643): delsq_u adjoint on edges.
template <typename R>
__global__ void k_ad_del4_e(MeshDev<R> m, int B, AdWork<R> w) {
  const int nE = m.nE;
  MPSW_GRID_LOOP(t, (long long)nE * B) {
    const int e = (int)(t / B), b = (int)(t - (long long)e * B);
    const R dv = ld(m.e_dv, e), dc = ld(m.e_dc, e);
    R du = R(0);
    du = du - dv * w.dd_ad[(size_t)ld(m.e_c2, e) * B + b];
    du = du + dv * w.dd_ad[(size_t)ld(m.e_c1, e) * B + b];
    du = du + dc * w.dc_ad[(size_t)ld(m.e_v2, e) * B + b];
    du = du - dc * w.dc_ad[(size_t)ld(m.e_v1, e) * B + b];
    w.du_ad[(size_t)e * B + b] = du;
  }
}

// Cell stage: gradPVn adjoint onto pv_cell (:202-213), gravity/ke terms of the tendency
// adjoint (:696-699), drag ke terms, del2/del4 divergence adjoints, h_edge adjoint (:358-369),
// then the 1/areaCell scalings of ke_ad and divergence_ad (:306-326).
template <typename R, typename A>
__global__ void k_ad_cell(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in, AdSeeds<R> sd,
                          AdWork<R> w) {
  const int nC = m.nC;
  MPSW_GRID_LOOP(t, (long long)nC * B) {
    const int c = (int)(t / B), b = (int)(t - (long long)c * B);
    const int n = ld(m.c_n, c);
    R pc_ad = sd.pc ? sd.pc[c] : R(0);
    R ke_ad = sd.ke ? sd.ke[c] : R(0);
    R div_ad = sd.div ? sd.div[c] : R(0);
    R hd = R(0);
    for (int k = 0; k < n; k++) {
      const int e = ld(m.c_es, (size_t)k * nC + c);
      const R sg = R(m.c_esg[(size_t)k * nC + c]);
      const size_t oe = (size_t)e * B + b;
      const R Te = in.tu[(size_t)e * B + b];
      const R dce = ld(m.e_dc, e);
      pc_ad = pc_ad + (-sg) * (w.gpn_ad[oe] / dce);
      ke_ad = ke_ad + sg * (Te / dce);
      hd = hd + sg * ((R(GRAVITY) / dce) * Te);
      if (ph.drag) {
        const R sq = sqrt(R(2) * (R(0.5) * (ld(bs.ke, ld(m.e_c1, e)) + ld(bs.ke, ld(m.e_c2, e)))));
        const R kea = -(((((R(0.5) * R(1.0e-3)) * ld(bs.u, e)) * R(2)) / sq) / ld(bs.he, e)) * Te;
        ke_ad = ke_ad + R(0.5) * kea;
      }
      if (ph.visc2 > R(0)) {
        const R ud2 = (ld(m.e_sc2, e) * ph.visc2) * Te;
        div_ad = div_ad + (-sg) * (ud2 / dce);
      }
      if (ph.visc4 > R(0)) div_ad = div_ad + (-sg) * (w.du_ad[oe] / dce);
      hd = hd + R(0.5) * w.he_ad[oe];
    }
    const R area = ld(m.c_area, c);
    const size_t o = (size_t)c * B + b;
    w.pc_ad[o] = pc_ad;
    w.ke_ad[o] = ke_ad / area;
    w.div_ad[o] = div_ad * (R(1) / area);
    w.hd[o] = hd;
  }
}

// Vertex stage: pv_cell -> pv_vertex (:215-229), pv_edge -> pv_vertex (:244-252),
// gradPVt -> pv_vertex (:254-262), del2/del4 vorticity adjoints, pv_vertex -> h_vertex and
// vorticity (:268-284), vorticity -> circulation (:343-349).
template <typename R, typename A>
__global__ void k_ad_vertex(MeshDev<R> m, int B, Base<R> bs, Phys<R> ph, AdIn<R> in,
                            AdSeeds<R> sd, AdWork<R> w) {
  const int nV = m.nV;
  MPSW_GRID_LOOP(t, (long long)nV * B) {
    const int v = (int)(t / B), b = (int)(t - (long long)v * B);
    R pvv_ad = sd.pvv ? sd.pvv[v] : R(0);
    R vort_ad = sd.vort ? sd.vort[v] : R(0);
#pragma unroll
    for (int i = 0; i < VDEG; i++) {
      const int c = ld(m.v_c, (size_t)i * nV + v);
      const R ka = ld(m.v_k, (size_t)i * nV + v) / ld(m.c_area, c);
      if (sd.vc) vort_ad = vort_ad + ka * sd.vc[c];
      pvv_ad = pvv_ad + ka * w.pc_ad[(size_t)c * B + b];
    }
#pragma unroll
    for (int i = 0; i < VDEG; i++)
      pvv_ad = pvv_ad + R(0.5) * w.pe_ad[(size_t)ld(m.v_e, (size_t)i * nV + v) * B + b];
#pragma unroll
    for (int k = 0; k < VDEG; k++) {
      const int e = ld(m.v_es, (size_t)k * nV + v);
      const R sg = R(m.v_esg[(size_t)k * nV + v]);
      const R dve = ld(m.e_dv, e);
      const size_t oe = (size_t)e * B + b;
      pvv_ad = pvv_ad + sg * (w.gpt_ad[oe] / dve);
      if (ph.visc2 > R(0)) {
        const R ud2 = (ld(m.e_sc2, e) * ph.visc2) * in.tu[(size_t)e * B + b];
        vort_ad = vort_ad + (-sg) * (ud2 / dve);
      }
      if (ph.visc4 > R(0)) vort_ad = vort_ad + (-sg) * (w.du_ad[oe] / dve);
    }
    const R hv = ld(bs.hv, v), area = ld(m.v_area, v);
    R hv_ad = sd.hv ? sd.hv[v] : R(0);
    hv_ad = hv_ad - ((ld(m.v_f, v) + ld(bs.vort, v)) / (hv * hv)) * pvv_ad;
    vort_ad = vort_ad + pvv_ad / hv;
    hv_ad = hv_ad / area;
    const R circ_ad = (sd.circ ? sd.circ[v] : R(0)) + vort_ad / area;
    const size_t o = (size_t)v * B + b;
    w.hv_ad[o] = hv_ad;
    w.circ_ad[o] = circ_ad;
  }
}

template <typename R, typename A>
__device__ __forceinline__ void ad_emit(const AdOut<R, A> &out, int is_edge, size_t o, R pad, R area) {
  A *acc = is_edge ? out.acc_u : out.acc_h;
  const A *x2 = is_edge ? out.x2u : out.x2h;
  R *tn = is_edge ? out.tu_next : out.th_next;
  const A wn = is_edge ? out.wu : out.wh, cn = is_edge ? out.cu : out.ch;
  A next;
  if (out.mode == AD_FINAL) {
    A *dst = is_edge ? out.dst_u : out.dst_h;
    const A d = (acc[o] + x2[o]) + A(pad);
    dst[o] = d;
    next = wn * d;
  } else {
    if (out.mode == AD_SET) acc[o] = A(pad);
    else acc[o] = acc[o] + A(pad);
    next = (x2 ? wn * x2[o] : A(0)) + cn * A(pad);
  }
  if (tn) tn[o] = is_edge ? R(next) : R(next / A(area));
}

// Final stage of the adjoint: h_vertex -> h (:286-289) on cells, and on edges the transposed
// tangential velocity (:296-303), ke (:306-317), divergence (:327-340) and circulation
// (:350-355) adjoints.  One grid covers N*B cell threads then E*B edge threads.
template <typename R, typename A>
__global__ void k_ad_final(MeshDev<R> m, int B, Base<R> bs, AdWork<R> w, AdOut<R, A> out) {
  const int nC = m.nC, nE = m.nE;
  const long long tc = (long long)nC * B;
  MPSW_GRID_LOOP(t, tc + (long long)nE * B) {
    if (t < tc) {
      const int c = (int)(t / B), b = (int)(t - (long long)c * B);
      const int n = ld(m.c_n, c);
      R ph_ = w.hd[(size_t)c * B + b];
      for (int k = 0; k < n; k++)
        ph_ = ph_ + ld(m.c_vk, (size_t)k * nC + c) * w.hv_ad[(size_t)ld(m.c_vs, (size_t)k * nC + c) * B + b];
      ad_emit(out, 0, (size_t)c * B + b, ph_, ld(m.c_area, c));
    } else {
      const long long t2 = t - tc;
      const int e = (int)(t2 / B), b = (int)(t2 - (long long)e * B);
      const int n = ld(m.e_n, e);
      R pu = w.ud[(size_t)e * B + b];
      for (int j = 0; j < n; j++) {
        const int nb = ld(m.e_eoe, (size_t)j * nE + e);
        pu = pu + ld(m.e_wrev, (size_t)j * nE + e) * w.v_ad[(size_t)nb * B + b];
      }
      const int c1 = ld(m.e_c1, e), c2 = ld(m.e_c2, e), v1 = ld(m.e_v1, e), v2 = ld(m.e_v2, e);
      const R dc = ld(m.e_dc, e), dv = ld(m.e_dv, e);
      const R kc = (((R(0.25) * dc) * dv) * R(2)) * ld(bs.u, e);
      pu = pu + kc * w.ke_ad[(size_t)c1 * B + b];
      pu = pu + kc * w.ke_ad[(size_t)c2 * B + b];
      pu = pu - dv * w.div_ad[(size_t)c2 * B + b];
      pu = pu + dv * w.div_ad[(size_t)c1 * B + b];
      pu = pu + dc * w.circ_ad[(size_t)v2 * B + b];
      pu = pu - dc * w.circ_ad[(size_t)v1 * B + b];
      ad_emit(out, 1, (size_t)e * B + b, pu, R(1));
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
static __global__ void k_convert_list(ConvList L) {
  for (int i = 0; i < L.count; i++) {
    const double *__restrict__ s = L.src[i];
    float *__restrict__ d = L.dst[i];
    MPSW_GRID_LOOP(t, L.n[i]) d[t] = float(s[t]);
  }
}

}  // namespace mpsw
