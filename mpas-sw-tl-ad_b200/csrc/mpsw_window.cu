// Batched tangent-linear / adjoint window of the engine (mpsw_window_* in include/mpsw.h).
//
// One nonlinear trajectory (FP64) is shared by B members that ride the trailing dimension of
// the member arrays.  Per RK stage the trajectory's diagnostics (the linearisation point) are
// computed once and read by all members; in precision 1 they are rounded to FP32 once per
// stage and the member stencils run in FP32 while the members' RK4 states and accumulators
// stay in FP64.
//
// Storage of the trajectory: checkpoints every `every` steps; the adjoint sweep replays one
// segment at a time from its checkpoint (two-level checkpointing: one extra forward pass in
// total) and recomputes the four RK stages of each step before its adjoint, as
// src/mpas_sw_module.f90:815-878 does inside sw_rk4_adj.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cstdio>
#include <string>
#include <cstring>

#include "mpsw.h"
#include "mpsw_engine.h"
#include "mpsw_launch.h"

namespace mpsw {

namespace {

using L64 = Launch<double, double>;

template <typename R>
struct MemberBufs {
  Diag<R> d{};
  // tangent-linear provisional states of stages 2-4 (pu / ph [0..2]) and, for FP32 members, the
  // step's rounded input state (pu / ph [3]): the tangent-linear members', which stages 1-3 form
  // their provisional states from, or in adjoint sweeps the adjoint state's, which stages 4-2
  // form the next tendency adjoint from
  R *pu[4] = {}, *ph[4] = {};
  AdWork<R> w{};
  R *pad_u[2] = {}, *pad_h[2] = {};
  // per-stage tendencies (tangent linear) or contributions (adjoint) of the first three stages
  // of a step, summed into the FP64 members by its last stage
  R *tk_u[3] = {}, *tk_h[3] = {};
};

template <typename R>
R *walloc(Window::Members &M, size_t n, cudaStream_t s) {
  void *p = nullptr;
  cuda_check(cudaMalloc(&p, sizeof(R) * (n ? n : 1)), "cudaMalloc window");
  cuda_check(cudaMemsetAsync(p, 0, sizeof(R) * (n ? n : 1), s), "memset window");
  M.mem.push_back(p);
  return (R *)p;
}

template <typename R>
void free_members(Window::Members &M) {
  for (void *p : M.mem) cudaFree(p);
  M.mem.clear();
  delete (MemberBufs<R> *)M.bufs;
  M.bufs = nullptr;
  M.B = 0;
  M.acc_u = M.acc_h = nullptr;
  M.x_u = M.x_h = nullptr;
}

template <typename R>
MemberBufs<R> *members(Engine &E, int prec, int B, cudaStream_t s) {
  Window::Members &M = E.win.ms[prec];
  if (M.bufs && M.B >= B) return (MemberBufs<R> *)M.bufs;
  E.graphs_free();  // captured steps point at the buffers about to be replaced
  free_members<R>(M);
  auto *mb = new MemberBufs<R>();
  const size_t C = (size_t)E.nC * B, Ed = (size_t)E.nE * B, V = (size_t)E.nV * B;
  Diag<R> &d = mb->d;
  d.circ = nullptr;
  d.vort = walloc<R>(M, V, s); d.hv = nullptr; d.pvv = walloc<R>(M, V, s);
  d.div = walloc<R>(M, C, s); d.ke = walloc<R>(M, C, s); d.pc = walloc<R>(M, C, s); d.vc = nullptr;
  d.gpt = nullptr; d.gpn = nullptr;
  d.pe = walloc<R>(M, Ed, s); d.he = walloc<R>(M, Ed, s);
  // FP32 members keep the tangent PV flux in d.v (read by tl_edge_tend); FP64 needs no v'
  d.v = sizeof(R) == 4 ? walloc<R>(M, Ed, s) : nullptr;
  d.dsq_u = walloc<R>(M, Ed, s); d.dsq_vort = walloc<R>(M, V, s); d.dsq_div = walloc<R>(M, C, s);
  for (int k = 0; k < 4; k++) {
    mb->pu[k] = walloc<R>(M, Ed, s);
    mb->ph[k] = walloc<R>(M, C, s);
  }
  AdWork<R> &w = mb->w;
  w.pe_ad = walloc<R>(M, Ed, s); w.he_ad = walloc<R>(M, Ed, s); w.ud = walloc<R>(M, Ed, s);
  // gradPVn_ad, gradPVt_ad, v_ad: re-formed from pv_edge_ad by their readers (no seeds here)
  w.gpn_ad = nullptr; w.gpt_ad = nullptr; w.v_ad = nullptr;
  w.du_ad = walloc<R>(M, Ed, s);
  w.pc_ad = walloc<R>(M, C, s); w.ke_ad = walloc<R>(M, C, s); w.div_ad = walloc<R>(M, C, s);
  w.hd = walloc<R>(M, C, s); w.dd_ad = walloc<R>(M, C, s);
  w.hv_ad = walloc<R>(M, V, s); w.circ_ad = walloc<R>(M, V, s); w.dc_ad = walloc<R>(M, V, s);
  for (int k = 0; k < 2; k++) {
    mb->pad_u[k] = walloc<R>(M, Ed, s);
    mb->pad_h[k] = walloc<R>(M, C, s);
  }
  for (int k = 0; k < 3; k++) {
    mb->tk_u[k] = walloc<R>(M, Ed, s);
    mb->tk_h[k] = walloc<R>(M, C, s);
  }
  M.acc_u = walloc<double>(M, Ed, s);
  M.acc_h = walloc<double>(M, C, s);
  M.x_u = walloc<double>(M, Ed, s);
  M.x_h = walloc<double>(M, C, s);
  M.bufs = mb;
  M.B = B;
  return mb;
}

// The member rows a window sweep passes between its kernels.  divergence' and vorticity' feed
// only the del2 / del4 terms, and divergence_ad is zero without them (the sweeps have no
// diagnostic seeds), so without viscosity the kernels neither write nor read those rows.
template <typename R>
Diag<R> tl_rows(const MemberBufs<R> *mb, const Phys<R> &ph) {
  Diag<R> d = mb->d;
  if (!(ph.visc2 > R(0)) && !(ph.visc4 > R(0))) d.div = d.vort = nullptr;
  return d;
}
template <typename R>
AdWork<R> ad_rows(const MemberBufs<R> *mb, const Phys<R> &ph) {
  AdWork<R> w = mb->w;
  if (!(ph.visc2 > R(0)) && !(ph.visc4 > R(0))) w.div_ad = nullptr;
  return w;
}

Base<double> base64(const Window &W, int k) {
  const Diag<double> &d = W.sd[k];
  Base<double> b{};
  b.u = W.su[k]; b.he = d.he; b.v = d.v; b.gpt = d.gpt; b.gpn = d.gpn; b.pe = d.pe;
  b.vort = d.vort; b.hv = d.hv; b.ke = d.ke;
  return b;
}

Base<float> base32(const Window &W, int k) {
  const Diag<float> &d = W.sd32[k];
  Base<float> b{};
  b.u = W.su32[k]; b.he = d.he; b.v = d.v; b.gpt = d.gpt; b.gpn = d.gpn; b.pe = d.pe;
  b.vort = d.vort; b.hv = d.hv; b.ke = d.ke;
  return b;
}

template <typename R>
Base<R> base_for(const Window &W, int k);
template <>
Base<double> base_for<double>(const Window &W, int k) { return base64(W, k); }
template <>
Base<float> base_for<float>(const Window &W, int k) { return base32(W, k); }

// Base fields of stage k of step n in the store of precision prec (R is its element type)
template <typename R>
R *store_field(const Window::Store &S, int n, int k, int f) {
  return (R *)S.mem + ((size_t)n * 4 + k) * S.slot + S.off[f];
}
template <typename R>
Base<R> stored_base(const Window &W, int prec, int n, int k) {
  const Window::Store &S = W.st[prec];
  Base<R> b{};
  b.u = store_field<R>(S, n, k, 0); b.he = store_field<R>(S, n, k, 1); b.v = store_field<R>(S, n, k, 2);
  b.gpt = store_field<R>(S, n, k, 3); b.gpn = store_field<R>(S, n, k, 4); b.pe = store_field<R>(S, n, k, 5);
  b.vort = store_field<R>(S, n, k, 6); b.hv = store_field<R>(S, n, k, 7); b.ke = store_field<R>(S, n, k, 8);
  return b;
}

template <typename R>
const MeshDev<R> &mesh_for(const Engine &E);
template <>
const MeshDev<double> &mesh_for<double>(const Engine &E) { return E.m64; }
template <>
const MeshDev<float> &mesh_for<float>(const Engine &E) { return E.m32; }

template <typename R>
Phys<R> phys_as(const Phys<double> &p) {
  Phys<R> q{};
  q.dt = R(p.dt); q.apvm = R(p.apvm); q.visc2 = R(p.visc2); q.visc4 = R(p.visc4);
  q.wind = p.wind; q.drag = p.drag; q.tc1 = p.tc1; q.sphere = p.sphere; q.bad = p.bad;
  return q;
}

void rk_coeffs(double dt, double w[4], double c[4]) {
  w[0] = dt / 6.; w[1] = dt / 3.; w[2] = dt / 3.; w[3] = dt / 6.;
  c[0] = dt / 2.; c[1] = dt / 2.; c[2] = dt; c[3] = 0.;
}

}  // namespace

void Engine::graphs_free() {
  for (auto &g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs.clear();
}

GraphKey Engine::graph_key(int kind, int prec, int B, const void *p1, const void *p2) const {
  const Phys<double> ph = phys();
  GraphKey k;
  k.kind = kind; k.prec = prec; k.B = B; k.p1 = p1; k.p2 = p2;
  k.dt = ph.dt; k.apvm = ph.apvm; k.visc2 = ph.visc2; k.visc4 = ph.visc4;
  k.flags = ph.wind | (ph.drag << 1) | (ph.tc1 << 2) | (ph.sphere << 3);
  return k;
}

void Engine::window_free() {
  Window &W = win;
  graphs_free();
  free_members<double>(W.ms[0]);
  free_members<float>(W.ms[1]);
  window_free_trajectory();
}

void Engine::window_store_free(int prec) {
  Window::Store &S = win.st[prec];
  if (S.mem) {
    graphs_free();
    cudaFree(S.mem);
  }
  S.mem = nullptr;
  S.cap = S.valid = 0;
}

// Storage mode of the next windows: -1 automatic, 0 checkpoints only, or a mask of the
// precisions whose linearisation points are stored (1 FP64, 2 FP32).
void Engine::window_storage(int mode, double max_bytes) {
  if (mode < -1 || mode > 3) throw EngineError(MPSW_ERR_ARG, "storage mode must be -1..3");
  if (max_bytes < 0) throw EngineError(MPSW_ERR_ARG, "storage budget must be >= 0");
  win.store_mode = mode;
  win.store_budget = max_bytes;
  for (int p = 0; p < 2; p++) win.st[p].valid = 0;  // takes effect at the next window_init
}

// (Re)allocate the stores of the precisions the storage mode selects for `nsteps` steps.  In
// automatic mode FP64 and FP32 are both stored when they fit the budget, else FP32 alone when
// it fits, else neither (the sweeps then recompute stages from checkpoints).
void Engine::window_store_alloc(int nsteps) {
  Window &W = win;
  const size_t pad = 64;
  auto up = [&](size_t n) { return (n + pad - 1) / pad * pad; };
  size_t off[9], slot = 0;
  for (int f = 0; f < 9; f++) {
    off[f] = slot;
    slot += up(f < 6 ? (size_t)nE : f < 8 ? (size_t)nV : (size_t)nC);
  }
  const size_t per = (size_t)nsteps * 4 * slot;
  int mask = W.store_mode;
  if (mask < 0) {
    double budget = W.store_budget;
    if (budget <= 0) {
      size_t fr = 0, tot = 0;
      cuda_check(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
      double held = 0;
      for (int p = 0; p < 2; p++)
        if (W.st[p].mem) held += (double)W.st[p].cap * 4 * W.st[p].slot * (p ? 4 : 8);
      budget = 0.4 * ((double)fr + held);
    }
    mask = (double)per * 12 <= budget ? 3 : (double)per * 4 <= budget ? 2 : 0;
  }
  for (int p = 0; p < 2; p++) {
    Window::Store &S = W.st[p];
    S.valid = 0;
    if (!((mask >> p) & 1)) {
      window_store_free(p);
      continue;
    }
    if (!S.mem || S.cap < nsteps || S.slot != slot) {
      window_store_free(p);
      cuda_check(cudaMalloc(&S.mem, per * (p ? sizeof(float) : sizeof(double))), "cudaMalloc window store");
      S.cap = nsteps;
    }
    S.slot = slot;
    for (int f = 0; f < 9; f++) S.off[f] = off[f];
  }
}

void Engine::window_free_trajectory() {
  Window &W = win;
  graphs_free();
  window_store_free(0);
  window_store_free(1);
  for (double *p : W.ck_u) cudaFree(p);
  for (double *p : W.ck_h) cudaFree(p);
  W.ck_u.clear();
  W.ck_h.clear();
  for (double *p : W.sn_u) cudaFree(p);
  for (double *p : W.sn_h) cudaFree(p);
  W.sn_u.clear();
  W.sn_h.clear();
  W.snaps = 0;
  for (void *p : {(void *)W.seg_u, (void *)W.seg_h, (void *)W.fin_u, (void *)W.fin_h, (void *)W.x_u,
                  (void *)W.x_h})
    if (p) cudaFree(p);
  W.seg_u = W.seg_h = W.fin_u = W.fin_h = W.x_u = W.x_h = nullptr;
  for (int k = 0; k < 4; k++) {
    for (double *p : {W.sd[k].circ, W.sd[k].vort, W.sd[k].hv, W.sd[k].pvv, W.sd[k].div, W.sd[k].ke,
                      W.sd[k].pc, W.sd[k].vc, W.sd[k].v, W.sd[k].gpt, W.sd[k].pe, W.sd[k].gpn,
                      W.sd[k].he, W.sd[k].dsq_u, W.sd[k].dsq_vort, W.sd[k].dsq_div})
      if (p) cudaFree(p);
    for (float *p : {W.sd32[k].vort, W.sd32[k].hv, W.sd32[k].ke, W.sd32[k].v, W.sd32[k].gpt,
                     W.sd32[k].pe, W.sd32[k].gpn, W.sd32[k].he, W.su32[k]})
      if (p) cudaFree(p);
    if (k > 0 && W.su[k]) cudaFree(W.su[k]);
    if (W.sh[k]) cudaFree(W.sh[k]);
    W.sd[k] = Diag<double>{};
    W.sd32[k] = Diag<float>{};
    W.su[k] = W.sh[k] = nullptr;
    W.su32[k] = nullptr;
  }
  W.nsteps = W.every = W.nckpt = 0;
}

// One nonlinear FP64 step of the window's trajectory from (x_u, x_h) in place.  The four
// stages' diagnostics and provisional states are left in sd[k] / su[k] (su[0] is the step's
// start state); in precision 1 their base fields are rounded to FP32 (sd32, su32), and with
// store_step >= 0 they are written to that step's slots of the valid stores.  hook(k) runs
// after each stage.
template <typename Hook>
static void traj_step(Engine &E, bool in_place, int prec, Hook &&hook, int store_step = -1) {
  Window &W = E.win;
  const Phys<double> ph = E.phys();
  double w[4], c[4];
  rk_coeffs(ph.dt, w, c);
  double *u0 = W.x_u, *h0 = W.x_h;
  const bool st64 = store_step >= 0 && W.st[0].mem, st32 = store_step >= 0 && W.st[1].mem;
  for (int k = 0; k < 4; k++) {
    W.su[0] = u0;
    const double *ui = W.su[k];
    const double *hi = k == 0 ? h0 : W.sh[k];
    RK<double, double> ru{u0, k == 0 ? u0 : E.acc_u, (k == 3 && in_place) ? u0 : E.acc_u,
                          k < 3 ? W.su[k + 1] : nullptr, c[k], w[k], 0.0, ph.tc1};
    RK<double, double> rh{h0, k == 0 ? h0 : E.acc_h, (k == 3 && in_place) ? h0 : E.acc_h,
                          k < 3 ? W.sh[k + 1] : nullptr, c[k], w[k], 0.0, 0};
    E.fwd_stage(ui, hi, W.sd[k], ph, ru, rh, nullptr, nullptr);
    if (prec == 1 || st64 || st32) {
      ConvList L{};
      const Diag<double> &d = W.sd[k];
      const Diag<float> &f = W.sd32[k];
      const double *src[] = {ui, d.he, d.v, d.gpt, d.gpn, d.pe, d.vort, d.hv, d.ke};
      float *dst[] = {W.su32[k], f.he, f.v, f.gpt, f.gpn, f.pe, f.vort, f.hv, f.ke};
      const long long n[] = {E.nE, E.nE, E.nE, E.nE, E.nE, E.nE, E.nV, E.nV, E.nC};
      for (int i = 0; i < 9; i++) {
        L.src[i] = src[i];
        L.dst[i] = st32 ? store_field<float>(W.st[1], store_step, k, i) : prec == 1 ? dst[i] : nullptr;
        L.dst64[i] = st64 ? store_field<double>(W.st[0], store_step, k, i) : nullptr;
        L.n[i] = n[i];
      }
      L.count = 9;
      convert_list(L, E.nE, E.stream);
    }
    hook(k);
  }
}

// Snapshots of the following windows: 0 two-level checkpointing (default), s > 0 binomial
// reversal with s snapshot slots.
void Engine::window_snapshots(int snapshots) {
  if (snapshots < 0 || snapshots > 4096) throw EngineError(MPSW_ERR_ARG, "snapshots must be 0..4096");
  win.snap_req = snapshots;
}

// Least forward steps T(n, s) to reverse n steps from a held start state with s free snapshot
// slots, and the first advance that attains it (Griewank's binomial checkpointing, by dynamic
// programming over T(n, s) = min_m m + T(n - m, s - 1) + T(m, s), T(1, s) = 0, and with no slot
// T(n, 0) = n (n - 1) / 2: every step recomputed from the start).
static void binomial_tables(int N, int S, std::vector<long long> &T, std::vector<int> &split) {
  if ((double)N * N * S > 4e9) throw EngineError(MPSW_ERR_UNSUPPORTED, "binomial schedule too large: use fewer steps or snapshots");
  const size_t L = (size_t)N + 1;
  T.assign(L * (S + 1), 0);
  split.assign(L * (S + 1), 0);
  for (int s = 0; s <= S; s++)
    for (int n = 2; n <= N; n++) {
      if (s == 0) {
        T[n] = (long long)n * (n - 1) / 2;
        split[n] = n - 1;
        continue;
      }
      long long best = -1;
      int bm = 1;
      for (int m = 1; m < n; m++) {
        const long long c = m + T[(size_t)(s - 1) * L + (n - m)] + T[(size_t)s * L + m];
        if (best < 0 || c < best) {
          best = c;
          bm = m;
        }
      }
      T[(size_t)s * L + n] = best;
      split[(size_t)s * L + n] = bm;
    }
}

void Engine::window_init(int nsteps, int every, cudaStream_t s) {
  if (nsteps < 1 || every < 1) throw EngineError(MPSW_ERR_ARG, "window needs nsteps >= 1 and ckpt_every >= 1");
  prepare();
  Window &W = win;
  const int snaps = W.snap_req;
  // binomial reversal keeps only the start state as a checkpoint
  const int ev = snaps ? nsteps : std::min(every, nsteps), nck = (nsteps + ev - 1) / ev;
  if (W.nsteps && W.every == ev && W.nckpt == nck && W.snaps == snaps && W.x_u) {
    W.nsteps = nsteps;  // same checkpoint layout: reuse every buffer
    window_store_alloc(nsteps);
    window_capture_state(s);
    return;
  }
  window_free_trajectory();
  W.nsteps = nsteps;
  W.every = ev;
  W.nckpt = nck;
  W.snaps = snaps;
  if (snaps) binomial_tables(nsteps, snaps, W.bin_cost, W.bin_split);
  // zero-filled, so the autotuner's first timings (before the forward sweep has written the
  // stage buffers) read finite values
  auto D = [&](size_t n) {
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, sizeof(double) * n), "cudaMalloc window");
    cuda_check(cudaMemsetAsync(p, 0, sizeof(double) * n, stream), "memset window");
    return (double *)p;
  };
  auto F = [&](size_t n) {
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, sizeof(float) * n), "cudaMalloc window");
    cuda_check(cudaMemsetAsync(p, 0, sizeof(float) * n, stream), "memset window");
    return (float *)p;
  };
  for (int i = 0; i < W.nckpt; i++) {
    W.ck_u.push_back(D(nE));
    W.ck_h.push_back(D(nC));
  }
  if (!snaps) {
    W.seg_u = D((size_t)W.every * nE);
    W.seg_h = D((size_t)W.every * nC);
  }
  for (int i = 0; i < snaps; i++) {
    W.sn_u.push_back(D(nE));
    W.sn_h.push_back(D(nC));
  }
  W.fin_u = D(nE);
  W.fin_h = D(nC);
  W.x_u = D(nE);
  W.x_h = D(nC);
  for (int k = 0; k < 4; k++) {
    Diag<double> &d = W.sd[k];
    d.circ = nullptr; d.vc = nullptr;
    d.vort = D(nV); d.hv = D(nV); d.pvv = D(nV); d.div = D(nC); d.ke = D(nC); d.pc = D(nC);
    d.v = D(nE); d.gpt = D(nE); d.pe = D(nE); d.gpn = D(nE); d.he = D(nE);
    d.dsq_u = D(nE); d.dsq_vort = D(nV); d.dsq_div = D(nC);
    Diag<float> &f = W.sd32[k];
    f.vort = F(nV); f.hv = F(nV); f.ke = F(nC); f.v = F(nE); f.gpt = F(nE); f.pe = F(nE);
    f.gpn = F(nE); f.he = F(nE);
    W.su32[k] = F(nE);
    W.su[k] = k == 0 ? nullptr : D(nE);
    W.sh[k] = k == 0 ? nullptr : D(nC);
  }
  window_store_alloc(nsteps);
  window_capture_state(s);
}

// The window starts from the module's level-1 state as it is now: copy it (after the caller's
// stream) and leave the forward sweep to the first call that needs it (window_ensure), which
// lets a tangent-linear sweep over stored stages run it alongside.
void Engine::window_capture_state(cudaStream_t s) {
  Window &W = win;
  cuda_check(cudaStreamSynchronize(s), "window sync");
  cuda_check(cudaMemcpyAsync(W.x_u, dv("u"), sizeof(double) * nE, cudaMemcpyDeviceToDevice, stream), "copy");
  cuda_check(cudaMemcpyAsync(W.x_h, dv("h"), sizeof(double) * nC, cudaMemcpyDeviceToDevice, stream), "copy");
  cuda_check(cudaStreamSynchronize(stream), "window_init");
  for (int p = 0; p < 2; p++) W.st[p].valid = 0;
  W.pending = true;
}

static void window_checkpoint(Engine &E, int n) {
  Window &W = E.win;
  if (n % W.every == 0) {
    cuda_check(cudaMemcpyAsync(W.ck_u[n / W.every], W.x_u, sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "ckpt");
    cuda_check(cudaMemcpyAsync(W.ck_h[n / W.every], W.x_h, sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "ckpt");
  }
}

// After the forward sweep: keep the final state, mark the stores written.
static void window_forward_done(Engine &E) {
  Window &W = E.win;
  cuda_check(cudaMemcpyAsync(W.fin_u, W.x_u, sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "final");
  cuda_check(cudaMemcpyAsync(W.fin_h, W.x_h, sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "final");
  cuda_check(cudaGetLastError(), "window forward");
  for (int p = 0; p < 2; p++) W.st[p].valid = W.st[p].mem ? W.nsteps : 0;
  W.pending = false;
}

// Forward over the window from the captured start state, checkpointing every `every` steps
// and, when stores are allocated, writing every stage's linearisation point to them (the
// whole window is then one CUDA graph, since every step writes different slots).
void Engine::window_forward() {
  Window &W = win;
  const int nsteps = W.nsteps;
  if (W.st[0].mem || W.st[1].mem) {
    GraphKey key = graph_key(6, 0, nsteps, W.st[0].mem, W.st[1].mem);
    key.n2 = W.every;
    run_graph(key, [&]() {
      for (int n = 0; n < nsteps; n++) {
        window_checkpoint(*this, n);
        traj_step(*this, true, 0, [](int) {}, n);
      }
    });
  } else {
    for (int n = 0; n < nsteps; n++) {
      window_checkpoint(*this, n);
      run_graph(graph_key(1, 0, 1, nullptr, nullptr), [&]() { traj_step(*this, true, 0, [](int) {}); });
    }
  }
  window_forward_done(*this);
}

void Engine::window_ensure() {
  if (win.pending) window_forward();
}

// Members per chunk of the fused stage kernels for B members of precision R (0: the split member
// kernels run instead: FP64 members, physics beyond the fused kernels, or no fused tiles).
template <typename R>
static int fused_members(const Engine &E, int B, const Phys<R> &ph) {
  if constexpr (std::is_same<R, double>::value) {
    return 0;
  } else {
    // the chunk the tiles were sized for, else the largest smaller one B is a multiple of
    for (int M = E.fused.M; M >= 4; M /= 2)
      if (Launch<R, double>::fused_ok(E.fused, B, ph, M)) return M;
    return 0;
  }
}

// Member work of tangent-linear stage k about the linearisation point bs.
//
// Stage 1 reads the FP64 member state directly when R is double; otherwise its FP32 rounding in
// pu[3] / ph[3], made here when `round_in` (the first step of a sweep, or every step where the
// previous one did not leave it: per-step graphs, test case 1's frozen wind) and otherwise
// written by the previous step's stage 4 as it formed the new state.  FP32 members then form the
// provisional states of stages 2-4 from that rounded input (x + c dt tend in FP32: four bytes a
// value instead of the FP64 state's eight); the FP64 state is read only by stage 4, which
// accumulates the step.
template <typename R>
static void tl_member_stage(Engine &E, int prec, int B, double *du, double *dh, MemberBufs<R> *mb,
                            const Phys<R> &ph, const double w[4], const double c[4], int k, const Base<R> &bs,
                            cudaStream_t st, bool round_in) {
  const MeshDev<R> &m = mesh_for<R>(E);
  const R *uti = k == 0 ? nullptr : mb->pu[k - 1];
  const R *hti = k == 0 ? nullptr : mb->ph[k - 1];
  constexpr bool f64 = std::is_same<R, double>::value;
  const bool hand_on = !f64 && !ph.tc1;  // stage 4 leaves the next step's rounded input
  if (k == 0) {
    if constexpr (f64) {
      uti = du;
      hti = dh;
    } else {
      if (round_in || ph.tc1) {
        convert_d2f((long long)E.nE * B, du, mb->pu[3], st);
        convert_d2f((long long)E.nC * B, dh, mb->ph[3], st);
      }
      uti = mb->pu[3];
      hti = mb->ph[3];
    }
  }
  // stages 1-3 keep their tendencies; stage 4 sums them into the FP64 members (deferred RK4
  // accumulation, the same FP64 additions as accumulating stage by stage)
  R *nu = k < 3 ? mb->pu[k] : (hand_on ? mb->pu[3] : nullptr);
  R *nh = k < 3 ? mb->ph[k] : (hand_on ? mb->ph[3] : nullptr);
  RK<R, double> rut{du, nullptr, k == 3 ? du : nullptr, nu, c[k], w[k], R(0), ph.tc1};
  RK<R, double> rht{dh, nullptr, k == 3 ? dh : nullptr, nh, c[k], w[k], R(0), 0};
  if (k < 3) {
    rut.t_out = mb->tk_u[k];
    rht.t_out = mb->tk_h[k];
    if (hand_on) {
      rut.x0r = mb->pu[3];
      rht.x0r = mb->ph[3];
    }
  } else {
    for (int j = 0; j < 3; j++) {
      rut.t_in[j] = mb->tk_u[j];
      rht.t_in[j] = mb->tk_h[j];
      rut.wt[j] = rht.wt[j] = w[j];
    }
  }
  if (const int M = fused_members<R>(E, B, ph)) {
    Launch<R, double>::tl_fused(E.fused, M, m, B, bs, uti, hti, ph, rut, rht, st);
    return;
  }
  const Diag<R> d = tl_rows(mb, ph);
  Launch<R, double>::tl_vertex(m, B, bs, uti, hti, d, st);
  Launch<R, double>::tl_cell(m, B, bs, uti, hti, d, rht, nullptr, st);
  Launch<R, double>::tl_edge_diag(m, B, bs, uti, hti, d, ph, st);
  if (ph.visc4 > R(0)) Launch<R, double>::del4_vc(m, B, d.dsq_u, d.dsq_vort, d.dsq_div, st);
  Launch<R, double>::tl_edge_tend(m, B, bs, uti, hti, d, ph, rut, nullptr, st);
}

// Copy B members' FP64 states between a caller's buffers and the engine's (internal order).
static void members_copy(Engine &E, int B, double *dst_u, double *dst_h, const double *src_u, const double *src_h) {
  cuda_check(cudaMemcpyAsync(dst_u, src_u, sizeof(double) * E.nE * B, cudaMemcpyDeviceToDevice, E.stream), "members");
  cuda_check(cudaMemcpyAsync(dst_h, src_h, sizeof(double) * E.nC * B, cudaMemcpyDeviceToDevice, E.stream), "members");
}

template <typename R>
static void window_tl_impl(Engine &E, int prec, int B, double *user_u, double *user_h) {
  Window &W = E.win;
  MemberBufs<R> *mb = members<R>(E, prec, B, E.stream);
  double *du = W.ms[prec].x_u, *dh = W.ms[prec].x_h;
  members_copy(E, B, du, dh, user_u, user_h);
  const Phys<double> ph64 = E.phys();
  const Phys<R> ph = phys_as<R>(ph64);
  double w[4], c[4];
  rk_coeffs(ph64.dt, w, c);
  if (W.pending && W.st[prec].mem) {
    // forward sweep and tangent linear in one graph: the forward on the engine stream, the
    // members on the side stream, step n of the members after step n of the forward has
    // stored its stages, so the thin forward kernels run alongside the member kernels
    GraphKey key = E.graph_key(7, prec, B, du, dh);
    key.p3 = W.st[prec].mem;
    key.n2 = ((long long)W.nsteps << 20) | W.every;
    StableBaseScope stable(true);  // the members read only stored stages
    E.run_graph(key, [&]() {
      cuda_check(cudaEventRecord(E.ev_fork, E.stream), "event record");
      cuda_check(cudaStreamWaitEvent(E.side, E.ev_fork, 0), "event wait");
      for (int n = 0; n < W.nsteps; n++) {
        window_checkpoint(E, n);
        traj_step(E, true, 0, [](int) {}, n);
        cuda_check(cudaEventRecord(E.ev_step, E.stream), "event record");
        cuda_check(cudaStreamWaitEvent(E.side, E.ev_step, 0), "event wait");
        for (int k = 0; k < 4; k++)
          tl_member_stage<R>(E, prec, B, du, dh, mb, ph, w, c, k, stored_base<R>(W, prec, n, k), E.side, n == 0);
      }
      cuda_check(cudaEventRecord(E.ev_join, E.side), "event record");
      cuda_check(cudaStreamWaitEvent(E.stream, E.ev_join, 0), "event wait");
    });
    window_forward_done(E);
  } else if (W.st[prec].valid >= W.nsteps) {
    // stored linearisation points: the whole sweep is one graph of member kernels
    GraphKey key = E.graph_key(4, prec, B, du, dh);
    key.p3 = W.st[prec].mem;
    key.n2 = W.nsteps;
    StableBaseScope stable(true);
    E.run_graph(key, [&]() {
      for (int n = 0; n < W.nsteps; n++)
        for (int k = 0; k < 4; k++)
          tl_member_stage<R>(E, prec, B, du, dh, mb, ph, w, c, k, stored_base<R>(W, prec, n, k), E.stream, n == 0);
    });
  } else {
    E.window_ensure();
    cuda_check(cudaMemcpyAsync(W.x_u, W.ck_u[0], sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "copy");
    cuda_check(cudaMemcpyAsync(W.x_h, W.ck_h[0], sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "copy");
    // recompute each step's stages; the member work of stage k runs right after stage k (the
    // FP64 base of stage 1 is the step's start state, which stage 4 overwrites)
    const GraphKey key = E.graph_key(2, prec, B, du, dh);
    for (int n = 0; n < W.nsteps; n++)
      E.run_graph(key, [&]() {
        traj_step(E, true, prec, [&](int k) {
          tl_member_stage<R>(E, prec, B, du, dh, mb, ph, w, c, k, base_for<R>(W, k), E.stream, true);
        });
      });
  }
  members_copy(E, B, user_u, user_h, du, dh);
  cuda_check(cudaGetLastError(), "window_tl");
}

// Adjoint member work of one step (stages 4..1) about the linearisation points base(k).
template <typename R, typename BaseOf>
static void ad_member_step(Engine &E, int prec, int B, double *au, double *ah, MemberBufs<R> *mb,
                           const Phys<R> &ph, const double w[4], const double c[4], BaseOf &&base) {
  const MeshDev<R> &m = mesh_for<R>(E);
  Window::Members &M = E.win.ms[prec];
  const AdSeeds<R> none{};
  const double wu4 = ph.tc1 ? 0.0 : w[3];
  for (int k = 3; k >= 0; k--) {
    AdIn<R> in{mb->pad_u[(3 - k) & 1], mb->pad_h[(3 - k) & 1]};
    AdOut<R, double> out{};
    out.acc_u = M.acc_u; out.acc_h = M.acc_h;
    // stages 4, 3, 2 keep their contributions; stage 1 sums them (deferred accumulation)
    if (k > 0) {
      out.pad_out_u = mb->tk_u[3 - k];
      out.pad_out_h = mb->tk_h[3 - k];
    } else {
      for (int j = 0; j < 3; j++) {
        out.pad_in_u[j] = mb->tk_u[j];
        out.pad_in_h[j] = mb->tk_h[j];
      }
    }
    out.x2u = au; out.x2h = ah; out.dst_u = au; out.dst_h = ah;
    out.mode = k == 3 ? AD_SET : k == 0 ? AD_FINAL : AD_ADD;
    if (sizeof(R) == 4 && !ph.tc1) {  // the adjoint state rounded once per step (ad_tinit / AD_FINAL)
      out.x2r_u = mb->pu[3];
      out.x2r_h = mb->ph[3];
    }
    out.tu_next = mb->pad_u[(4 - k) & 1];
    out.th_next = mb->pad_h[(4 - k) & 1];
    if (k > 0) {
      out.wu = ph.tc1 ? 0.0 : w[k - 1];
      out.cu = ph.tc1 ? 0.0 : c[k - 1];
      out.wh = w[k - 1];
      out.ch = c[k - 1];
    } else {  // stage 4 of the preceding step: tend_ad = w4 * (this step's input adjoint)
      out.wu = wu4;
      out.wh = w[3];
    }
    if (const int M = fused_members<R>(E, B, ph))
      Launch<R, double>::ad_fused(E.fused, M, m, B, base(k), ph, in, out, E.stream);
    else
      Launch<R, double>::ad_stage(m, B, base(k), ph, in, none, ad_rows(mb, ph), out, E.stream);
  }
}

template <typename R>
static void window_ad_impl(Engine &E, int prec, int B, double *user_u, double *user_h) {
  Window &W = E.win;
  MemberBufs<R> *mb = members<R>(E, prec, B, E.stream);
  double *au = W.ms[prec].x_u, *ah = W.ms[prec].x_h;
  W.forward_steps = 0;
  members_copy(E, B, au, ah, user_u, user_h);
  const MeshDev<R> &m = mesh_for<R>(E);
  const Phys<double> ph64 = E.phys();
  const Phys<R> ph = phys_as<R>(ph64);
  double w[4], c[4];
  rk_coeffs(ph64.dt, w, c);
  const double wu4 = ph64.tc1 ? 0.0 : w[3];
  // tendency adjoint of the last stage of the last step; later steps get theirs from the
  // final stage of the step after them
  auto tinit = [&]() {
    Launch<R, double>::ad_tinit(m, B, au, ah, nullptr, nullptr, wu4, w[3], mb->pad_u[0], mb->pad_h[0], E.stream);
    if constexpr (sizeof(R) == 4) {
      if (!ph64.tc1) {  // the rounded adjoint state of the last step's stages
        convert_d2f((long long)E.nE * B, au, mb->pu[3], E.stream);
        convert_d2f((long long)E.nC * B, ah, mb->ph[3], E.stream);
      }
    }
  };
  if (W.st[prec].valid >= W.nsteps) {
    // stored linearisation points: the whole sweep is one graph of member kernels
    GraphKey key = E.graph_key(5, prec, B, au, ah);
    key.p3 = W.st[prec].mem;
    key.n2 = W.nsteps;
    StableBaseScope stable(true);
    E.run_graph(key, [&]() {
      tinit();
      for (int n = W.nsteps - 1; n >= 0; n--)
        ad_member_step<R>(E, prec, B, au, ah, mb, ph, w, c, [&](int k) { return stored_base<R>(W, prec, n, k); });
    });
    members_copy(E, B, user_u, user_h, au, ah);
    cuda_check(cudaGetLastError(), "window_ad");
    return;
  }
  tinit();
  auto copy_state = [&](double *du_, double *dh_, const double *su_, const double *sh_) {
    cuda_check(cudaMemcpyAsync(du_, su_, sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "copy");
    cuda_check(cudaMemcpyAsync(dh_, sh_, sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "copy");
  };
  auto advance = [&](int k) {  // k nonlinear steps of the state in x_u, x_h
    for (int i = 0; i < k; i++) E.run_graph(E.graph_key(1, 0, 1, nullptr, nullptr), [&]() { traj_step(E, true, 0, [](int) {}); });
    W.forward_steps += k;
  };
  auto adjoint_step = [&]() {  // the adjoint of the step that starts at x_u, x_h
    E.run_graph(E.graph_key(3, prec, B, au, ah), [&]() {
      traj_step(E, false, prec, [](int) {});
      ad_member_step<R>(E, prec, B, au, ah, mb, ph, w, c, [&](int k) { return base_for<R>(W, k); });
    });
  };
  if (W.snaps) {
    // binomial reversal: steps [a, a + n) from the start state (su, sh) with s free slots; the
    // slot a level writes is slot s - 1, below every slot an enclosing level still holds
    const size_t L = (size_t)W.nsteps + 1;
    std::function<void(int, int, int, const double *, const double *)> rev = [&](int a, int n, int s,
                                                                                 const double *su, const double *sh) {
      if (n == 1) {
        copy_state(W.x_u, W.x_h, su, sh);
        adjoint_step();
        return;
      }
      if (s == 0) {  // no slot: recompute each step from the start, last step first
        for (int i = n - 1; i >= 0; i--) {
          copy_state(W.x_u, W.x_h, su, sh);
          advance(i);
          adjoint_step();
        }
        return;
      }
      const int m = W.bin_split[(size_t)s * L + n];
      copy_state(W.x_u, W.x_h, su, sh);
      advance(m);
      copy_state(W.sn_u[s - 1], W.sn_h[s - 1], W.x_u, W.x_h);
      rev(a + m, n - m, s - 1, W.sn_u[s - 1], W.sn_h[s - 1]);
      rev(a, m, s, su, sh);
    };
    rev(0, W.nsteps, W.snaps, W.ck_u[0], W.ck_h[0]);
    members_copy(E, B, user_u, user_h, au, ah);
    cuda_check(cudaGetLastError(), "window_ad");
    return;
  }
  for (int s = W.nckpt - 1; s >= 0; s--) {
    const int first = s * W.every, len = std::min(W.every, W.nsteps - first);
    // replay the segment, keeping the start state of every step
    cuda_check(cudaMemcpyAsync(W.x_u, W.ck_u[s], sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "copy");
    cuda_check(cudaMemcpyAsync(W.x_h, W.ck_h[s], sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "copy");
    for (int j = 0; j < len; j++) {
      cuda_check(cudaMemcpyAsync(W.seg_u + (size_t)j * E.nE, W.x_u, sizeof(double) * E.nE, cudaMemcpyDeviceToDevice, E.stream), "seg");
      cuda_check(cudaMemcpyAsync(W.seg_h + (size_t)j * E.nC, W.x_h, sizeof(double) * E.nC, cudaMemcpyDeviceToDevice, E.stream), "seg");
      if (j + 1 < len) advance(1);
    }
    for (int j = len - 1; j >= 0; j--) {
      copy_state(W.x_u, W.x_h, W.seg_u + (size_t)j * E.nE, W.seg_h + (size_t)j * E.nC);
      adjoint_step();  // recomputes this step's four stages, then their adjoints
    }
  }
  members_copy(E, B, user_u, user_h, au, ah);
  cuda_check(cudaGetLastError(), "window_ad");
}

static void join(cudaStream_t user, cudaStream_t mine, bool before) {
  // order the engine stream after (before=true) or before (false) the caller's stream
  cudaEvent_t ev;
  cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
  if (before) {
    cuda_check(cudaEventRecord(ev, user), "event record");
    cuda_check(cudaStreamWaitEvent(mine, ev, 0), "event wait");
  } else {
    cuda_check(cudaEventRecord(ev, mine), "event record");
    cuda_check(cudaStreamWaitEvent(user, ev, 0), "event wait");
  }
  cuda_check(cudaEventDestroy(ev), "event destroy");
}

void Engine::window_tl(int prec, int B, double *du, double *dh, cudaStream_t s) {
  if (!win.nsteps) throw EngineError(MPSW_ERR_STATE, "mpsw_window_init has not been called");
  if (B < 1 || !du || !dh) throw EngineError(MPSW_ERR_ARG, "window_tl needs B >= 1 and member buffers");
  if (mesh_dirty) throw EngineError(MPSW_ERR_STATE, "mesh changed since mpsw_window_init");
  if (prec != 0 && prec != 1) throw EngineError(MPSW_ERR_ARG, "precision must be 0 or 1");
  join(s, stream, true);
  TuneScope scope(tuning(prec, B));
  nonfinite_clear();  // after the autotuner, whose timings run on arbitrary buffer contents
  if (prec == 0) window_tl_impl<double>(*this, prec, B, du, dh);
  else window_tl_impl<float>(*this, prec, B, du, dh);
  nonfinite_check("window_tl");
  join(s, stream, false);
}

void Engine::window_ad(int prec, int B, double *au, double *ah, cudaStream_t s) {
  if (!win.nsteps) throw EngineError(MPSW_ERR_STATE, "mpsw_window_init has not been called");
  if (B < 1 || !au || !ah) throw EngineError(MPSW_ERR_ARG, "window_ad needs B >= 1 and member buffers");
  if (mesh_dirty) throw EngineError(MPSW_ERR_STATE, "mesh changed since mpsw_window_init");
  if (prec != 0 && prec != 1) throw EngineError(MPSW_ERR_ARG, "precision must be 0 or 1");
  join(s, stream, true);
  window_ensure();
  TuneScope scope(tuning(prec, B));
  nonfinite_clear();  // after the autotuner, whose timings run on arbitrary buffer contents
  if (prec == 0) window_ad_impl<double>(*this, prec, B, au, ah);
  else window_ad_impl<float>(*this, prec, B, au, ah);
  nonfinite_check("window_ad");
  join(s, stream, false);
}

void Engine::window_final(double *u, double *h, cudaStream_t s) {
  if (!win.nsteps) throw EngineError(MPSW_ERR_STATE, "mpsw_window_init has not been called");
  join(s, stream, true);
  window_ensure();
  cuda_check(cudaMemcpyAsync(u, win.fin_u, sizeof(double) * nE, cudaMemcpyDeviceToDevice, stream), "final u");
  cuda_check(cudaMemcpyAsync(h, win.fin_h, sizeof(double) * nC, cudaMemcpyDeviceToDevice, stream), "final h");
  join(s, stream, false);
}

void Engine::to_internal(int kind, int B, const double *src, double *dst, cudaStream_t s) {
  if (!mesh_built) throw EngineError(MPSW_ERR_STATE, "mesh not initialised");
  if (kind < 0 || kind > 2 || B < 1) throw EngineError(MPSW_ERR_ARG, "bad kind or B");
  const int n = kind == 0 ? nC : kind == 1 ? nE : nV;
  L64::to_internal(n, B, d_perm[kind], src, dst, s);
  cuda_check(cudaGetLastError(), "to_internal");
}

void Engine::to_reference(int kind, int B, const double *src, double *dst, cudaStream_t s) {
  if (!mesh_built) throw EngineError(MPSW_ERR_STATE, "mesh not initialised");
  if (kind < 0 || kind > 2 || B < 1) throw EngineError(MPSW_ERR_ARG, "bad kind or B");
  const int n = kind == 0 ? nC : kind == 1 ? nE : nV;
  L64::to_reference(n, B, d_perm[kind], src, dst, s);
  cuda_check(cudaGetLastError(), "to_reference");
}

void Engine::state_from_device(const double *u, const double *h, cudaStream_t s) {
  prepare();
  join(s, stream, true);
  L64::to_internal(nE, 1, d_perm[1], u, dv("u"), stream);
  L64::to_internal(nC, 1, d_perm[0], h, dv("h"), stream);
  cuda_check(cudaGetLastError(), "state_from_device");
  cuda_check(cudaStreamSynchronize(stream), "state_from_device");
  mark_written(var("u"), true);
  mark_written(var("h"), true);
  pending_diag = 1;
  for (const char *n : {"v", "h_edge", "h_vertex", "pv_edge", "pv_vertex", "pv_cell", "circulation",
                        "vorticity", "divergence", "ke", "vh", "vorticity_cell", "gradPVn", "gradPVt"}) {
    mark_written(var(n), true);
    var(n).lazy_diag = true;
  }
}

void Engine::state_to_device(double *u, double *h, cudaStream_t s) {
  prepare();
  join(s, stream, true);
  L64::to_reference(nE, 1, d_perm[1], dv("u"), u, stream);
  L64::to_reference(nC, 1, d_perm[0], dv("h"), h, stream);
  cuda_check(cudaGetLastError(), "state_to_device");
  join(s, stream, false);
}

// Average launch time of member kernel `which` (or a whole stage, 8 / 9).  cold: each launch is
// timed alone, after a write of a buffer larger than L2 (the step's inputs are then read from
// HBM, as in a sweep over a large mesh); otherwise `iters` launches run back to back.
template <typename R>
static double time_kernel_impl(Engine &E, int which, int prec, int B, int iters, bool cold = false) {
  Window &W = E.win;
  MemberBufs<R> *mb = members<R>(E, prec, B, E.stream);
  const MeshDev<R> &m = mesh_for<R>(E);
  const Phys<double> ph64 = E.phys();
  const Phys<R> ph = phys_as<R>(ph64);
  const Base<R> bs = W.st[prec].valid ? stored_base<R>(W, prec, 0, 1) : base_for<R>(W, 1);
  double w[4], c[4];
  rk_coeffs(ph64.dt, w, c);
  // a middle stage as the sweeps run it: x0 read, next state and tendency written (deferred
  // accumulation); the adjoint likewise stores its contribution
  RK<R, double> rku{W.ms[prec].acc_u, nullptr, nullptr, mb->pu[1], c[1], w[1], R(0), 0};
  RK<R, double> rkh{W.ms[prec].acc_h, nullptr, nullptr, mb->ph[1], c[1], w[1], R(0), 0};
  rku.t_out = mb->tk_u[1];
  rkh.t_out = mb->tk_h[1];
  if (sizeof(R) == 4) {  // FP32 members read the step's rounded input
    rku.x0r = mb->pu[3];
    rkh.x0r = mb->ph[3];
  }
  AdIn<R> in{mb->pad_u[0], mb->pad_h[0]};
  AdOut<R, double> out{};
  out.acc_u = W.ms[prec].acc_u; out.acc_h = W.ms[prec].acc_h; out.mode = AD_ADD;
  out.x2u = W.ms[prec].acc_u; out.x2h = W.ms[prec].acc_h;
  out.tu_next = mb->pad_u[1]; out.th_next = mb->pad_h[1];
  out.pad_out_u = mb->tk_u[1]; out.pad_out_h = mb->tk_h[1];
  out.wu = w[1]; out.cu = c[1]; out.wh = w[1]; out.ch = c[1];
  if (sizeof(R) == 4) {
    out.x2r_u = mb->pu[3];
    out.x2r_h = mb->ph[3];
  }
  StableBaseScope stable(true);  // the timed kernels write no linearisation point
  const Diag<R> d = tl_rows(mb, ph);
  const AdWork<R> aw = ad_rows(mb, ph);
  auto launch = [&]() {
    using LR = Launch<R, double>;
    switch (which) {
      case 0: LR::tl_vertex(m, B, bs, mb->pu[0], mb->ph[0], d, E.stream); break;
      case 1: LR::tl_cell(m, B, bs, mb->pu[0], mb->ph[0], d, rkh, nullptr, E.stream); break;
      case 2: LR::tl_edge_diag(m, B, bs, mb->pu[0], mb->ph[0], d, ph, E.stream); break;
      case 3: LR::tl_edge_tend(m, B, bs, mb->pu[0], mb->ph[0], d, ph, rku, nullptr, E.stream); break;
      case 8:  // one whole tangent-linear stage, as the sweeps run it
        if (const int M = fused_members<R>(E, B, ph)) {
          LR::tl_fused(E.fused, M, m, B, bs, mb->pu[0], mb->ph[0], ph, rku, rkh, E.stream);
          break;
        }
        LR::tl_vertex(m, B, bs, mb->pu[0], mb->ph[0], d, E.stream);
        LR::tl_cell(m, B, bs, mb->pu[0], mb->ph[0], d, rkh, nullptr, E.stream);
        LR::tl_edge_diag(m, B, bs, mb->pu[0], mb->ph[0], d, ph, E.stream);
        if (ph.visc4 > R(0)) LR::del4_vc(m, B, d.dsq_u, d.dsq_vort, d.dsq_div, E.stream);
        LR::tl_edge_tend(m, B, bs, mb->pu[0], mb->ph[0], d, ph, rku, nullptr, E.stream);
        break;
      case 9: {  // one whole adjoint stage, as the sweeps run it
        const AdSeeds<R> none{};
        if (const int M = fused_members<R>(E, B, ph))
          LR::ad_fused(E.fused, M, m, B, bs, ph, in, out, E.stream);
        else
          LR::ad_stage(m, B, bs, ph, in, none, aw, out, E.stream);
        break;
      }
      default: LR::ad_part(which - 4, m, B, bs, ph, in, aw, out, E.stream); break;
    }
  };
  launch();  // warm-up
  cudaEvent_t a, b;
  cuda_check(cudaEventCreate(&a), "event");
  cuda_check(cudaEventCreate(&b), "event");
  double total = 0;
  for (int rep = 0; rep < (cold ? iters : 1); rep++) {
    if (cold) cuda_check(cudaMemsetAsync(E.l2_flush_buffer(), rep & 0xff, Engine::kL2Flush, E.stream), "L2 flush");
    cuda_check(cudaEventRecord(a, E.stream), "event");
    for (int i = 0; i < (cold ? 1 : iters); i++) launch();
    cuda_check(cudaEventRecord(b, E.stream), "event");
    cuda_check(cudaEventSynchronize(b), "event");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, a, b), "event");
    total += ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cuda_check(cudaGetLastError(), "time_kernel");
  return total / iters;
}

double Engine::time_kernel(int which, int prec, int B, int iters) {
  if (!win.nsteps) throw EngineError(MPSW_ERR_STATE, "mpsw_window_init has not been called");
  if (which < 0 || which > 9 || B < 1 || iters < 1) throw EngineError(MPSW_ERR_ARG, "bad kernel timing request");
  window_ensure();
  TuneScope scope(tuned_for(prec, B));  // the launch choices the sweeps use
  return prec == 1 ? time_kernel_impl<float>(*this, which, prec, B, iters, true)
                   : time_kernel_impl<double>(*this, which, prec, B, iters, true);
}

// Autotuner of the member kernels: for each of the eight tangent-linear / adjoint kernels, time
// every (members per thread, threads per block) pair the member count allows on the window's own
// buffers (mpsw_time_kernel's launch of a middle stage; the better of two 8-launch averages) and
// keep the fastest.  Runs once per
// (precision, B) before the first sweep captures its graphs, so the graphs bake in the choice;
// MPSW_TUNE=0 keeps the default choices.
template <typename R>
static TuneTable tune_members(Engine &E, int prec, int B) {
  TuneTable best{};
  const int vs[] = {1, 2, 4, 8}, blocks[] = {64, 128, 256};
  for (int k = 0; k < K_TUNED; k++) {
    double tbest = 1e30;
    for (int v : vs) {
      if (B % v || (sizeof(R) == 8 && v > 4) || (sizeof(R) == 4 && v < 2 && B % 2 == 0)) continue;
      for (int bl : blocks) {
        TuneTable trial = best;
        trial.k[k].v = v;
        trial.k[k].block = bl;
        TuneScope scope(&trial);
        const double t = std::min(time_kernel_impl<R>(E, k, prec, B, 8), time_kernel_impl<R>(E, k, prec, B, 8));
        if (t < tbest) {
          tbest = t;
          best.k[k] = trial.k[k];
        }
      }
    }
  }
  return best;
}

// Tuning results can be kept in a text file (MPSW_TUNE_CACHE=path), one line per key:
// "<device name>|<nCells>|<nEdges>|<nVertices>|<precision>|<B>" then 8 pairs "v block".  A
// process finding its key there skips the timing (so, for example, a profiled run uses the
// choices of an unprofiled one).
static std::string tune_key(const Engine &E, int prec, int B) {
  int dev = 0;
  cudaDeviceProp p{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) p.name[0] = 0;
  std::string name(p.name);
  for (char &c : name)
    if (c == ' ' || c == '|') c = '_';
  return name + "|" + std::to_string(E.nC) + "|" + std::to_string(E.nE) + "|" + std::to_string(E.nV) + "|" +
         std::to_string(prec) + "|" + std::to_string(B);
}

static bool tune_cache_read(const std::string &path, const std::string &key, TuneTable *t) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof line, f)) {
    char k[512];
    int v[2 * K_TUNED];
    if (sscanf(line, "%511s %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d", k, &v[0], &v[1], &v[2], &v[3], &v[4],
               &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &v[11], &v[12], &v[13], &v[14], &v[15]) != 17 ||
        key != k)
      continue;
    for (int i = 0; i < K_TUNED; i++) {
      t->k[i].v = v[2 * i];
      t->k[i].block = v[2 * i + 1];
    }
    found = true;  // the last line for a key wins
  }
  fclose(f);
  return found;
}

static void tune_cache_append(const std::string &path, const std::string &key, const TuneTable &t) {
  FILE *f = fopen(path.c_str(), "a");
  if (!f) return;  // a cache that cannot be written only costs a re-tune
  fprintf(f, "%s", key.c_str());
  for (int i = 0; i < K_TUNED; i++) fprintf(f, " %d %d", t.k[i].v, t.k[i].block);
  fprintf(f, "\n");
  fclose(f);
}

// The table for (prec, B), tuning it first when needed (before any graph of it is captured).
const TuneTable *Engine::tuning(int prec, int B) {
  static const bool enabled = !(getenv("MPSW_TUNE") && atoi(getenv("MPSW_TUNE")) == 0);
  if (!enabled) return nullptr;
  auto it = win.tune[prec].find(B);
  if (it != win.tune[prec].end()) return &it->second;
  const char *cache = getenv("MPSW_TUNE_CACHE");
  const std::string key = tune_key(*this, prec, B);
  TuneTable t{};
  if (!(cache && *cache && tune_cache_read(cache, key, &t))) {
    t = prec == 1 ? tune_members<float>(*this, prec, B) : tune_members<double>(*this, prec, B);
    if (cache && *cache) tune_cache_append(cache, key, t);
  }
  graphs_free();  // nothing captured before this point may keep the untuned choices
  return &(win.tune[prec][B] = t);
}

// The table for (prec, B) if it has been tuned, else null (defaults).
const TuneTable *Engine::tuned_for(int prec, int B) {
  auto it = win.tune[prec].find(B);
  return it == win.tune[prec].end() ? nullptr : &it->second;
}

}  // namespace mpsw

// ---- C ABI of the window -----------------------------------------------------------------
extern "C" {
int mpsw_to_internal(mpsw_handle *h, int kind, int B, const double *src, double *dst, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.to_internal(kind, B, src, dst, (cudaStream_t)stream); });
}
int mpsw_to_reference(mpsw_handle *h, int kind, int B, const double *src, double *dst, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.to_reference(kind, B, src, dst, (cudaStream_t)stream); });
}
int mpsw_window_tuning(mpsw_handle *h, int precision, int B, int *v_block) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!v_block) throw mpsw::EngineError(MPSW_ERR_ARG, "null output");
    if (precision != 0 && precision != 1) throw mpsw::EngineError(MPSW_ERR_ARG, "precision must be 0 or 1");
    const mpsw::TuneTable *t = e.tuned_for(precision, B);
    for (int k = 0; k < mpsw::K_TUNED; k++) {
      v_block[2 * k] = t ? t->k[k].v : 0;
      v_block[2 * k + 1] = t ? t->k[k].block : 0;
    }
  });
}
int mpsw_window_fused(mpsw_handle *h, int precision, int B, int *members_per_block, int *tile_cells) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!members_per_block || !tile_cells) throw mpsw::EngineError(MPSW_ERR_ARG, "null output");
    if (precision != 0 && precision != 1) throw mpsw::EngineError(MPSW_ERR_ARG, "precision must be 0 or 1");
    if (B < 1) throw mpsw::EngineError(MPSW_ERR_ARG, "B must be positive");
    e.prepare();
    *members_per_block =
        precision == 1 ? mpsw::fused_members<float>(e, B, mpsw::phys_as<float>(e.phys())) : 0;
    *tile_cells = *members_per_block ? e.fused_K : 0;
  });
}
int mpsw_window_snapshots(mpsw_handle *h, int snapshots) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_snapshots(snapshots); });
}
int mpsw_window_forward_steps(mpsw_handle *h, long long *steps) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!steps) throw mpsw::EngineError(MPSW_ERR_ARG, "null output");
    *steps = e.win.forward_steps;
  });
}
int mpsw_window_storage(mpsw_handle *h, int mode, double max_bytes) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_storage(mode, max_bytes); });
}
int mpsw_window_init(mpsw_handle *h, int nsteps, int ckpt_every, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_init(nsteps, ckpt_every, (cudaStream_t)stream); });
}
int mpsw_window_tl(mpsw_handle *h, int precision, int B, double *du, double *dh, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_tl(precision, B, du, dh, (cudaStream_t)stream); });
}
int mpsw_window_ad(mpsw_handle *h, int precision, int B, double *au, double *ah, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_ad(precision, B, au, ah, (cudaStream_t)stream); });
}
int mpsw_state_from_device(mpsw_handle *h, const double *u, const double *hh, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.state_from_device(u, hh, (cudaStream_t)stream); });
}
int mpsw_state_to_device(mpsw_handle *h, double *u, double *hh, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.state_to_device(u, hh, (cudaStream_t)stream); });
}
long long mpsw_launch_count(void) { return mpsw::g_launches; }
int mpsw_time_kernel(mpsw_handle *h, int which, int precision, int B, int iters, double *ms_per_launch) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!ms_per_launch) throw mpsw::EngineError(MPSW_ERR_ARG, "null output");
    *ms_per_launch = e.time_kernel(which, precision, B, iters);
  });
}
int mpsw_window_final_state(mpsw_handle *h, double *u, double *hh, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.window_final(u, hh, (cudaStream_t)stream); });
}
}
