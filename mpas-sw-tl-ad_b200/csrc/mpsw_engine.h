// Engine behind the C ABI (include/mpsw.h): one module instance, its variables, device mesh,
// work buffers and the batched tangent-linear / adjoint window.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <initializer_list>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpsw_internal.h"
#include "mpsw_launch.h"
#include "mpsw_setup.h"
#include "mpsw_tiles.h"

namespace mpsw {

struct EngineError : std::runtime_error {
  int code;
  EngineError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

std::string lower(const char *s);
void cuda_check(cudaError_t e, const char *what);

struct Var {
  std::string name, dims_spec;
  int group = 0, is_int = 0, ent = 0, mesh = 0, lead = 1;
  std::vector<long long> dims;
  long long count = 0;
  std::vector<double> hr;
  std::vector<int> hi;
  double *dev = nullptr;  // [lead][n] internal order (state, diagnostics, tendencies)
  bool allocated = false, host_valid = true, dev_valid = true;
  bool nonzero = false;    // may hold nonzero values (adjoint seeds are skipped when false)
  bool lazy_diag = false;  // device value is produced on demand from the level-1 state
};

// Storage of the batched tangent-linear / adjoint window (mpsw_window_*).
struct Window {
  int nsteps = 0, every = 0, nckpt = 0;
  bool pending = false;  // start state captured in x_u / x_h, forward sweep not yet run
  std::vector<double *> ck_u, ck_h;    // checkpointed nonlinear states (internal order)
  double *seg_u = nullptr, *seg_h = nullptr;  // states of one segment, [every][n]
  double *fin_u = nullptr, *fin_h = nullptr;  // final state
  // single-trajectory work of the window (FP64)
  double *x_u = nullptr, *x_h = nullptr;
  Diag<double> sd[4];
  double *su[4] = {}, *sh[4] = {};
  Diag<float> sd32[4];
  float *su32[4] = {};
  // Stored linearisation points: the nine base fields of every RK stage of every step, per
  // precision (0 FP64, 1 FP32).  A slot is one stage: u, h_edge, v, gradPVt, gradPVn, pv_edge
  // (edges), vorticity, h_vertex (vertices), ke (cells), each padded to 64 elements.
  struct Store {
    void *mem = nullptr;
    int cap = 0;       // steps the allocation holds
    int valid = 0;     // steps written by the last forward pass (0: sweeps recompute)
    size_t slot = 0;   // elements per stage slot
    size_t off[9] = {};
  } st[2];
  // Binomial reversal (snapshots > 0): the window keeps only its start state and reverses the
  // adjoint with `snaps` snapshot slots, recomputing states by the schedule of least forward
  // steps (bin_cost / bin_split over steps x snapshots); 0: two-level checkpointing.
  int snap_req = 0;          // snapshots of the next windows (mpsw_window_snapshots)
  int snaps = 0;             // snapshots of the current window
  std::vector<double *> sn_u, sn_h;
  std::vector<long long> bin_cost;
  std::vector<int> bin_split;
  long long forward_steps = 0;  // trajectory steps recomputed by the last adjoint sweep
  int store_mode = -1;        // -1 automatic, else a mask of the precisions to store
  double store_budget = 0;    // bytes for automatic mode (0: 40% of free device memory)
  // member buffers per precision (0 FP64, 1 FP32), allocated for the largest B seen
  struct Members {
    int B = 0;
    std::vector<void *> mem;
    void *bufs = nullptr;  // MemberBufs<R>
    double *acc_u = nullptr, *acc_h = nullptr;
    // the members' FP64 states during a sweep: callers' buffers are copied in and out, so the
    // captured graphs do not depend on where the caller keeps its members
    double *x_u = nullptr, *x_h = nullptr;
  } ms[2];
  // autotuned launch choices of the member kernels, per precision and member count
  std::map<int, TuneTable> tune[2];
};

// A captured CUDA graph of one window step, keyed by what its kernels bake in.
struct GraphKey {
  int kind = 0, prec = 0, B = 0;
  const void *p1 = nullptr, *p2 = nullptr;
  const void *p3 = nullptr;
  long long n2 = 0;
  double dt = 0, apvm = 0, visc2 = 0, visc4 = 0;
  int flags = 0;
  bool operator==(const GraphKey &o) const {
    return kind == o.kind && prec == o.prec && B == o.B && p1 == o.p1 && p2 == o.p2 && p3 == o.p3 &&
           n2 == o.n2 && dt == o.dt && apvm == o.apvm && visc2 == o.visc2 && visc4 == o.visc4 &&
           flags == o.flags;
  }
};
struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;  // kernel launches recorded in the graph
};

struct Engine {
  std::string err;
  std::vector<GraphEntry> graphs;
  std::map<std::string, double> scal;
  std::vector<Var> vars;
  std::map<std::string, int> index;
  bool allocated[3] = {false, false, false};
  int nC = 0, nE = 0, nV = 0, mE = 0, mE2 = 0, vd = 0, nT = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                 // second stream for work forked inside a graph
  cudaEvent_t ev_fork = nullptr, ev_step = nullptr, ev_join = nullptr;

  // device mesh
  bool mesh_built = false, mesh_dirty = true;
  BuiltMesh bm;
  MeshDev<double> m64{};
  MeshDev<float> m32{};
  std::vector<void *> mesh_bufs;
  const int *d_perm[3] = {nullptr, nullptr, nullptr};
  const int *d_cnb = nullptr;  // [MAXE][nCells] the cell across each edge of a cell
  int mesh_device = -1;        // the CUDA device the mesh (and everything derived) lives on
  FusedDev fused;              // halo tiles and coefficients of the fused member stages
  int fused_K = 0;             // owned cells per tile of `fused` (0: not built)
  void build_fused();

  // work
  std::vector<void *> work;
  std::vector<double> staging;
  Diag<double> stage[5]{};
  Diag<double> tl_diag{};
  double *sp_u[4] = {}, *sp_h[4] = {}, *tp_u[4] = {}, *tp_h[4] = {};
  double *acc_u = nullptr, *acc_h = nullptr, *tacc_u = nullptr, *tacc_h = nullptr;
  AdWork<double> adw{};
  double *tu_[2] = {}, *th_[2] = {}, *xacc_u = nullptr, *xacc_h = nullptr;
  Diag<float> d32{};                          // FP32-stencil forward (precision 1)
  float *s32_u[4] = {}, *s32_h[4] = {};
  double *trc = nullptr;  // tracer transport work ([6][nT][nC]), see tracer_bufs
  long long trc_n = 0;
  int pending_diag = 0;  // 1: diagnostics of the level-1 state owed, 2: and their tangents
  Phys<double> phys_cache{};  // physics scalars, refreshed whenever a scalar is assigned
  // buffer larger than L2 that kernel timing writes between launches (allocated on first use)
  static constexpr size_t kL2Flush = (size_t)256 << 20;
  void *l2_flush = nullptr;
  void *l2_flush_buffer();
  void refresh_phys();
  Window win;

  Engine();
  ~Engine();

  Var *find(const std::string &lname);
  Var &var(const char *name);
  double sc(const char *name) const;
  long long dim_of(const std::string &sym) const;
  void need_device();
  void *dalloc(size_t bytes);
  void allocate_group(int g);
  const std::vector<int> &perm_of(int ent) const;
  void upload(Var &v);
  void download(Var &v);
  void set_var(const char *name, const void *src, long long count);
  void get_var(const char *name, void *dst, long long count);
  void mark_written(Var &v, bool maybe_nonzero);
  template <typename T, typename S>
  const T *up(const std::vector<S> &h, std::vector<void *> &own);
  template <typename R>
  void fill_mesh(MeshDev<R> &m);
  void free_device_mesh();
  RefMesh ref_mesh();
  void build_device_mesh();
  void ensure_mesh();
  void sync_inputs();
  void prepare();
  double *wbuf(size_t n);
  Diag<double> new_diag(int B);
  void alloc_work();
  double *dv(const char *name, int level = 0);
  Diag<double> module_diag(int g);
  void mark_diag(int g, bool lazy);
  void mark_recon(int g);
  Phys<double> phys() const;
  bool tracers_advected();
  double *tracer_bufs();
  void tracers_upload(double *dst);
  void tracers_download(const double *src, const double *tend);
  void fwd_diag(const double *u, const double *h, const Diag<double> &d, const Phys<double> &ph);
  void fwd_stage(const double *u, const double *h, const Diag<double> &d, const Phys<double> &ph,
                 const RK<double, double> &rku, const RK<double, double> &rkh, double *tu, double *th);
  void tl_diag_run(const Base<double> &bs, const double *ut, const double *ht, const Diag<double> &d,
                   const Phys<double> &ph);
  void check_launch(const char *what);
  int *d_bad = nullptr;  // non-finite flag of the tendency kernels (Phys::bad)
  void nonfinite_clear();
  void nonfinite_check(const char *what);
  void materialize_pending();
  void finish_levels(std::initializer_list<const char *> names);
  AdSeeds<double> seeds(bool *any);
  void zero_ad_seeds();
  bool recon_seeds_nonzero();

  // module subroutines
  void init_block();
  void rk4(int nsteps);
  void forward(int prec, int nsteps);
  void rk4_tlm(int nsteps);
  void rk4_adj();
  void solve_diagnostics(int tl);
  void compute_tend(int tl);
  void reconstruct(int tl);
  void adjoint_at_state();
  void test_case(int tc);  // Williamson test case on the GPU (mpsw_testcases.cu)

  // batched window (mpsw_window.cu)
  void graphs_free();
  GraphKey graph_key(int kind, int prec, int B, const void *p1, const void *p2) const;
  template <typename F>
  void run_graph(const GraphKey &k, F &&body);
  void window_free();
  void window_free_trajectory();
  void window_init(int nsteps, int every, cudaStream_t s);
  void window_storage(int mode, double max_bytes);
  void window_snapshots(int snapshots);
  void window_store_alloc(int nsteps);
  void window_store_free(int prec);
  void window_capture_state(cudaStream_t s);
  void window_forward();
  void window_ensure();
  void window_tl(int prec, int B, double *du, double *dh, cudaStream_t s);
  void window_ad(int prec, int B, double *au, double *ah, cudaStream_t s);
  void window_final(double *u, double *h, cudaStream_t s);
  double time_kernel(int which, int prec, int B, int iters);
  const TuneTable *tuning(int prec, int B);
  const TuneTable *tuned_for(int prec, int B);
  void state_from_device(const double *u, const double *h, cudaStream_t s);
  void state_to_device(double *u, double *h, cudaStream_t s);
  void to_internal(int kind, int B, const double *src, double *dst, cudaStream_t s);
  void to_reference(int kind, int B, const double *src, double *dst, cudaStream_t s);
};

// Run `body` (kernel launches on the engine stream, no allocation, no synchronisation) as a
// CUDA graph: captured on first use for this key, replayed afterwards.  MPSW_GRAPHS=0 runs it
// eagerly instead.
constexpr size_t kMaxGraphs = 24;  // captured graphs kept per engine

template <typename F>
inline void Engine::run_graph(const GraphKey &k, F &&body) {
  static const bool enabled = !(getenv("MPSW_GRAPHS") && atoi(getenv("MPSW_GRAPHS")) == 0);
  if (!enabled) {
    body();
    return;
  }
  for (size_t i = 0; i < graphs.size(); i++)
    if (graphs[i].key == k) {
      if (i + 1 < graphs.size()) std::rotate(graphs.begin() + i, graphs.begin() + i + 1, graphs.end());
      GraphEntry &g = graphs.back();  // most recently used last
      cuda_check(cudaGraphLaunch(g.exec, stream), "cudaGraphLaunch");
      g_launches += g.kernels;
      return;
    }
  if (graphs.size() >= kMaxGraphs) {  // evict the least recently used
    cudaGraphExecDestroy(graphs.front().exec);
    graphs.erase(graphs.begin());
  }
  cudaGraph_t graph = nullptr;
  const long long before = g_launches;
  cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  cuda_check(cudaStreamEndCapture(stream, &graph), "end capture");
  GraphEntry e;
  e.key = k;
  e.kernels = g_launches - before;  // counted once here, then once per replay
  const cudaError_t st = cudaGraphInstantiate(&e.exec, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(st, "cudaGraphInstantiate");
  graphs.push_back(e);
  cuda_check(cudaGraphLaunch(e.exec, stream), "cudaGraphLaunch");
}

}  // namespace mpsw

// The opaque handle of the C ABI.
struct mpsw_handle {
  mpsw::Engine eng;
};

namespace mpsw {
// Prepares the current device for mpsw_compute_tend_noalloc (mpsw_noalloc.cu): looks up the
// address of its scratch array and loads the kernels it launches, so that the entry point
// itself allocates and loads nothing.
void noalloc_prepare_device();

// Runs f on the handle's engine, turning exceptions into status codes (none cross the ABI).
template <typename F>
int guarded(mpsw_handle *h, F &&f) {
  if (!h) return 1;
  try {
    f(h->eng);
    h->eng.err.clear();
    return 0;
  } catch (const EngineError &e) {
    h->eng.err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    h->eng.err = e.what();
    return 1;
  }
}
}  // namespace mpsw
