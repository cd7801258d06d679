// Module-instance engine behind include/mpsw.h: the f2py surface of `mpas_sw_module`
// (variables by name, argument-less subroutines) on top of the device stencils.
//
// Variables live twice: a host mirror in the reference layout and, for the state, diagnostic
// and tendency arrays, a device copy in internal (Hilbert) order.  Each side carries a valid
// flag; transfers happen lazily (before a routine runs for dirty inputs, on get_var for stale
// outputs), so a driver that calls sw_rk4 every step and reads h only at output times moves
// only what it reads.  Mesh arrays stay on the host until a routine needs the device mesh; the
// device mesh is rebuilt whenever a mesh array changed since the last build.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cctype>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpsw.h"
#include "mpsw_engine.h"
#include "mpsw_launch.h"
#include "mpsw_setup.h"

using namespace mpsw;

namespace mpsw {

std::string lower(const char *s) {
  std::string o(s ? s : "");
  for (auto &c : o) c = (char)std::tolower((unsigned char)c);
  return o;
}

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw EngineError(MPSW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------
// Variable table (src/mpas_sw_module.f90:57-201, allocation shapes :211-493)
// ---------------------------------------------------------------------------------------
namespace {

struct VarSpec {
  const char *name;
  int group;   // 0 var_allocation, 1 _tlm, 2 _adj
  int is_int;
  int ent;     // 0 host only, 1 cell, 2 edge, 3 vertex (entity of the last dimension)
  int mesh;    // read by the device mesh build
  const char *dims;  // Fortran dims, comma separated symbols
};

const char *kDiagNames[] = {"uReconstructX", "uReconstructY", "uReconstructZ", "uReconstructZonal",
                            "uReconstructMeridional", "v", "h_edge", "h_vertex", "pv_edge",
                            "pv_vertex", "pv_cell", "circulation", "vorticity", "divergence", "ke",
                            "vh", "vorticity_cell", "gradPVn", "gradPVt"};
const int kDiagEnt[] = {1, 1, 1, 1, 1, 2, 2, 3, 2, 3, 1, 3, 3, 1, 1, 2, 1, 2, 2};

std::vector<VarSpec> make_specs() {
  std::vector<VarSpec> s = {
      {"u", 0, 0, 2, 0, "2,L,E"}, {"h", 0, 0, 1, 0, "2,L,C"}, {"tracers", 0, 0, 0, 0, "2,T,L,C"},
      {"u_src", 0, 0, 0, 1, "L,E"}, {"h_s", 0, 0, 0, 1, "C"}, {"fCell", 0, 0, 0, 0, "C"},
      {"fVertex", 0, 0, 0, 1, "V"}, {"fEdge", 0, 0, 0, 0, "E"}, {"areaTriangle", 0, 0, 0, 1, "V"},
      {"areaCell", 0, 0, 0, 1, "C"}, {"dvEdge", 0, 0, 0, 1, "E"}, {"dcEdge", 0, 0, 0, 1, "E"},
      {"weightsOnEdge", 0, 0, 0, 1, "M2,E"}, {"kiteAreasOnVertex", 0, 0, 0, 1, "D,V"},
      {"meshDensity", 0, 0, 0, 1, "C"}, {"boundaryCell", 0, 1, 0, 0, "L,C"},
      {"boundaryEdge", 0, 1, 0, 1, "L,E"}, {"advCells", 0, 1, 0, 0, "21,C"},
      {"cellsOnCell", 0, 1, 0, 0, "M,C"}, {"cellsOnEdge", 0, 1, 0, 1, "2,E"},
      {"cellsOnVertex", 0, 1, 0, 1, "D,V"}, {"edgesOnCell", 0, 1, 0, 1, "M,C"},
      {"edgesOnEdge", 0, 1, 0, 1, "M2,E"}, {"edgesOnVertex", 0, 1, 0, 1, "D,V"},
      {"verticesOnCell", 0, 1, 0, 0, "M,C"}, {"verticesOnEdge", 0, 1, 0, 1, "2,E"},
      {"nEdgesOnCell", 0, 1, 0, 1, "C"}, {"nEdgesOnEdge", 0, 1, 0, 1, "E"},
      {"latCell", 0, 0, 0, 1, "C"}, {"lonCell", 0, 0, 0, 1, "C"}, {"xCell", 0, 0, 0, 1, "C"},
      {"yCell", 0, 0, 0, 1, "C"}, {"zCell", 0, 0, 0, 1, "C"},
      {"meshScalingDel2", 0, 0, 0, 1, "E"}, {"meshScalingDel4", 0, 0, 0, 1, "E"},
      {"deriv_two", 0, 0, 0, 1, "15,2,E"}, {"latEdge", 0, 0, 0, 0, "E"}, {"lonEdge", 0, 0, 0, 0, "E"},
      {"xEdge", 0, 0, 0, 1, "E"}, {"yEdge", 0, 0, 0, 1, "E"}, {"zEdge", 0, 0, 0, 1, "E"},
      {"angleEdge", 0, 0, 0, 0, "E"}, {"latVertex", 0, 0, 0, 0, "V"}, {"lonVertex", 0, 0, 0, 0, "V"},
      {"xVertex", 0, 0, 0, 1, "V"}, {"yVertex", 0, 0, 0, 1, "V"}, {"zVertex", 0, 0, 0, 1, "V"},
      {"defc_a", 0, 0, 0, 0, "M,C"}, {"defc_b", 0, 0, 0, 0, "M,C"},
      {"localVerticalUnitVectors", 0, 0, 0, 0, "R3,C"}, {"edgeNormalVectors", 0, 0, 0, 0, "R3,E"},
      {"cellTangentPlane", 0, 0, 0, 0, "R3,2,C"}, {"coeffs_reconstruct", 0, 0, 0, 1, "R3,M,C"},
      {"tend_u", 0, 0, 2, 0, "L,E"}, {"tend_h", 0, 0, 1, 0, "L,C"}, {"tend_tracer", 0, 0, 0, 0, "T,L,C"},
      {"u_tl", 1, 0, 2, 0, "2,L,E"}, {"h_tl", 1, 0, 1, 0, "2,L,C"}, {"tracers_tl", 1, 0, 0, 0, "2,T,L,C"},
      {"tend_u_tl", 1, 0, 2, 0, "L,E"}, {"tend_h_tl", 1, 0, 1, 0, "L,C"},
      {"tend_tracer_tl", 1, 0, 0, 0, "T,L,C"},
      {"u_ad", 2, 0, 2, 0, "2,L,E"}, {"h_ad", 2, 0, 1, 0, "2,L,C"}, {"tracers_ad", 2, 0, 0, 0, "2,T,L,C"},
      {"tend_u_ad", 2, 0, 2, 0, "L,E"}, {"tend_h_ad", 2, 0, 1, 0, "L,C"},
      {"tend_tracer_ad", 2, 0, 0, 0, "T,L,C"},
  };
  static std::vector<std::string> names;  // storage for the generated diagnostic names
  if (names.empty())
    for (int g = 0; g < 3; g++)
      for (int i = 0; i < 19; i++) names.push_back(std::string(kDiagNames[i]) + (g == 1 ? "_tl" : g == 2 ? "_ad" : ""));
  for (int g = 0; g < 3; g++)
    for (int i = 0; i < 19; i++) {
      const int e = kDiagEnt[i];
      s.push_back({names[g * 19 + i].c_str(), g, 0, e, 0, e == 1 ? "L,C" : e == 2 ? "L,E" : "L,V"});
    }
  return s;
}

const std::vector<VarSpec> &specs() {
  static std::vector<VarSpec> s = make_specs();
  return s;
}

struct ScalarSpec {
  const char *name;
  double def;
  int readonly;
};
const ScalarSpec kScalars[] = {
    // src/mpas_sw_module.f90:8-18 constants
    {"pii", 3.141592653589793, 1}, {"a", 6371229.0, 1}, {"omega", 7.29212e-5, 1},
    {"gravity", 9.80616, 1}, {"rgas", 287.0, 1}, {"rv", 461.6, 1}, {"rvord", 461.6 / 287.0, 1},
    {"cp", 7. * 287.0 / 2., 1}, {"cv", 7. * 287.0 / 2. - 287.0, 1},
    {"cvpm", -(7. * 287.0 / 2. - 287.0) / (7. * 287.0 / 2.), 1}, {"prandtl", 1.0, 1},
    // :23-42 configuration
    {"config_test_case", 5, 0}, {"config_dt", 150.0, 0}, {"config_stats_interval", 100, 0},
    {"config_h_scalewithmesh", 0, 0}, {"config_h_mom_eddy_visc2", 0.0, 0},
    {"config_h_mom_eddy_visc4", 0.0, 0}, {"config_h_tracer_eddy_diff2", 0.0, 0},
    {"config_h_tracer_eddy_diff4", 0.0, 0}, {"config_thickness_adv_order", 2, 0},
    {"config_tracer_adv_order", 2, 0}, {"config_positive_definite", 0, 0},
    {"config_monotonic", 0, 0}, {"config_wind_stress", 0, 0}, {"config_bottom_drag", 0, 0},
    {"config_apvm_upwinding", 0.5, 0}, {"config_num_halos", 2, 0},
    // tracer transport in sw_rk4 (no counterpart in the reference, which leaves it out): off
    {"config_advect_tracers", 0, 0},
    // :45-55 dimensions
    {"nvertlevels", 1, 0}, {"ncells", 0, 0}, {"nedges", 0, 0}, {"nvertices", 0, 0},
    {"ntracers", 0, 0}, {"cellstart", 0, 0}, {"cellend", 0, 0}, {"vertexstart", 0, 0},
    {"vertexend", 0, 0}, {"edgestart", 0, 0}, {"edgeend", 0, 0}, {"vertexdegree", 0, 0},
    {"ncellssolve", 0, 0}, {"nedgessolve", 0, 0}, {"maxedges", 0, 0}, {"maxedges2", 0, 0},
    {"cellsolvestart", 0, 0}, {"cellsolveend", 0, 0}, {"edgesolvestart", 0, 0},
    {"edgesolveend", 0, 0}, {"r3", 0, 0},
    // :73-75, :117, :206-207
    {"on_a_sphere", 0, 0}, {"is_periodic", 0, 0}, {"x_period", 0.0, 0}, {"y_period", 0.0, 0},
    {"sphere_radius", 0.0, 0}, {"rk_step", 0, 0}, {"lhs", 0.0, 0}, {"rhs", 0.0, 0}, {"pt", 0.0, 0},
};

}  // namespace

// ---------------------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------------------
Var *Engine::find(const std::string &lname) {
  auto it = index.find(lname);
  return it == index.end() ? nullptr : &vars[it->second];
}
Var &Engine::var(const char *name) {
  Var *v = find(lower(name));
  if (!v) throw EngineError(MPSW_ERR_ARG, std::string("unknown module variable ") + name);
  return *v;
}

double Engine::sc(const char *name) const {
  auto it = scal.find(name);
  return it == scal.end() ? 0.0 : it->second;
}

long long Engine::dim_of(const std::string &sym) const {
  if (sym == "L") return (long long)sc("nvertlevels");
  if (sym == "C") return nC;
  if (sym == "E") return nE;
  if (sym == "V") return nV;
  if (sym == "M") return mE;
  if (sym == "M2") return mE2;
  if (sym == "D") return vd;
  if (sym == "T") return nT;
  if (sym == "R3") return (long long)sc("r3");
  return std::stoll(sym);
}

Engine::Engine() {
  for (const auto &s : kScalars) scal[s.name] = s.def;
  refresh_phys();
  for (const auto &s : specs()) {
    Var v;
    v.name = s.name;
    v.group = s.group;
    v.is_int = s.is_int;
    v.ent = s.ent;
    v.mesh = s.mesh;
    v.dims_spec = s.dims;
    index[lower(s.name)] = (int)vars.size();
    vars.push_back(std::move(v));
  }
}

// The CUDA context is touched only when a routine first needs the device, so handles can be
// created, filled and inspected on a machine without a GPU.
void Engine::need_device() {
  if (stream) return;
  cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "cudaStreamCreate");
  for (cudaEvent_t *ev : {&ev_fork, &ev_step, &ev_join})
    cuda_check(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaMalloc(&d_bad, sizeof(int)), "cudaMalloc flag");
  cuda_check(cudaMemsetAsync(d_bad, 0, sizeof(int), stream), "clear flag");
}

Engine::~Engine() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto &v : vars)
    if (v.dev) cudaFree(v.dev);
  free_device_mesh();
  for (void *p : work) cudaFree(p);
  if (trc) cudaFree(trc);
  window_free();
  if (l2_flush) cudaFree(l2_flush);
  if (d_bad) cudaFree(d_bad);
  for (cudaEvent_t ev : {ev_fork, ev_step, ev_join})
    if (ev) cudaEventDestroy(ev);
  if (side) cudaStreamDestroy(side);
  if (stream) cudaStreamDestroy(stream);
}

void *Engine::l2_flush_buffer() {
  if (!l2_flush) cuda_check(cudaMalloc(&l2_flush, kL2Flush), "cudaMalloc L2 flush buffer");
  return l2_flush;
}

void *Engine::dalloc(size_t bytes) {
  need_device();
  void *p = nullptr;
  cuda_check(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc");
  cuda_check(cudaMemsetAsync(p, 0, bytes ? bytes : 16, stream), "cudaMemset");
  return p;
}

void Engine::allocate_group(int g) {
  if (g == 0) {
    nC = (int)sc("ncells");
    nE = (int)sc("nedges");
    nV = (int)sc("nvertices");
    mE = (int)sc("maxedges");
    mE2 = (int)sc("maxedges2");
    vd = (int)sc("vertexdegree");
    nT = (int)sc("ntracers");
    if (nC <= 0 || nE <= 0 || nV <= 0) throw EngineError(MPSW_ERR_STATE, "dimensions not set before var_allocation");
    if ((int)sc("nvertlevels") != 1) throw EngineError(MPSW_ERR_UNSUPPORTED, "nVertLevels must be 1");
    if ((int)sc("r3") == 0) scal["r3"] = 3;
  } else if (!allocated[0]) {
    throw EngineError(MPSW_ERR_STATE, "var_allocation must be called first");
  }
  for (auto &v : vars) {
    if (v.group != g) continue;
    v.dims.clear();
    size_t start = 0;
    const std::string d = v.dims_spec;
    while (start <= d.size()) {
      size_t comma = d.find(',', start);
      if (comma == std::string::npos) comma = d.size();
      v.dims.push_back(dim_of(d.substr(start, comma - start)));
      start = comma + 1;
    }
    long long n = 1;
    for (auto x : v.dims) n *= x;
    v.count = n;
    if (v.is_int) v.hi.assign(n, 0); else v.hr.assign(n, 0.0);
    v.allocated = true;
    v.host_valid = true;
    v.nonzero = false;
    if (v.ent) {
      const long long ne = v.ent == 1 ? nC : v.ent == 2 ? nE : nV;
      v.lead = (int)(n / ne);
      if (v.dev) {
        graphs_free();  // captured launches hold variable pointers
        cudaFree(v.dev);
      }
      v.dev = nullptr;      // allocated when a routine first needs the device
      v.dev_valid = false;
    }
  }
  allocated[g] = true;
  if (g == 0) mesh_dirty = true;
}

// ---- transfers -------------------------------------------------------------------------
const std::vector<int> &Engine::perm_of(int ent) const {
  return ent == 1 ? bm.perm_c : ent == 2 ? bm.perm_e : bm.perm_v;
}

void Engine::upload(Var &v) {
  if (!v.ent || (v.dev && v.dev_valid)) return;
  if (!v.dev) v.dev = (double *)dalloc(sizeof(double) * v.count);
  if (!mesh_built) throw EngineError(MPSW_ERR_STATE, "mesh not initialised (call sw_mpas_init_block)");
  const auto &p = perm_of(v.ent);
  const long long n = (long long)p.size();
  staging.resize(v.count);
  for (long long i = 0; i < n; i++)
    for (int l = 0; l < v.lead; l++) staging[(size_t)l * n + p[i]] = v.hr[(size_t)l + (size_t)v.lead * i];
  cuda_check(cudaMemcpyAsync(v.dev, staging.data(), sizeof(double) * v.count, cudaMemcpyHostToDevice, stream), "upload");
  cuda_check(cudaStreamSynchronize(stream), "upload sync");
  v.dev_valid = true;
}

void Engine::download(Var &v) {
  if (!v.ent || v.host_valid) return;
  const auto &p = perm_of(v.ent);
  const long long n = (long long)p.size();
  staging.resize(v.count);
  cuda_check(cudaMemcpyAsync(staging.data(), v.dev, sizeof(double) * v.count, cudaMemcpyDeviceToHost, stream), "download");
  cuda_check(cudaStreamSynchronize(stream), "download sync");
  for (long long i = 0; i < n; i++)
    for (int l = 0; l < v.lead; l++) v.hr[(size_t)l + (size_t)v.lead * i] = staging[(size_t)l * n + p[i]];
  v.host_valid = true;
}

void Engine::set_var(const char *name, const void *src, long long count) {
  Var &v = var(name);
  if (!v.allocated) throw EngineError(MPSW_ERR_STATE, std::string(name) + " is not allocated");
  if (count != v.count) throw EngineError(MPSW_ERR_ARG, std::string(name) + ": element count mismatch");
  if (!src && count) throw EngineError(MPSW_ERR_ARG, "null source buffer");
  if (v.is_int) {
    std::memcpy(v.hi.data(), src, sizeof(int) * count);
  } else {
    std::memcpy(v.hr.data(), src, sizeof(double) * count);
    v.nonzero = std::any_of(v.hr.begin(), v.hr.end(), [](double x) { return x != 0.0; });
  }
  v.host_valid = true;
  if (v.ent) v.dev_valid = false;
  if (v.mesh) mesh_dirty = true;
}

void Engine::get_var(const char *name, void *dst, long long count) {
  Var &v = var(name);
  if (!v.allocated) throw EngineError(MPSW_ERR_STATE, std::string(name) + " is not allocated");
  if (count != v.count) throw EngineError(MPSW_ERR_ARG, std::string(name) + ": element count mismatch");
  if (!dst && count) throw EngineError(MPSW_ERR_ARG, "null destination buffer");
  if (v.ent && !v.host_valid) {
    if (v.lazy_diag) materialize_pending();
    download(v);
  }
  if (v.is_int) std::memcpy(dst, v.hi.data(), sizeof(int) * count);
  else std::memcpy(dst, v.hr.data(), sizeof(double) * count);
}

void Engine::mark_written(Var &v, bool maybe_nonzero) {
  v.dev_valid = true;
  v.host_valid = false;
  v.nonzero = maybe_nonzero;
}

// ---- device mesh -----------------------------------------------------------------------
template <typename T, typename S>
const T *Engine::up(const std::vector<S> &h, std::vector<void *> &own) {
  std::vector<T> t(h.begin(), h.end());
  void *p = nullptr;
  cuda_check(cudaMalloc(&p, sizeof(T) * (t.empty() ? 1 : t.size())), "cudaMalloc mesh");
  if (!t.empty()) cuda_check(cudaMemcpy(p, t.data(), sizeof(T) * t.size(), cudaMemcpyHostToDevice), "mesh upload");
  own.push_back(p);
  return (const T *)p;
}

template <typename R>
void Engine::fill_mesh(MeshDev<R> &m) {
  auto &o = mesh_bufs;
  m.nC = bm.nC;
  m.nE = bm.nE;
  m.nV = bm.nV;
  m.max_eoe = bm.e_n.empty() ? 0 : *std::max_element(bm.e_n.begin(), bm.e_n.end());
  m.max_eoc = bm.c_n.empty() ? 0 : *std::max_element(bm.c_n.begin(), bm.c_n.end());
  m.c_n = up<int>(bm.c_n, o);
  m.c_eoc = up<int>(bm.c_eoc, o);
  m.c_es = up<int>(bm.c_es, o);
  m.c_esg = up<signed char>(bm.c_esg, o);

  m.c_vs = up<int>(bm.c_vs, o);
  m.c_vk = up<R>(bm.c_vk, o);
  m.c_area = up<R>(bm.c_area, o);
  m.c_hs = up<R>(bm.c_hs, o);
  m.c_coef = up<R>(bm.c_coef, o);
  m.c_trig = up<R>(bm.c_trig, o);
  m.e_c1 = up<int>(bm.e_c1, o);
  m.e_c2 = up<int>(bm.e_c2, o);
  m.e_v1 = up<int>(bm.e_v1, o);
  m.e_v2 = up<int>(bm.e_v2, o);
  m.e_va = up<int>(bm.e_va, o);
  m.e_vb = up<int>(bm.e_vb, o);
  m.e_slot1 = up<int>(bm.e_slot1, o);
  m.e_slot2 = up<int>(bm.e_slot2, o);
  m.e_n = up<int>(bm.e_n, o);
  m.e_eoe = up<int>(bm.e_eoe, o);
  m.e_rev = up<int>(bm.e_rev, o);
  m.e_w = up<R>(bm.e_w, o);
  m.e_wrev = up<R>(bm.e_wrev, o);
  m.e_dc = up<R>(bm.e_dc, o);
  m.e_dv = up<R>(bm.e_dv, o);
  m.e_sc2 = up<R>(bm.e_sc2, o);
  m.e_sc4 = up<R>(bm.e_sc4, o);
  m.e_usrc = up<R>(bm.e_usrc, o);
  m.v_es = up<int>(bm.v_es, o);
  m.v_esg = up<signed char>(bm.v_esg, o);
  m.v_c = up<int>(bm.v_c, o);
  m.v_k = up<R>(bm.v_k, o);
  m.v_e = up<int>(bm.v_e, o);
  m.v_area = up<R>(bm.v_area, o);
  m.v_f = up<R>(bm.v_f, o);
}

void Engine::free_device_mesh() {
  graphs_free();  // captured launches hold mesh pointers
  for (void *p : mesh_bufs) cudaFree(p);
  mesh_bufs.clear();
  mesh_built = false;
  fused = FusedDev();
  fused_K = 0;
}

// Halo tiles of the fused FP32 member stages (meshes with at most 6 edges per cell and 10
// edgesOnEdge), built when MPSW_FUSED=1 is set as the mesh goes to the device (the sweeps use
// the split member kernels otherwise).  MPSW_FUSED_M sets the members per chunk the tiles are
// sized for (4, 8, 16 or 32; default 8), MPSW_FUSED_NT the threads per block (256, 512 or 1024;
// default 512), MPSW_FUSED_SMEM the shared memory of a tile's block in KB (default 110) and
// MPSW_FUSED_K the most cells a tile owns (default 1024).
void Engine::build_fused() {
  fused = FusedDev();
  fused_K = 0;
  const char *on = getenv("MPSW_FUSED");
  if (!on || atoi(on) != 1) return;
  if (m32.max_eoe > 10 || m32.max_eoc > 6) return;  // the tiles hold 10 edgesOnEdge, 6 edges per cell
  auto env = [](const char *n, int dflt) {
    const char *e = getenv(n);
    return e && atoi(e) > 0 ? atoi(e) : dflt;
  };
  const int K = env("MPSW_FUSED_K", 1024), M = env("MPSW_FUSED_M", 8), NT = env("MPSW_FUSED_NT", 512);
  const size_t budget = (size_t)env("MPSW_FUSED_SMEM", 110) << 10;
  if (M != 4 && M != 8 && M != 16 && M != 32) throw EngineError(MPSW_ERR_ARG, "MPSW_FUSED_M must be 4, 8, 16 or 32");
  if (NT != 256 && NT != 512 && NT != 1024) throw EngineError(MPSW_ERR_ARG, "MPSW_FUSED_NT must be 256, 512 or 1024");
  TileSetHost th[2];
  for (int a = 0; a < 2; a++) {
    const std::string err = build_tiles(bm, budget, K, M, a == 1, &th[a]);
    if (!err.empty()) throw EngineError(MPSW_ERR_MESH, "fused tiles: " + err);
  }
  auto &o = mesh_bufs;
  for (int a = 0; a < 2; a++) {
    TileSetDev &d = a ? fused.ad : fused.tl;
    const TileSetHost &t = th[a];
    d.ntiles = t.ntiles;
    d.cnt = up<int>(t.cnt, o);
    d.blob_off = up<long long>(t.blob_off, o);
    d.blob = up<unsigned char>(t.blob, o);
    for (int i = 0; i < 4; i++) d.smem[i] = t.smem[i];
  }
  fused.M = M;
  fused.nt = NT;
  cuda_check(Launch<float, double>::fused_prepare(fused), "fused stage shared-memory limit");
  fused.ok = true;
  fused_K = K;
}

RefMesh Engine::ref_mesh() {
  RefMesh r;
  r.nC = nC; r.nE = nE; r.nV = nV; r.maxEdges = mE; r.maxEdges2 = mE2; r.vd = vd;
  auto I = [&](const char *n) { return var(n).hi.data(); };
  auto D = [&](const char *n) { return var(n).hr.data(); };
  r.cellsOnEdge = I("cellsOnEdge"); r.verticesOnEdge = I("verticesOnEdge");
  r.edgesOnEdge = I("edgesOnEdge"); r.nEdgesOnEdge = I("nEdgesOnEdge");
  r.edgesOnCell = I("edgesOnCell"); r.nEdgesOnCell = I("nEdgesOnCell");
  r.cellsOnVertex = I("cellsOnVertex"); r.edgesOnVertex = I("edgesOnVertex");
  r.weightsOnEdge = D("weightsOnEdge"); r.kiteAreasOnVertex = D("kiteAreasOnVertex");
  r.dcEdge = D("dcEdge"); r.dvEdge = D("dvEdge"); r.areaCell = D("areaCell");
  r.areaTriangle = D("areaTriangle"); r.fVertex = D("fVertex"); r.h_s = D("h_s");
  r.u_src = D("u_src"); r.meshDensity = D("meshDensity");
  r.xCell = D("xCell"); r.yCell = D("yCell"); r.zCell = D("zCell");
  r.xEdge = D("xEdge"); r.yEdge = D("yEdge"); r.zEdge = D("zEdge");
  r.xVertex = D("xVertex"); r.yVertex = D("yVertex"); r.zVertex = D("zVertex");
  r.latCell = D("latCell"); r.lonCell = D("lonCell");
  r.on_a_sphere = sc("on_a_sphere") != 0.0;
  r.h_ScaleWithMesh = sc("config_h_scalewithmesh") != 0.0;
  return r;
}

void Engine::build_device_mesh() {
  // states on the device are in the old internal order: bring them home first
  for (auto &v : vars)
    if (v.ent && v.allocated && !v.host_valid) {
      if (v.lazy_diag) materialize_pending();
      download(v);
    }
  RefMesh r = ref_mesh();
  std::string e = validate_mesh(r);
  if (!e.empty()) throw EngineError(MPSW_ERR_MESH, e);
  for (double x : var("deriv_two").hr)
    if (x != 0.0 && (int)sc("config_thickness_adv_order") != 2)
      throw EngineError(MPSW_ERR_UNSUPPORTED, "thickness_adv_order 3/4 with nonzero deriv_two is not supported");
  for (int x : var("boundaryEdge").hi)
    if (x != 0) throw EngineError(MPSW_ERR_UNSUPPORTED, "boundary edges (regional meshes) are not supported");
  RefGeometry g;
  g.meshScalingDel2 = var("meshScalingDel2").hr;
  g.meshScalingDel4 = var("meshScalingDel4").hr;
  g.coeffs_reconstruct = var("coeffs_reconstruct").hr;
  const char *sfc_env = getenv("MPSW_SFC");
  const int sfc = sfc_env ? atoi(sfc_env) : 1;
  bm = BuiltMesh();
  e = build_mesh(r, g, sfc, &bm);
  if (!e.empty()) throw EngineError(MPSW_ERR_MESH, e);
  graphs_free();
  free_device_mesh();
  fill_mesh(m64);
  fill_mesh(m32);
  {  // the cell across each edge of a cell, in the order of c_es
    std::vector<int> nb(bm.c_es.size(), 0);
    for (int k = 0; k < MAXE; k++)
      for (int c = 0; c < bm.nC; c++) {
        const size_t i = (size_t)k * bm.nC + c;
        if (k >= bm.c_n[c]) continue;
        const int e = bm.c_es[i];
        nb[i] = bm.e_c1[e] == c ? bm.e_c2[e] : bm.e_c1[e];
      }
    d_cnb = up<int>(nb, mesh_bufs);
  }
  d_perm[0] = up<int>(bm.perm_c, mesh_bufs);
  d_perm[1] = up<int>(bm.perm_e, mesh_bufs);
  d_perm[2] = up<int>(bm.perm_v, mesh_bufs);
  cuda_check(cudaGetDevice(&mesh_device), "cudaGetDevice");
  build_fused();
  noalloc_prepare_device();
  mesh_built = true;
  mesh_dirty = false;
  for (auto &v : vars)
    if (v.ent && v.allocated) v.dev_valid = false;
  alloc_work();
  window_free();
}

void Engine::ensure_mesh() {
  if (!allocated[0]) throw EngineError(MPSW_ERR_STATE, "var_allocation has not been called");
  need_device();
  if (mesh_dirty || !mesh_built) build_device_mesh();
}

void Engine::sync_inputs() {
  for (auto &v : vars)
    if (v.ent && v.allocated && (!v.dev || !v.dev_valid)) upload(v);
}

// ---- work buffers ------------------------------------------------------------------------
double *Engine::wbuf(size_t n) {
  void *p = dalloc(sizeof(double) * n);
  work.push_back(p);
  return (double *)p;
}

Diag<double> Engine::new_diag(int B) {
  Diag<double> d{};
  d.circ = wbuf((size_t)nV * B); d.vort = wbuf((size_t)nV * B); d.hv = wbuf((size_t)nV * B);
  d.pvv = wbuf((size_t)nV * B); d.div = wbuf((size_t)nC * B); d.ke = wbuf((size_t)nC * B);
  d.pc = wbuf((size_t)nC * B); d.vc = wbuf((size_t)nC * B); d.v = wbuf((size_t)nE * B);
  d.gpt = wbuf((size_t)nE * B); d.pe = wbuf((size_t)nE * B); d.gpn = wbuf((size_t)nE * B);
  d.he = wbuf((size_t)nE * B); d.dsq_u = wbuf((size_t)nE * B); d.dsq_vort = wbuf((size_t)nV * B);
  d.dsq_div = wbuf((size_t)nC * B);
  return d;
}

void Engine::alloc_work() {
  graphs_free();  // captured launches hold work-buffer pointers
  for (void *p : work) cudaFree(p);
  work.clear();
  for (int k = 0; k < 5; k++) stage[k] = new_diag(1);
  tl_diag = new_diag(1);
  for (int k = 0; k < 4; k++) {
    sp_u[k] = wbuf(nE); sp_h[k] = wbuf(nC);
    tp_u[k] = wbuf(nE); tp_h[k] = wbuf(nC);
  }
  acc_u = wbuf(nE); acc_h = wbuf(nC); tacc_u = wbuf(nE); tacc_h = wbuf(nC);
  adw.pe_ad = wbuf(nE); adw.he_ad = wbuf(nE); adw.ud = wbuf(nE); adw.gpn_ad = wbuf(nE);
  adw.gpt_ad = wbuf(nE); adw.v_ad = wbuf(nE); adw.du_ad = wbuf(nE);
  adw.pc_ad = wbuf(nC); adw.ke_ad = wbuf(nC); adw.div_ad = wbuf(nC); adw.hd = wbuf(nC); adw.dd_ad = wbuf(nC);
  adw.hv_ad = wbuf(nV); adw.circ_ad = wbuf(nV); adw.dc_ad = wbuf(nV);
  for (int k = 0; k < 2; k++) { tu_[k] = wbuf(nE); th_[k] = wbuf(nC); }
  auto fbuf = [&](size_t n) {
    void *p = dalloc(sizeof(float) * n);
    work.push_back(p);
    return (float *)p;
  };
  d32 = Diag<float>{};
  d32.vort = fbuf(nV); d32.hv = fbuf(nV); d32.pvv = fbuf(nV); d32.div = fbuf(nC); d32.ke = fbuf(nC);
  d32.pc = fbuf(nC); d32.v = fbuf(nE); d32.gpt = fbuf(nE); d32.pe = fbuf(nE); d32.gpn = fbuf(nE);
  d32.he = fbuf(nE); d32.dsq_u = fbuf(nE); d32.dsq_vort = fbuf(nV); d32.dsq_div = fbuf(nC);
  for (int k = 0; k < 4; k++) { s32_u[k] = fbuf(nE); s32_h[k] = fbuf(nC); }
  xacc_u = wbuf(nE); xacc_h = wbuf(nC);
}

// ---- module diagnostics as kernel arguments ----------------------------------------------
double *Engine::dv(const char *name, int level) {
  Var &v = var(name);
  const long long ne = v.ent == 1 ? nC : v.ent == 2 ? nE : nV;
  return v.dev + (size_t)level * ne;
}

Diag<double> Engine::module_diag(int g) {
  const char *sfx = g == 1 ? "_tl" : g == 2 ? "_ad" : "";
  auto P = [&](const char *n) { return dv((std::string(n) + sfx).c_str()); };
  Diag<double> d{};
  d.circ = P("circulation"); d.vort = P("vorticity"); d.hv = P("h_vertex"); d.pvv = P("pv_vertex");
  d.div = P("divergence"); d.ke = P("ke"); d.pc = P("pv_cell"); d.vc = P("vorticity_cell");
  d.v = P("v"); d.gpt = P("gradPVt"); d.pe = P("pv_edge"); d.gpn = P("gradPVn"); d.he = P("h_edge");
  const Diag<double> &sc_ = g == 1 ? tl_diag : stage[0];
  d.dsq_u = sc_.dsq_u; d.dsq_vort = sc_.dsq_vort; d.dsq_div = sc_.dsq_div;
  return d;
}

void Engine::mark_diag(int g, bool lazy) {
  const char *sfx = g == 1 ? "_tl" : g == 2 ? "_ad" : "";
  for (int i = 5; i < 19; i++) {
    Var &v = var((std::string(kDiagNames[i]) + sfx).c_str());
    mark_written(v, true);
    v.lazy_diag = lazy;
  }
}

void Engine::mark_recon(int g) {
  const char *sfx = g == 1 ? "_tl" : g == 2 ? "_ad" : "";
  for (int i = 0; i < 5; i++) mark_written(var((std::string(kDiagNames[i]) + sfx).c_str()), g != 2);
}

Phys<double> Engine::phys() const {
  Phys<double> p = phys_cache;
  p.bad = d_bad;
  return p;
}

// The flag the tendency kernels raise on a non-finite value: cleared at the start of a routine
// (prepare, or a window sweep), read when it has finished.
void Engine::nonfinite_clear() {
  if (d_bad) cuda_check(cudaMemsetAsync(d_bad, 0, sizeof(int), stream), "clear non-finite flag");
}
void Engine::nonfinite_check(const char *what) {
  if (!d_bad) return;
  int v = 0;
  cuda_check(cudaMemcpyAsync(&v, d_bad, sizeof(int), cudaMemcpyDeviceToHost, stream), "read non-finite flag");
  cuda_check(cudaStreamSynchronize(stream), what);
  if (v)
    throw EngineError(MPSW_ERR_NONFINITE, std::string(what) +
                                              ": a tendency became non-finite (NaN or Inf); the state or the "
                                              "members are corrupt or the time step is unstable");
}

void Engine::refresh_phys() {
  Phys<double> &p = phys_cache;
  p.dt = sc("config_dt");
  p.apvm = sc("config_apvm_upwinding");
  p.visc2 = sc("config_h_mom_eddy_visc2");
  p.visc4 = sc("config_h_mom_eddy_visc4");
  p.wind = sc("config_wind_stress") != 0.0;
  p.drag = sc("config_bottom_drag") != 0.0;
  p.tc1 = (int)sc("config_test_case") == 1;
  p.sphere = sc("on_a_sphere") != 0.0;
}

// ---- stage building blocks ---------------------------------------------------------------
using L64 = Launch<double, double>;

void Engine::fwd_diag(const double *u, const double *h, const Diag<double> &d, const Phys<double> &ph) {
  RK<double, double> none{};
  L64::fwd_vertex(m64, u, h, 0.0, d, stream);
  L64::fwd_cell(m64, d_cnb, u, h, 0.0, d, none, nullptr, stream);
  L64::fwd_edge_diag(m64, u, h, 0.0, d, ph, stream);
  if (ph.visc4 > 0) L64::del4_vc(m64, 1, d.dsq_u, d.dsq_vort, d.dsq_div, stream);
}

void Engine::fwd_stage(const double *u, const double *h, const Diag<double> &d, const Phys<double> &ph,
                       const RK<double, double> &rku, const RK<double, double> &rkh, double *tu, double *th) {
  L64::fwd_vertex(m64, u, h, 0.0, d, stream);
  L64::fwd_cell(m64, d_cnb, u, h, 0.0, d, rkh, th, stream);
  L64::fwd_edge_diag(m64, u, h, 0.0, d, ph, stream);
  if (ph.visc4 > 0) L64::del4_vc(m64, 1, d.dsq_u, d.dsq_vort, d.dsq_div, stream);
  L64::fwd_edge_tend(m64, u, h, 0.0, d, ph, rku, tu, stream);
}

static Base<double> base_of(const Diag<double> &d, const double *u) {
  Base<double> b{};
  b.u = u; b.he = d.he; b.v = d.v; b.gpt = d.gpt; b.gpn = d.gpn; b.pe = d.pe;
  b.vort = d.vort; b.hv = d.hv; b.ke = d.ke;
  return b;
}

void Engine::tl_diag_run(const Base<double> &bs, const double *ut, const double *ht, const Diag<double> &d,
                         const Phys<double> &ph) {
  RK<double, double> none{};
  L64::tl_vertex(m64, 1, bs, ut, ht, d, stream);
  L64::tl_cell(m64, 1, bs, ut, ht, d, none, nullptr, stream);
  L64::tl_edge_diag(m64, 1, bs, ut, ht, d, ph, stream);
  if (ph.visc4 > 0) L64::del4_vc(m64, 1, d.dsq_u, d.dsq_vort, d.dsq_div, stream);
}

void Engine::check_launch(const char *what) {
  cuda_check(cudaGetLastError(), what);
  cuda_check(cudaStreamSynchronize(stream), what);
}

// Lazily computed diagnostics of the state left by the last routine (the reference's final
// sw_compute_solve_diagnostics call of sw_rk4 / sw_rk4_tlm, src/mpas_sw_module.f90:616,754).
void Engine::materialize_pending() {
  if (!pending_diag) return;
  const Phys<double> ph = phys();
  Diag<double> d = module_diag(0);
  fwd_diag(dv("u"), dv("h"), d, ph);
  if (pending_diag == 2) {
    Diag<double> dt = module_diag(1);
    tl_diag_run(base_of(d, dv("u")), dv("u_tl"), dv("h_tl"), dt, ph);
  }
  check_launch("diagnostics");
  for (int g = 0; g < (pending_diag == 2 ? 2 : 1); g++) {
    const char *sfx = g == 1 ? "_tl" : "";
    for (int i = 5; i < 19; i++) var((std::string(kDiagNames[i]) + sfx).c_str()).lazy_diag = false;
  }
  pending_diag = 0;
}

// ---------------------------------------------------------------------------------------
// Module subroutines
// ---------------------------------------------------------------------------------------
void Engine::init_block() {  // src/mpas_sw_module.f90:495-526
  if (!allocated[0]) throw EngineError(MPSW_ERR_STATE, "var_allocation has not been called");
  RefMesh r = ref_mesh();
  std::string e = validate_mesh(r);
  if (!e.empty()) throw EngineError(MPSW_ERR_MESH, e);
  RefGeometry g;
  compute_geometry(r, &g);
  var("meshScalingDel2").hr = g.meshScalingDel2;
  var("meshScalingDel4").hr = g.meshScalingDel4;
  var("localVerticalUnitVectors").hr = g.localVerticalUnitVectors;
  var("edgeNormalVectors").hr = g.edgeNormalVectors;
  var("cellTangentPlane").hr = g.cellTangentPlane;
  var("coeffs_reconstruct").hr = g.coeffs_reconstruct;
  mesh_dirty = true;
  ensure_mesh();
  sync_inputs();
  pending_diag = 0;
  const Phys<double> ph = phys();
  fwd_diag(dv("u"), dv("h"), module_diag(0), ph);
  L64::recon(m64, 1, ph.sphere, dv("u"), dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  check_launch("sw_mpas_init_block");
  mark_diag(0, false);
  mark_recon(0);
}

void Engine::prepare() {
  ensure_mesh();
  sync_inputs();
  nonfinite_clear();
}

// rk weights (src/mpas_sw_module.f90:567-575)
static void rk_coeffs(double dt, double w[4], double c[4]) {
  w[0] = dt / 6.; w[1] = dt / 3.; w[2] = dt / 3.; w[3] = dt / 6.;
  c[0] = dt / 2.; c[1] = dt / 2.; c[2] = dt; c[3] = 0.;
}

// ---- tracer transport -------------------------------------------------------------------
bool Engine::tracers_advected() {
  if (sc("config_advect_tracers") == 0.0 || nT <= 0) return false;
  if (!var("tracers").allocated) throw EngineError(MPSW_ERR_STATE, "tracers are not allocated");
  if (sc("config_tracer_adv_order") != 2.0 || sc("config_h_tracer_eddy_diff2") != 0.0 ||
      sc("config_h_tracer_eddy_diff4") != 0.0)
    throw EngineError(MPSW_ERR_UNSUPPORTED, "tracer transport supports config_tracer_adv_order 2 without eddy diffusion");
  return true;
}

// six [nT][nC] device blocks, reallocated (and the step graphs dropped) when nT or nC changes
double *Engine::tracer_bufs() {
  const long long n = 6LL * nT * nC;
  if (trc_n != n) {
    graphs_free();
    if (trc) cudaFree(trc);
    trc = (double *)dalloc(sizeof(double) * n);
    trc_n = n;
  }
  return trc;
}

// tracers(1, :, 1, c) -> [nT][nC] in internal cell order
void Engine::tracers_upload(double *dst) {
  const Var &v = var("tracers");
  const auto &p = perm_of(1);
  staging.assign((size_t)nT * nC, 0.0);
  for (int i = 0; i < nC; i++)
    for (int t = 0; t < nT; t++) staging[(size_t)t * nC + p[i]] = v.hr[2 * ((size_t)t + (size_t)nT * i)];
  cuda_check(cudaMemcpyAsync(dst, staging.data(), sizeof(double) * staging.size(), cudaMemcpyHostToDevice, stream),
             "tracers upload");
  cuda_check(cudaStreamSynchronize(stream), "tracers upload");
}

// both time levels of tracers and tend_tracer (the last stage's tendency) back into the module
void Engine::tracers_download(const double *src, const double *tend) {
  const auto &p = perm_of(1);
  Var &v = var("tracers");
  staging.resize((size_t)nT * nC);
  cuda_check(cudaMemcpyAsync(staging.data(), src, sizeof(double) * staging.size(), cudaMemcpyDeviceToHost, stream),
             "tracers download");
  cuda_check(cudaStreamSynchronize(stream), "tracers download");
  for (int i = 0; i < nC; i++)
    for (int t = 0; t < nT; t++) {
      const double x = staging[(size_t)t * nC + p[i]];
      v.hr[2 * ((size_t)t + (size_t)nT * i)] = x;
      v.hr[2 * ((size_t)t + (size_t)nT * i) + 1] = x;
    }
  v.nonzero = true;
  Var &tt = var("tend_tracer");
  if (!tt.allocated) return;
  cuda_check(cudaMemcpyAsync(staging.data(), tend, sizeof(double) * staging.size(), cudaMemcpyDeviceToHost, stream),
             "tend_tracer download");
  cuda_check(cudaStreamSynchronize(stream), "tend_tracer download");
  for (int i = 0; i < nC; i++)
    for (int t = 0; t < nT; t++) tt.hr[(size_t)t + (size_t)nT * i] = staging[(size_t)t * nC + p[i]];
  tt.nonzero = true;
}

void Engine::rk4(int nsteps) {  // src/mpas_sw_module.f90:528-635
  prepare();
  const Phys<double> ph = phys();
  double w[4], c[4];
  rk_coeffs(ph.dt, w, c);
  double *u0 = dv("u"), *h0 = dv("h");
  // tracer transport (config_advect_tracers): tracers(1) on the device for the whole call,
  // [nT][nC] blocks: the state, three provisional stages, the accumulator, the last tendency
  const bool adv = tracers_advected();
  double *tr0 = nullptr, *trp[3] = {}, *tracc = nullptr, *trtend = nullptr;
  if (adv) {
    tr0 = tracer_bufs();
    const size_t n = (size_t)nT * nC;
    for (int k = 0; k < 3; k++) trp[k] = tr0 + (k + 1) * n;
    tracc = tr0 + 4 * n;
    trtend = tr0 + 5 * n;
    tracers_upload(tr0);
  }
  auto step = [&]() {
    for (int k = 0; k < 4; k++) {
      const double *ui = k == 0 ? u0 : sp_u[k - 1];
      const double *hi = k == 0 ? h0 : sp_h[k - 1];
      RK<double, double> ru{u0, k == 0 ? u0 : acc_u, k == 3 ? u0 : acc_u, k < 3 ? sp_u[k] : nullptr, c[k], w[k], 0.0, ph.tc1};
      RK<double, double> rh{h0, k == 0 ? h0 : acc_h, k == 3 ? h0 : acc_h, k < 3 ? sp_h[k] : nullptr, c[k], w[k], 0.0, 0};
      fwd_stage(ui, hi, stage[0], ph, ru, rh, k == 3 ? dv("tend_u") : nullptr, k == 3 ? dv("tend_h") : nullptr);
      // after the stage: its h_edge is in stage[0], the next provisional h in sp_h[k] and, in
      // stage 4, the new h in h0
      if (adv)
        L64::tracer_stage(m64, d_cnb, nT, ui, stage[0].he, k == 0 ? tr0 : trp[k - 1], tr0, h0, k < 3 ? sp_h[k] : h0,
                          k == 3 ? trtend : nullptr, tracc, k < 3 ? trp[k] : nullptr, c[k], w[k], k == 0, k == 3,
                          stream);
    }
  };
  // one CUDA graph per step (its buffers are fixed), captured on the first step
  GraphKey key = graph_key(8, 0, 1, u0, h0);
  if (adv) {
    key.p3 = tr0;
    key.n2 = nT;
  }
  for (int n = 0; n < nsteps; n++) run_graph(key, step);
  if (adv) tracers_download(tr0, trtend);
  finish_levels({"u", "h"});
  L64::recon(m64, 1, ph.sphere, u0, dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  check_launch("sw_rk4");
  for (const char *n : {"u", "h", "tend_u", "tend_h"}) mark_written(var(n), true);
  mark_recon(0);
  mark_diag(0, true);
  pending_diag = 1;
  nonfinite_check("sw_rk4");  // after the bookkeeping: the outputs are on the device either way
}

// nsteps RK4 steps of the level-1 state.  Precision 0 is sw_rk4 repeated (bit-identical);
// precision 1 runs the stencils in FP32 and keeps the RK4 state and its accumulation in FP64:
// each step rounds u(1) and h(1) - h_ref to FP32 (h_ref: the mean depth at the call, so FP32
// carries the deviations from it), the four stages work on FP32 provisional states, and their
// tendencies are accumulated into the FP64 state in the reference's order.  Afterwards the
// module holds the new state, its reconstruction and (lazily) its FP64 diagnostics, as after
// sw_rk4.
void Engine::forward(int prec, int nsteps) {
  if (prec == 0) {
    rk4(nsteps);
    return;
  }
  if (prec != 1) throw EngineError(MPSW_ERR_ARG, "precision must be 0 or 1");
  if (nsteps < 0) throw EngineError(MPSW_ERR_ARG, "nsteps must be >= 0");
  if (tracers_advected())
    throw EngineError(MPSW_ERR_UNSUPPORTED, "tracer transport (config_advect_tracers) runs with FP64 stencils only");
  prepare();
  const Phys<double> ph64 = phys();
  Phys<float> ph{};
  ph.dt = (float)ph64.dt; ph.apvm = (float)ph64.apvm; ph.visc2 = (float)ph64.visc2; ph.visc4 = (float)ph64.visc4;
  ph.wind = ph64.wind; ph.drag = ph64.drag; ph.tc1 = ph64.tc1; ph.sphere = ph64.sphere; ph.bad = ph64.bad;
  double w[4], c[4];
  rk_coeffs(ph64.dt, w, c);
  double *u0 = dv("u"), *h0 = dv("h");
  // reference depth: the mean of h(1), rounded to a whole metre (exact in FP32)
  staging.resize(nC);
  cuda_check(cudaMemcpyAsync(staging.data(), h0, sizeof(double) * nC, cudaMemcpyDeviceToHost, stream), "h download");
  cuda_check(cudaStreamSynchronize(stream), "h download");
  double sum = 0;
  for (int i = 0; i < nC; i++) sum += staging[i];
  const double off = nC ? std::round(sum / nC) : 0.0;
  const float offf = (float)off;
  using L32 = Launch<float, double>;
  auto step = [&]() {
    convert_d2f(nE, u0, s32_u[0], stream);
    convert_d2f_off(nC, h0, off, s32_h[0], stream);
    for (int k = 0; k < 4; k++) {
      const float *ui = s32_u[k], *hi = s32_h[k];
      RK<float, double> ru{u0, k == 0 ? u0 : acc_u, k == 3 ? u0 : acc_u, k < 3 ? s32_u[k + 1] : nullptr, c[k], w[k], 0.f, ph.tc1};
      RK<float, double> rh{h0, k == 0 ? h0 : acc_h, k == 3 ? h0 : acc_h, k < 3 ? s32_h[k + 1] : nullptr, c[k], w[k], offf, 0};
      L32::fwd_vertex(m32, ui, hi, offf, d32, stream);
      L32::fwd_cell(m32, d_cnb, ui, hi, offf, d32, rh, nullptr, stream);
      L32::fwd_edge_diag(m32, ui, hi, offf, d32, ph, stream);
      if (ph.visc4 > 0.f) L32::del4_vc(m32, 1, d32.dsq_u, d32.dsq_vort, d32.dsq_div, stream);
      L32::fwd_edge_tend(m32, ui, hi, offf, d32, ph, ru, nullptr, stream);
    }
  };
  GraphKey key = graph_key(9, 1, 1, u0, h0);
  std::memcpy(&key.n2, &off, sizeof(off));
  for (int n = 0; n < nsteps; n++) run_graph(key, step);
  finish_levels({"u", "h"});
  L64::recon(m64, 1, ph64.sphere, u0, dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  check_launch("forward");
  for (const char *n : {"u", "h"}) mark_written(var(n), true);
  mark_recon(0);
  mark_diag(0, true);
  pending_diag = 1;
  nonfinite_check("forward");
}

// u(2) = u(1) after a step (src/mpas_sw_module.f90:631-632, 774-777)
void Engine::finish_levels(std::initializer_list<const char *> names) {
  for (const char *n : names) {
    Var &v = var(n);
    const long long ne = v.ent == 1 ? nC : nE;
    cuda_check(cudaMemcpyAsync(v.dev + ne, v.dev, sizeof(double) * ne, cudaMemcpyDeviceToDevice, stream), "level copy");
  }
}

void Engine::rk4_tlm(int nsteps) {  // src/mpas_sw_module.f90:637-781
  if (!allocated[1]) throw EngineError(MPSW_ERR_STATE, "var_allocation_tlm has not been called");
  prepare();
  const Phys<double> ph = phys();
  double w[4], c[4];
  rk_coeffs(ph.dt, w, c);
  double *u0 = dv("u"), *h0 = dv("h"), *ut0 = dv("u_tl"), *ht0 = dv("h_tl");
  for (int step = 0; step < nsteps; step++) {
    for (int k = 0; k < 4; k++) {
      const double *ui = k == 0 ? u0 : sp_u[k - 1];
      const double *hi = k == 0 ? h0 : sp_h[k - 1];
      RK<double, double> ru{u0, k == 0 ? u0 : acc_u, k == 3 ? u0 : acc_u, k < 3 ? sp_u[k] : nullptr, c[k], w[k], 0.0, ph.tc1};
      RK<double, double> rh{h0, k == 0 ? h0 : acc_h, k == 3 ? h0 : acc_h, k < 3 ? sp_h[k] : nullptr, c[k], w[k], 0.0, 0};
      fwd_stage(ui, hi, stage[0], ph, ru, rh, k == 3 ? dv("tend_u") : nullptr, k == 3 ? dv("tend_h") : nullptr);
      const Base<double> bs = base_of(stage[0], ui);
      const double *uti = k == 0 ? ut0 : tp_u[k - 1];
      const double *hti = k == 0 ? ht0 : tp_h[k - 1];
      RK<double, double> rut{ut0, k == 0 ? ut0 : tacc_u, k == 3 ? ut0 : tacc_u, k < 3 ? tp_u[k] : nullptr, c[k], w[k], 0.0, ph.tc1};
      RK<double, double> rht{ht0, k == 0 ? ht0 : tacc_h, k == 3 ? ht0 : tacc_h, k < 3 ? tp_h[k] : nullptr, c[k], w[k], 0.0, 0};
      L64::tl_vertex(m64, 1, bs, uti, hti, tl_diag, stream);
      L64::tl_cell(m64, 1, bs, uti, hti, tl_diag, rht, k == 3 ? dv("tend_h_tl") : nullptr, stream);
      L64::tl_edge_diag(m64, 1, bs, uti, hti, tl_diag, ph, stream);
      if (ph.visc4 > 0) L64::del4_vc(m64, 1, tl_diag.dsq_u, tl_diag.dsq_vort, tl_diag.dsq_div, stream);
      L64::tl_edge_tend(m64, 1, bs, uti, hti, tl_diag, ph, rut, k == 3 ? dv("tend_u_tl") : nullptr, stream);
    }
  }
  finish_levels({"u", "h", "u_tl", "h_tl"});
  L64::recon(m64, 1, ph.sphere, u0, dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  L64::recon(m64, 1, ph.sphere, ut0, dv("uReconstructX_tl"), dv("uReconstructY_tl"), dv("uReconstructZ_tl"),
             dv("uReconstructZonal_tl"), dv("uReconstructMeridional_tl"), stream);
  check_launch("sw_rk4_tlm");
  for (const char *n : {"u", "h", "tend_u", "tend_h", "u_tl", "h_tl", "tend_u_tl", "tend_h_tl"}) mark_written(var(n), true);
  mark_recon(0);
  mark_recon(1);
  mark_diag(0, true);
  mark_diag(1, true);
  pending_diag = 2;
  nonfinite_check("sw_rk4_tlm");
}

AdSeeds<double> Engine::seeds(bool *any) {
  AdSeeds<double> s{};
  *any = false;
  auto S = [&](const char *n) -> const double * {
    Var &v = var(n);
    if (!v.nonzero) return nullptr;
    *any = true;
    return v.dev;
  };
  s.v = S("v_ad"); s.he = S("h_edge_ad"); s.hv = S("h_vertex_ad"); s.pe = S("pv_edge_ad");
  s.pvv = S("pv_vertex_ad"); s.pc = S("pv_cell_ad"); s.circ = S("circulation_ad");
  s.vort = S("vorticity_ad"); s.div = S("divergence_ad"); s.ke = S("ke_ad");
  s.vc = S("vorticity_cell_ad"); s.gpn = S("gradPVn_ad"); s.gpt = S("gradPVt_ad");
  return s;
}

void Engine::zero_ad_seeds() {
  for (int i = 0; i < 19; i++) {
    Var &v = var((std::string(kDiagNames[i]) + "_ad").c_str());
    cuda_check(cudaMemsetAsync(v.dev, 0, sizeof(double) * v.count, stream), "memset");
    mark_written(v, false);
  }
  for (const char *n : {"tend_u_ad", "tend_h_ad"}) {
    Var &v = var(n);
    cuda_check(cudaMemsetAsync(v.dev, 0, sizeof(double) * v.count, stream), "memset");
    mark_written(v, false);
  }
}

bool Engine::recon_seeds_nonzero() {
  for (int i = 0; i < 5; i++)
    if (var((std::string(kDiagNames[i]) + "_ad").c_str()).nonzero) return true;
  return false;
}

void Engine::rk4_adj() {  // src/mpas_sw_module.f90:783-1002
  if (!allocated[2]) throw EngineError(MPSW_ERR_STATE, "var_allocation_adj has not been called");
  prepare();
  const Phys<double> ph = phys();
  double w[4], c[4];
  rk_coeffs(ph.dt, w, c);
  double *u0 = dv("u"), *h0 = dv("h"), *u2 = dv("u", 1), *h2 = dv("h", 1);
  // forward sweep, keeping the diagnostics of every stage (:815-878)
  for (int k = 0; k < 4; k++) {
    const double *ui = k == 0 ? u0 : sp_u[k - 1];
    const double *hi = k == 0 ? h0 : sp_h[k - 1];
    RK<double, double> ru{u0, k == 0 ? u0 : acc_u, acc_u, k < 3 ? sp_u[k] : nullptr, c[k], w[k], 0.0, ph.tc1};
    RK<double, double> rh{h0, k == 0 ? h0 : acc_h, acc_h, k < 3 ? sp_h[k] : nullptr, c[k], w[k], 0.0, 0};
    fwd_stage(ui, hi, stage[k + 1], ph, ru, rh, nullptr, nullptr);
  }
  cuda_check(cudaMemcpyAsync(u2, ph.tc1 ? u0 : acc_u, sizeof(double) * nE, cudaMemcpyDeviceToDevice, stream), "u(2)");
  cuda_check(cudaMemcpyAsync(h2, acc_h, sizeof(double) * nC, cudaMemcpyDeviceToDevice, stream), "h(2)");
  L64::recon(m64, 1, ph.sphere, u0, dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  double *ua = dv("u_ad"), *ha = dv("h_ad");
  // adjoint of the output reconstruction and diagnostics at x(2) (:887-905)
  if (recon_seeds_nonzero())
    L64::recon_adj(m64, ph.sphere, dv("uReconstructX_ad"), dv("uReconstructY_ad"), dv("uReconstructZ_ad"),
                   dv("uReconstructZonal_ad"), dv("uReconstructMeridional_ad"), ua, stream);
  bool any = false;
  AdSeeds<double> sd = seeds(&any);
  if (any) {
    fwd_diag(u2, h2, stage[0], ph);
    cuda_check(cudaMemsetAsync(tu_[0], 0, sizeof(double) * nE, stream), "memset");
    cuda_check(cudaMemsetAsync(th_[0], 0, sizeof(double) * nC, stream), "memset");
    AdIn<double> in{tu_[0], th_[0]};
    AdOut<double, double> out{};
    out.acc_u = ua; out.acc_h = ha; out.mode = AD_ADD;
    L64::ad_stage(m64, 1, base_of(stage[0], u2), ph, in, sd, adw, out, stream);
  }
  // tendency adjoint of stage 4 (:913-914), with any seed left in tend_*_ad
  const double *stu = var("tend_u_ad").nonzero ? dv("tend_u_ad") : nullptr;
  const double *sth = var("tend_h_ad").nonzero ? dv("tend_h_ad") : nullptr;
  L64::ad_tinit(m64, 1, ua, ha, ph.tc1 ? nullptr : stu, sth, ph.tc1 ? 0.0 : w[3], w[3], tu_[0], th_[0], stream);
  AdSeeds<double> none{};
  for (int k = 3; k >= 0; k--) {  // :912-970
    const double *ui = k == 0 ? u0 : sp_u[k - 1];
    AdIn<double> in{tu_[(3 - k) & 1], th_[(3 - k) & 1]};
    AdOut<double, double> out{};
    out.acc_u = xacc_u; out.acc_h = xacc_h;
    out.x2u = ua; out.x2h = ha; out.dst_u = ua; out.dst_h = ha;
    out.mode = k == 3 ? AD_SET : k == 0 ? AD_FINAL : AD_ADD;
    if (k > 0) {
      out.tu_next = tu_[(4 - k) & 1];
      out.th_next = th_[(4 - k) & 1];
      out.wu = ph.tc1 ? 0.0 : w[k - 1];
      out.cu = ph.tc1 ? 0.0 : c[k - 1];
      out.wh = w[k - 1];
      out.ch = c[k - 1];
    }
    L64::ad_stage(m64, 1, base_of(stage[k + 1], ui), ph, in, none, adw, out, stream);
  }
  cuda_check(cudaMemsetAsync(dv("u_ad", 1), 0, sizeof(double) * nE, stream), "memset");
  cuda_check(cudaMemsetAsync(dv("h_ad", 1), 0, sizeof(double) * nC, stream), "memset");
  zero_ad_seeds();
  check_launch("sw_rk4_adj");
  for (const char *n : {"u", "h", "u_ad", "h_ad"}) mark_written(var(n), true);
  mark_recon(0);
  mark_diag(0, true);
  pending_diag = 1;
  nonfinite_check("sw_rk4_adj");
}

void Engine::solve_diagnostics(int tl) {
  prepare();
  pending_diag = 0;
  const Phys<double> ph = phys();
  Diag<double> d = module_diag(0);
  fwd_diag(dv("u"), dv("h"), d, ph);
  if (tl) {
    if (!allocated[1]) throw EngineError(MPSW_ERR_STATE, "var_allocation_tlm has not been called");
    tl_diag_run(base_of(d, dv("u")), dv("u_tl"), dv("h_tl"), module_diag(1), ph);
  }
  check_launch("solve_diagnostics");
  mark_diag(0, false);
  if (tl) mark_diag(1, false);
}

void Engine::compute_tend(int tl) {
  // the tendencies use the diagnostics of the current level-1 state, recomputed here
  solve_diagnostics(tl);
  const Phys<double> ph = phys();
  Diag<double> d = module_diag(0);
  RK<double, double> none{};
  L64::tend_h(m64, dv("u"), d.he, dv("tend_h"), stream);
  L64::fwd_edge_tend(m64, dv("u"), dv("h"), 0.0, d, ph, none, dv("tend_u"), stream);
  if (tl) {
    Diag<double> dt = module_diag(1);
    const Base<double> bs = base_of(d, dv("u"));
    L64::tl_cell(m64, 1, bs, dv("u_tl"), dv("h_tl"), dt, none, dv("tend_h_tl"), stream);
    L64::tl_edge_tend(m64, 1, bs, dv("u_tl"), dv("h_tl"), dt, ph, none, dv("tend_u_tl"), stream);
  }
  check_launch("compute_tend");
  mark_written(var("tend_u"), true);
  mark_written(var("tend_h"), true);
  if (tl) {
    mark_written(var("tend_u_tl"), true);
    mark_written(var("tend_h_tl"), true);
  }
  nonfinite_check("compute_tend");
}

void Engine::reconstruct(int tl) {
  prepare();
  const Phys<double> ph = phys();
  L64::recon(m64, 1, ph.sphere, dv("u"), dv("uReconstructX"), dv("uReconstructY"), dv("uReconstructZ"),
             dv("uReconstructZonal"), dv("uReconstructMeridional"), stream);
  if (tl)
    L64::recon(m64, 1, ph.sphere, dv("u_tl"), dv("uReconstructX_tl"), dv("uReconstructY_tl"),
               dv("uReconstructZ_tl"), dv("uReconstructZonal_tl"), dv("uReconstructMeridional_tl"), stream);
  check_launch("reconstruct");
  mark_recon(0);
  if (tl) mark_recon(1);
}

void Engine::adjoint_at_state() {  // src/mpas_sw_module.f90:1163-1206
  if (!allocated[2]) throw EngineError(MPSW_ERR_STATE, "var_allocation_adj has not been called");
  prepare();
  const Phys<double> ph = phys();
  double *u0 = dv("u"), *h0 = dv("h"), *ua = dv("u_ad"), *ha = dv("h_ad");
  fwd_diag(u0, h0, stage[0], ph);
  if (recon_seeds_nonzero())
    L64::recon_adj(m64, ph.sphere, dv("uReconstructX_ad"), dv("uReconstructY_ad"), dv("uReconstructZ_ad"),
                   dv("uReconstructZonal_ad"), dv("uReconstructMeridional_ad"), ua, stream);
  bool any = false;
  AdSeeds<double> sd = seeds(&any);
  const double *stu = var("tend_u_ad").nonzero && !ph.tc1 ? dv("tend_u_ad") : nullptr;
  const double *sth = var("tend_h_ad").nonzero ? dv("tend_h_ad") : nullptr;
  L64::ad_tinit(m64, 1, nullptr, nullptr, stu, sth, 0.0, 0.0, tu_[0], th_[0], stream);
  AdIn<double> in{tu_[0], th_[0]};
  AdOut<double, double> out{};
  out.acc_u = ua; out.acc_h = ha; out.mode = AD_ADD;
  L64::ad_stage(m64, 1, base_of(stage[0], u0), ph, in, sd, adw, out, stream);
  zero_ad_seeds();
  check_launch("adjoint_at_state");
  mark_written(var("u_ad"), true);
  mark_written(var("h_ad"), true);
  mark_recon(2);
}

}  // namespace mpsw

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
namespace {
thread_local std::string g_create_error;
}  // namespace

extern "C" {

int mpsw_create(mpsw_handle **out) {
  if (!out) return MPSW_ERR_ARG;
  *out = nullptr;
  try {
    *out = new mpsw_handle();
    return MPSW_OK;
  } catch (const mpsw::EngineError &e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return MPSW_ERR_CUDA;
  }
}

void mpsw_destroy(mpsw_handle *h) { delete h; }

const char *mpsw_last_error(const mpsw_handle *h) { return h ? h->eng.err.c_str() : g_create_error.c_str(); }

const char *mpsw_version(void) { return "mpsw-b200 0.1"; }

int mpsw_set_scalar(mpsw_handle *h, const char *name, double value) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    const std::string n = mpsw::lower(name);
    for (const auto &s : kScalars)
      if (n == s.name && s.readonly) throw mpsw::EngineError(MPSW_ERR_ARG, "cannot assign a parameter: " + n);
    if (n == "on_a_sphere" || n == "config_h_scalewithmesh") e.mesh_dirty = true;
    e.scal[n] = value;
    e.refresh_phys();
  });
}

int mpsw_get_scalar(mpsw_handle *h, const char *name, double *value) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!value) throw mpsw::EngineError(MPSW_ERR_ARG, "null output");
    auto it = e.scal.find(mpsw::lower(name));
    if (it == e.scal.end()) throw mpsw::EngineError(MPSW_ERR_ARG, std::string("unknown scalar ") + (name ? name : ""));
    *value = it->second;
  });
}

int mpsw_var_count(void) { return (int)specs().size(); }

const char *mpsw_var_name(int index) {
  if (index < 0 || index >= (int)specs().size()) return nullptr;
  return specs()[index].name;
}

int mpsw_var_info(mpsw_handle *h, const char *name, int *rank, long long dims[4], int *is_int, int *allocated) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    mpsw::Var &v = e.var(name);
    if (rank) *rank = (int)v.dims.size();
    if (dims)
      for (int i = 0; i < 4; i++) dims[i] = i < (int)v.dims.size() ? v.dims[i] : 0;
    if (is_int) *is_int = v.is_int;
    if (allocated) *allocated = v.allocated;
  });
}

int mpsw_set_var(mpsw_handle *h, const char *name, const void *src, long long count) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.set_var(name, src, count); });
}

int mpsw_get_var(mpsw_handle *h, const char *name, void *dst, long long count) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.get_var(name, dst, count); });
}

int mpsw_var_allocation(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.allocate_group(0); }); }
int mpsw_var_allocation_tlm(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.allocate_group(1); }); }
int mpsw_var_allocation_adj(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.allocate_group(2); }); }
int mpsw_sw_mpas_init_block(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.init_block(); }); }

int mpsw_get_stream(mpsw_handle *h, void **stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (!stream) throw mpsw::EngineError(MPSW_ERR_ARG, "null stream pointer");
    e.need_device();
    *stream = (void *)e.stream;
  });
}
int mpsw_forward(mpsw_handle *h, int precision, int nsteps) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.forward(precision, nsteps); });
}
int mpsw_sw_rk4(mpsw_handle *h, int nsteps) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (nsteps < 0) throw mpsw::EngineError(MPSW_ERR_ARG, "nsteps < 0");
    e.rk4(nsteps);
  });
}
int mpsw_sw_rk4_tlm(mpsw_handle *h, int nsteps) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    if (nsteps < 0) throw mpsw::EngineError(MPSW_ERR_ARG, "nsteps < 0");
    e.rk4_tlm(nsteps);
  });
}
int mpsw_sw_rk4_adj(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.rk4_adj(); }); }
int mpsw_solve_diagnostics(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.solve_diagnostics(0); }); }
int mpsw_compute_tend(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.compute_tend(0); }); }
int mpsw_reconstruct_2d(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.reconstruct(0); }); }
int mpsw_solve_diagnostics_tlm(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.solve_diagnostics(1); }); }
int mpsw_compute_tend_tlm(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.compute_tend(1); }); }
int mpsw_reconstruct_2d_tlm(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.reconstruct(1); }); }
int mpsw_adjoint_at_state(mpsw_handle *h) { return mpsw::guarded(h, [&](mpsw::Engine &e) { e.adjoint_at_state(); }); }

}  // extern "C"
