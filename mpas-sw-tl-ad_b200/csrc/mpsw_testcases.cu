// Williamson et al. (1992, J. Comput. Phys. 102) shallow-water test cases 1, 2, 5 and 6 on the
// GPU, as the reference module's sw_test_case_* subroutines set them up
// (src/mpas_sw_testcases.f90:1-398): the mesh is scaled by the Earth radius on the host, then
// one thread per vertex forms the stream function, one per edge the normal velocity
// u = -(psi(v2) - psi(v1)) / dvEdge and fEdge, one per vertex fVertex, and one per cell h, the
// mountain h_s and the tracers.  FP64 throughout, no contraction (--fmad=false).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mpsw.h"
#include "mpsw_engine.h"
#include "mpsw_launch.h"

namespace mpsw {
namespace {

constexpr double kPii = 3.141592653589793;

struct TcArgs {
  int tc, nC, nE, nV, nT;
  double a, omega, g;
  const double *latC, *lonC, *latE, *lonE, *latV, *lonV, *dvE;
  const int *voe;  // verticesOnEdge (2, nE), 1-based, column-major
  double *psi, *u, *fE, *fV, *h, *hs, *tr0, *tr1, *lonC_out;
};

// case constants (src/mpas_sw_testcases.f90:30-38, 68-80, 146-160, 262-275)
__device__ __forceinline__ double tc_u0(int tc, double a) {
  return tc == 5 ? 20. : 2.0 * kPii * a / (12.0 * 86400.0);
}
__device__ __forceinline__ double tc_alpha(int tc) { return tc == 1 ? kPii / 4.0 : 0.0; }

__global__ void k_tc_vertex(TcArgs t) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= t.nV) return;
  const double lat = t.latV[v], lon = t.lonV[v];
  double psi;
  if (t.tc == 6) {  // Rossby-Haurwitz stream function (:290-299)
    const double w = 7.848e-6, K = 7.848e-6, R = 4.0;
    psi = -t.a * t.a * w * sin(lat) + t.a * t.a * K * pow(cos(lat), R) * sin(lat) * cos(R * lon);
  } else {  // solid-body rotation about an axis tilted by alpha (:86-90, :163-167, :186-190)
    const double u0 = tc_u0(t.tc, t.a), alpha = tc_alpha(t.tc);
    psi = -t.a * u0 * (sin(lat) * cos(alpha) - cos(lon) * cos(lat) * sin(alpha));
  }
  t.psi[v] = psi;
  if (t.fV) {
    const double alpha = tc_alpha(t.tc);
    t.fV[v] = 2.0 * t.omega * (-cos(lon) * cos(lat) * sin(alpha) + sin(lat) * cos(alpha));
  }
}

__global__ void k_tc_edge(TcArgs t) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= t.nE) return;
  const int v1 = t.voe[2 * (size_t)e] - 1, v2 = t.voe[2 * (size_t)e + 1] - 1;
  t.u[e] = -1.0 * (t.psi[v2] - t.psi[v1]) / t.dvE[e];
  if (t.fE) {
    const double alpha = tc_alpha(t.tc), lat = t.latE[e], lon = t.lonE[e];
    t.fE[e] = 2.0 * t.omega * (-cos(lon) * cos(lat) * sin(alpha) + sin(lat) * cos(alpha));
  }
}

__global__ void k_tc_cell(TcArgs t) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= t.nC) return;
  const double lat = t.latC[c];
  double lon = t.lonC[c];
  if (t.tc == 1) {  // cosine bell (:96-110)
    const double h0 = 1000.0, theta_c = 0.0, lambda_c = 3.0 * kPii / 2.0;
    const double arg = sqrt(pow(sin(0.5 * (lat - theta_c)), 2.0) +
                            cos(theta_c) * cos(lat) * pow(sin(0.5 * (lon - lambda_c)), 2.0));
    const double r = 2. * t.a * asin(arg);
    t.h[c] = r < t.a / 3.0 ? (h0 / 2.0) * (1.0 + cos(kPii * r * 3.0 / t.a)) : h0 / 2.0;
    return;
  }
  if (t.tc == 6) {  // Rossby-Haurwitz height (:303-318)
    const double h0 = 8000.0, w = 7.848e-6, K = 7.848e-6, R = 4.0, om = t.omega;
    const double cl = cos(lat);
    const double aa = 0.5 * w * (2.0 * om + w) * pow(cl, 2.0) +
                      0.25 * K * K * pow(cl, 2.0 * R) *
                          ((R + 1.0) * pow(cl, 2.0) + 2.0 * R * R - R - 2.0 - 2.0 * R * R * pow(cl, -2.0));
    const double bb = (2.0 * (om + w) * K / ((R + 1.0) * (R + 2.0))) * pow(cl, R) *
                      ((R * R + 2.0 * R + 2.0) - pow((R + 1.0) * cl, 2.0));
    const double cc = 0.25 * K * K * pow(cl, 2.0 * R) * ((R + 1.0) * pow(cl, 2.0) - R - 2.0);
    t.h[c] = (t.g * h0 + t.a * t.a * aa + t.a * t.a * bb * cos(R * lon) + t.a * t.a * cc * cos(2.0 * R * lon)) / t.g;
    return;
  }
  // cases 2 and 5: geostrophic balance with the rotated solid-body flow (:171-175, :247-252)
  const double u0 = tc_u0(t.tc, t.a), alpha = tc_alpha(t.tc);
  const double gh0 = t.tc == 5 ? 5960.0 * t.g : 29400.0;
  double hs = 0.0;
  if (t.tc == 5) {  // isolated mountain and tracers (:220-245); lonCell is shifted in place first
    const double hs0 = 2000., theta_c = kPii / 6.0, lambda_c = 3.0 * kPii / 2.0, rr = kPii / 9.0;
    if (lon < 0.0) lon = lon + 2.0 * kPii;
    t.lonC_out[c] = lon;
    const double r = sqrt(fmin(pow(rr, 2.0), pow(lon - lambda_c, 2.0) + pow(lat - theta_c, 2.0)));
    hs = hs0 * (1.0 - r / rr);
    t.hs[c] = hs;
    if (t.tr0) t.tr0[c] = 1.0 - r / rr;
    if (t.tr1) {
      const double r2 = sqrt(fmin(pow(rr, 2.0), pow(lon - lambda_c, 2.0) + pow(lat - theta_c - kPii / 6.0, 2.0)));
      t.tr1[c] = 1.0 - r2 / rr;
    }
  }
  const double x = -cos(lon) * cos(lat) * sin(alpha) + sin(lat) * cos(alpha);
  double h = (gh0 - (t.a * t.omega * u0 + 0.5 * pow(u0, 2.0)) * pow(x, 2.0)) / t.g;
  if (t.tc == 5) h = h - hs;
  t.h[c] = h;
}

}  // namespace

// src/mpas_sw_testcases.f90: sw_test_case_1/2/5/6 on the module's variables.
void Engine::test_case(int tc) {
  if (!allocated[0]) throw EngineError(MPSW_ERR_STATE, "var_allocation has not been called");
  if (tc != 1 && tc != 2 && tc != 5 && tc != 6) throw EngineError(MPSW_ERR_ARG, "test case must be 1, 2, 5 or 6");
  need_device();
  const double a = sc("a");
  // the unit-sphere mesh scaled by the Earth radius (:173-186 and the same lines of each case)
  for (const char *n : {"xCell", "yCell", "zCell", "xVertex", "yVertex", "zVertex", "xEdge", "yEdge", "zEdge",
                        "dvEdge", "dcEdge"})
    for (double &x : var(n).hr) x = x * a;
  for (const char *n : {"areaCell", "areaTriangle", "kiteAreasOnVertex"})
    for (double &x : var(n).hr) x = x * pow(a, 2.0);
  mesh_dirty = true;
  // device temporaries: inputs, then outputs
  std::vector<void *> tmp;
  auto up = [&](const std::vector<double> &h) {
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, sizeof(double) * (h.empty() ? 1 : h.size())), "cudaMalloc test case");
    tmp.push_back(p);
    if (!h.empty()) cuda_check(cudaMemcpy(p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice), "upload");
    return (double *)p;
  };
  auto out = [&](size_t n) {
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, sizeof(double) * (n ? n : 1)), "cudaMalloc test case");
    tmp.push_back(p);
    return (double *)p;
  };
  TcArgs t{};
  t.tc = tc; t.nC = nC; t.nE = nE; t.nV = nV; t.nT = nT;
  t.a = a; t.omega = sc("omega"); t.g = sc("gravity");
  try {
    t.latC = up(var("latCell").hr); t.lonC = up(var("lonCell").hr);
    t.latE = up(var("latEdge").hr); t.lonE = up(var("lonEdge").hr);
    t.latV = up(var("latVertex").hr); t.lonV = up(var("lonVertex").hr);
    t.dvE = up(var("dvEdge").hr);
    {
      void *p = nullptr;
      const std::vector<int> &voe = var("verticesOnEdge").hi;
      cuda_check(cudaMalloc(&p, sizeof(int) * voe.size()), "cudaMalloc test case");
      tmp.push_back(p);
      cuda_check(cudaMemcpy(p, voe.data(), sizeof(int) * voe.size(), cudaMemcpyHostToDevice), "upload");
      t.voe = (const int *)p;
    }
    const bool cor = tc == 2 || tc == 5;  // cases 1 and 6 leave the Coriolis parameters as they are
    t.psi = out(nV); t.u = out(nE); t.h = out(nC);
    t.fE = cor ? out(nE) : nullptr;
    t.fV = cor ? out(nV) : nullptr;
    const bool trac = tc == 5 && var("tracers").allocated && nT >= 1;
    if (tc == 5) {
      t.hs = out(nC);
      t.lonC_out = out(nC);
      t.tr0 = trac ? out(nC) : nullptr;
      t.tr1 = trac && nT > 1 ? out(nC) : nullptr;
    }
    const int bt = 256;
    g_launches += 3;
    k_tc_vertex<<<(nV + bt - 1) / bt, bt, 0, stream>>>(t);
    k_tc_edge<<<(nE + bt - 1) / bt, bt, 0, stream>>>(t);
    k_tc_cell<<<(nC + bt - 1) / bt, bt, 0, stream>>>(t);
    cuda_check(cudaGetLastError(), "test case kernels");
    auto down = [&](const double *src, size_t n) {
      std::vector<double> h(n);
      cuda_check(cudaMemcpyAsync(h.data(), src, sizeof(double) * n, cudaMemcpyDeviceToHost, stream), "download");
      cuda_check(cudaStreamSynchronize(stream), "test case");
      return h;
    };
    auto set_level1 = [&](const char *name, const std::vector<double> &x, size_t stride, size_t first) {
      Var &v = var(name);
      if (v.ent && !v.host_valid) download(v);  // keep the other levels as they are
      for (size_t i = 0; i < x.size(); i++) v.hr[first + stride * i] = x[i];
      v.host_valid = true;
      if (v.ent) v.dev_valid = false;
      v.nonzero = true;
    };
    set_level1("u", down(t.u, nE), 2, 0);   // u(1,1,:), u is (2, 1, nEdges)
    set_level1("h", down(t.h, nC), 2, 0);   // h(1,1,:)
    if (cor) {
      var("fEdge").hr = down(t.fE, nE);
      var("fVertex").hr = down(t.fV, nV);
    }
    if (tc == 5) {
      var("h_s").hr = down(t.hs, nC);
      var("lonCell").hr = down(t.lonC_out, nC);
      if (trac) {  // tracers(1, 1..2, 1, :), tracers is (2, nTracers, 1, nCells)
        set_level1("tracers", down(t.tr0, nC), 2 * (size_t)nT, 0);
        if (t.tr1) set_level1("tracers", down(t.tr1, nC), 2 * (size_t)nT, 2);
      }
    }
  } catch (...) {
    for (void *p : tmp) cudaFree(p);
    throw;
  }
  for (void *p : tmp) cudaFree(p);
}

}  // namespace mpsw

extern "C" int mpsw_sw_test_case(mpsw_handle *h, int tc) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) { e.test_case(tc); });
}
