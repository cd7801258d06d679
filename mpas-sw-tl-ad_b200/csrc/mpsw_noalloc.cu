// Tendencies of a caller-supplied state with no device allocation (mpsw_compute_tend_noalloc).
//
// Some callers cannot allocate device memory at the moment they need the model: a data
// assimilation or coupling system that reserves all GPU memory for its own pool at start-up
// and forbids later cudaMalloc/cudaFree, code that must not synchronise the device (a
// cudaFree does), or a host that runs under a strict memory budget.  This entry point serves
// them: it computes the same tend_u / tend_h as mpsw_compute_tend (the reference's
// sw_solve_diagnostics + sw_compute_tend) for state buffers the caller owns, keeping the
// intermediate diagnostics in a fixed array that lives in the library's own device image
// instead of in allocated memory.
//
// The array below is file-scope device memory: every GPU that loads the library holds its
// kNoAllocScratchDoubles doubles (16 MiB) until the process exits.  Its name is only a
// host-side stand-in in host code, so the device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and passed to the kernels.  With lazy module
// loading (the CUDA default) that lookup is what loads the array onto the device, so the engine
// does it while it builds its mesh on a device (noalloc_prepare_device, called from
// sw_mpas_init_block), together with loading the kernels the entry point launches: the
// entry point itself then neither allocates nor loads anything.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "mpsw.h"
#include "mpsw_engine.h"
#include "mpsw_launch.h"

namespace mpsw {
namespace {

constexpr size_t kNoAllocScratchDoubles = (size_t)2 << 20;  // 16 MiB
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::atomic<double *> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mutex;

// Device address of the scratch array on the current device (looked up on first use).
double *scratch_on_current_device() {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw EngineError(MPSW_ERR_UNSUPPORTED, "device index out of range");
  double *p = g_scratch_addr[dev].load();
  if (p) return p;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  p = g_scratch_addr[dev].load();
  if (!p) {
    cuda_check(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    g_scratch_addr[dev].store(p);
  }
  return p;
}

}  // namespace

void noalloc_prepare_device() {
  (void)scratch_on_current_device();
  cuda_check(Launch<double, double>::preload_forward(), "loading the stage kernels");
}

}  // namespace mpsw

extern "C" int mpsw_compute_tend_noalloc(mpsw_handle *h, const double *u, const double *hh, double *tend_u,
                                         double *tend_h, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    using namespace mpsw;
    if (!u || !hh || !tend_u || !tend_h) throw EngineError(MPSW_ERR_ARG, "null state or tendency buffer");
    if (!e.mesh_built || e.mesh_dirty)
      throw EngineError(MPSW_ERR_STATE, "mesh not on the device: call sw_mpas_init_block first (this entry point does not build it)");
    int dev = -1;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != e.mesh_device)
      throw EngineError(MPSW_ERR_STATE, "current device " + std::to_string(dev) + " is not the device " +
                                            std::to_string(e.mesh_device) + " that holds this handle's mesh");
    const Phys<double> ph = e.phys();
    const size_t nC = (size_t)e.nC, nE = (size_t)e.nE, nV = (size_t)e.nV;
    // diagnostics kept: vorticity, h_vertex, pv_vertex; divergence, ke, pv_cell; pv_edge, h_edge;
    // and, with del4 viscosity, delsq_u, delsq_vorticity, delsq_divergence
    const size_t need = 3 * nV + 3 * nC + 2 * nE + (ph.visc4 > 0 ? nE + nV + nC : 0);
    if (need > kNoAllocScratchDoubles)
      throw EngineError(MPSW_ERR_UNSUPPORTED,
                        "mesh too large for the fixed scratch of mpsw_compute_tend_noalloc: needs " +
                            std::to_string(need) + " doubles, maximum " + std::to_string(kNoAllocScratchDoubles));
    double *p = scratch_on_current_device();
    Diag<double> d{};
    d.vort = p; p += nV;
    d.hv = p; p += nV;
    d.pvv = p; p += nV;
    d.div = p; p += nC;
    d.ke = p; p += nC;
    d.pc = p; p += nC;
    d.pe = p; p += nE;
    d.he = p; p += nE;
    if (ph.visc4 > 0) {
      d.dsq_u = p; p += nE;
      d.dsq_vort = p; p += nV;
      d.dsq_div = p; p += nC;
    }
    // every scratch element is written by an earlier kernel of this call before it is read,
    // so nothing left by a previous call needs clearing
    cudaStream_t s = (cudaStream_t)stream;
    using L = Launch<double, double>;
    const RK<double, double> none{};
    L::fwd_vertex(e.m64, u, hh, 0.0, d, s);
    L::fwd_cell(e.m64, e.d_cnb, u, hh, 0.0, d, none, tend_h, s);
    L::fwd_edge_diag(e.m64, u, hh, 0.0, d, ph, s);
    if (ph.visc4 > 0) L::del4_vc(e.m64, 1, d.dsq_u, d.dsq_vort, d.dsq_div, s);
    L::fwd_edge_tend(e.m64, u, hh, 0.0, d, ph, none, tend_u, s);
    cuda_check(cudaGetLastError(), "mpsw_compute_tend_noalloc");
  });
}
