// FP64 instantiation of the stencil launchers.  Built with --fmad=false so every multiply and
// add rounds separately, as in the reference's FP64 Fortran.
#include "mpsw_launch.cuh"

namespace mpsw {

long long g_launches = 0;
thread_local const TuneTable *g_tune = nullptr;
thread_local bool g_stable_base = false;

void convert_d2f(long long n, const double *src, float *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_convert<double, float>, launch_cfg(n), s, n, src, dst);
}
void convert_f2d(long long n, const float *src, double *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_convert<float, double>, launch_cfg(n), s, n, src, dst);
}

void convert_d2f_off(long long n, const double *src, double off, float *dst, cudaStream_t s) {
  g_launches++;
  launch_k(k_convert_off, launch_cfg(n), s, n, src, off, dst);
}

void convert_list(const ConvList &L, long long max_n, cudaStream_t s) {
  g_launches++;
  launch_k(k_convert_list, launch_cfg(max_n), s, L);
}

template struct Launch<double, double>;

}  // namespace mpsw
