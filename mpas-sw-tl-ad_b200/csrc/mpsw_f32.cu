// FP32-stencil / FP64-accumulation instantiation of the stencil launchers (contraction allowed).
#include "mpsw_launch.cuh"

namespace mpsw {

template struct Launch<float, double>;

}  // namespace mpsw
