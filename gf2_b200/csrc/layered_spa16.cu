// gf2cuda layered-schedule kernels: sum-product with the exact numerics (GF2C_ALGO_SPA), FP16 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_spa16_kernel(int dcmax, int maxt, bool stage) { return lay_t<L_SPA, 1>(dcmax, maxt, stage); }

}  // namespace gf2c
