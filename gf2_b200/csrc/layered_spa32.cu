// gf2cuda layered-schedule kernels: sum-product with the exact numerics (GF2C_ALGO_SPA), FP32 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_spa32_kernel(int dcmax, int maxt, bool stage, int bps) { return lay_t<L_SPA, 0>(dcmax, maxt, stage, bps); }

}  // namespace gf2c
