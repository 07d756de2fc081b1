// gf2cuda layered-schedule kernels: sum-product on the SFU (GF2C_ALGO_SPA_FAST), FP32 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_sfu32_kernel(int dcmax, int maxt, bool stage, int bps) { return lay_t<L_SPA_FAST, 0>(dcmax, maxt, stage, bps); }

}  // namespace gf2c
