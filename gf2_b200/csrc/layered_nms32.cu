// gf2cuda layered-schedule kernels: normalised / offset min-sum (GF2C_ALGO_NMS, and GF2C_ALGO_MINSUM as alpha 1, beta 0), FP32 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_nms32_kernel(int dcmax, int maxt, bool stage, int bps) { return lay_t<L_NMS, 0>(dcmax, maxt, stage, bps); }

}  // namespace gf2c
