// gf2cuda layered-schedule kernels: sum-product on the SFU (GF2C_ALGO_SPA_FAST), FP16 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_sfu16_kernel(int dcmax, int maxt, bool stage, int bps) { return lay_t<L_SPA_FAST, 1>(dcmax, maxt, stage, bps); }

}  // namespace gf2c
