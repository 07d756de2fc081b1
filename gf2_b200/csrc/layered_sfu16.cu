// gf2cuda layered-schedule kernels: sum-product on the SFU (GF2C_ALGO_SPA_FAST), FP16 messages.
#include "layered_impl.cuh"

namespace gf2c {

const void* layered_sfu16_kernel(int dcmax, int maxt, bool stage) { return lay_t<L_SPA_FAST, 1>(dcmax, maxt, stage); }

}  // namespace gf2c
