// gf2cuda layered-schedule decoder (sm_100a): host-side kernel selection.
// The device code is in layered_impl.cuh; the kernels are instantiated in
// layered_{sfu,nms,spa}{16,32}.cu (one translation unit per check-node rule
// and message type, so that they compile in parallel).
#include "internal.h"

namespace gf2c {

enum { L_MS = 0, L_SPA = 1, L_NMS = 2, L_SPA_FAST = 3 };

const void* layered_sfu16_kernel(int dcmax, int maxt, bool stage, int bps);
const void* layered_sfu32_kernel(int dcmax, int maxt, bool stage, int bps);
const void* layered_nms16_kernel(int dcmax, int maxt, bool stage, int bps);
const void* layered_nms32_kernel(int dcmax, int maxt, bool stage, int bps);
const void* layered_spa16_kernel(int dcmax, int maxt, bool stage, int bps);
const void* layered_spa32_kernel(int dcmax, int maxt, bool stage, int bps);

int layered_dcmax_bucket(int max_dc) {
  static const int buckets[] = {7, 9, 10, 11, 13, 14, 18, 19, 22, 26, 32};
  for (int b : buckets)
    if (max_dc <= b) return b;
  return -1;
}

// Layered min-sum runs on the normalised / offset min-sum kernels with
// alpha = 1, beta = 0 (the decoder supplies those weights): 1 * max(m - 0, 0)
// is m exactly, so the messages are bit-identical to plain min-sum.
const void* layered_kernel_ptr(int algo, int msg16, int dcmax, int maxt, bool stage, int bps) {
  switch (algo) {
    case L_MS:
    case L_NMS:
      return msg16 ? layered_nms16_kernel(dcmax, maxt, stage, bps) : layered_nms32_kernel(dcmax, maxt, stage, bps);
    case L_SPA:
      return msg16 ? layered_spa16_kernel(dcmax, maxt, stage, bps) : layered_spa32_kernel(dcmax, maxt, stage, bps);
    case L_SPA_FAST:
      return msg16 ? layered_sfu16_kernel(dcmax, maxt, stage, bps) : layered_sfu32_kernel(dcmax, maxt, stage, bps);
  }
  return nullptr;
}

size_t layered_smem_bytes(int smem_app_floats, int bitmap_words) {
  return (size_t)((bitmap_words * 4 + 15) & ~15) + (size_t)smem_app_floats * 4;
}

}  // namespace gf2c
