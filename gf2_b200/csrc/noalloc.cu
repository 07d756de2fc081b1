// gf2cuda: decoding without any device allocation.
//
// gf2c_decode_batch_noalloc is for callers that cannot call cudaMalloc: code
// running while a stream is being captured into a CUDA graph (allocation is
// not a stream operation and is refused there), processes whose device memory
// is owned by a pool or budget that the library must not grow, and real-time
// paths that forbid the allocator.  It runs the reference min-sum flooding
// decoder with the kernel gf2c_decode_batch uses for the default options (the
// check-state kernel, bit-identical results; codes it does not cover use the
// generic flooding kernel) with all of its device scratch -- the code's
// tables, the frame queue counter and the per-CTA workspace -- carved out of
// one file-scope static device array of kScratchBytes (64 MiB), which every
// GPU that loads the library holds until the process exits.
//
// The array's name is only a host-side stand-in in host code, so its device
// address is obtained once per device with cudaGetSymbolAddress (with that
// device current) during the first call on the device; that first call also
// sets the kernels' shared-memory attributes and should come before any
// stream capture.  Every call shares the array and it keeps the last call's
// contents: the tables of the last code stay resident and are re-copied only
// when a different code is decoded, and the queue counter is cleared on every
// call.  Calls that overlap on the GPU (other streams, other host threads) race
// on the array and must be serialised by the caller.
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "internal.h"

namespace gf2c {

static constexpr size_t kScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct DeviceScratch {
  bool ready = false;
  unsigned char* base = nullptr;       // device address of g_noalloc_scratch
  const HostCode* resident = nullptr;  // code whose tables are in the array
  uint64_t resident_serial = 0;
  DevCode dev{};                       // tables' device view (pointers into the array)
  size_t tables_end = 0;
  int sms = 0;
  // launch configuration of the last kernel / dynamic shared memory set up
  const void* kern = nullptr;
  size_t kern_smem = 0;
  int kern_occ = 0;
};

std::mutex g_mu;
DeviceScratch g_dev[64];

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

}  // namespace gf2c

using namespace gf2c;

extern "C" int gf2c_decode_batch_noalloc(const gf2c_code* code, const float* llr, int64_t frames,
                                         int32_t max_iter, uint64_t* msg_bits, int32_t* iterations,
                                         uint8_t* converged, uint8_t* syndrome_ok, void* stream) {
  if (!code || frames < 0 || max_iter < 0 || (frames > 0 && !llr))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (frames == 0) return GF2C_OK;
  const HostCode& h = *code->h;
  int dev = 0;
  GF2C_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(GF2C_ERR_UNSUPPORTED, "device index above 63");
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceScratch& S = g_dev[dev];
  if (!S.ready) {  // once per device: the device address of the static array
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    S.base = (unsigned char*)p;
    S.ready = true;
  }

  // layout: [control 256 B][DevCode][tables...][per-CTA workspace...]
  const size_t off_code = 256;
  size_t off = align256(off_code + sizeof(DevCode));
  struct Part {
    const void* src;
    size_t bytes;
    size_t off;
  };
  // the generic flooding kernel's tables, then the check-state kernel's
  Part parts[14] = {{h.cg.data(), h.cg.size() * sizeof(int4), 0},
                    {h.chk_cg.data(), h.chk_cg.size() * sizeof(uint16_t), 0},
                    {h.slot_var.data(), h.slot_var.size() * sizeof(int), 0},
                    {h.slot_desc.data(), h.slot_desc.size() * sizeof(uint32_t), 0},
                    {h.vg.data(), h.vg.size() * sizeof(int2), 0},
                    {h.vg_slot.data(), h.vg_slot.size() * sizeof(int), 0},
                    {h.sp_cg.data(), h.sp_cg.size() * sizeof(int4), 0},
                    {h.sp_desc.data(), h.sp_desc.size() * sizeof(int2), 0},
                    {h.sp_absent.data(), h.sp_absent.size() * sizeof(uint32_t), 0},
                    {h.sp_cchunk.data(), h.sp_cchunk.size() * sizeof(int2), 0},
                    {h.sp_vg.data(), h.sp_vg.size() * sizeof(int2), 0},
                    {h.sp_ci.data(), h.sp_ci.size() * sizeof(int), 0},
                    {h.sp_vchunk.data(), h.sp_vchunk.size() * sizeof(int2), 0},
                    {h.sp_u2v.data(), h.sp_u2v.size() * sizeof(int), 0}};
  for (auto& pt : parts) {
    pt.off = off;
    off = align256(off + pt.bytes);
  }
  const size_t tables_end = off;

  // kernel and per-CTA workspace: the check-state kernel where it covers the
  // code (frame state on chip when it fits, else in the workspace), else the
  // generic flooding kernel with FP32 messages
  const int sf_dc = state_dcmax_bucket(h.max_dc);
  const bool state = sf_dc > 0 && !std::getenv("GF2C_NO_STATE_FLOOD");
  const int bitmap_words = (int)((h.n + 31) / 32);
  const size_t kSmemBudget = 200 * 1024;
  const void* kern = nullptr;
  int threads = 512, smem_app = 0;
  size_t smem = 0, work_stride = 0, c2v_bytes = 0, st_bytes = 0, sf_llr_off = 0, sf_st_off = 0, sf_app_off = 0;
  if (state) {
    st_bytes = (size_t)h.m * 16;
    const size_t app_bytes = (size_t)h.n * 4;
    const bool all_smem = st_bytes + app_bytes <= 224 * 1024;
    size_t o = 0;
    sf_llr_off = o;
    o += h.sp_u2v.empty() ? 0 : align256(app_bytes);
    sf_st_off = o;
    o += all_smem ? 0 : align256(st_bytes);
    sf_app_off = o;
    o += all_smem ? 0 : align256(app_bytes);
    work_stride = o;
    smem = all_smem ? st_bytes + app_bytes : 0;
    kern = state_flood_kernel_ptr(sf_dc, all_smem);
    threads = state_flood_threads();
  } else {
    const int dcmax = decode_dcmax_bucket(h.max_dc);
    if (dcmax < 0) return set_error(GF2C_ERR_UNSUPPORTED, "check degree above 64");
    smem_app = (decode_smem_bytes((int)h.n, bitmap_words) <= kSmemBudget) ? (int)h.n : 0;
    smem = decode_smem_bytes(smem_app, bitmap_words);
    c2v_bytes = align256((size_t)h.e_slots * sizeof(float));
    work_stride = c2v_bytes + (smem_app ? 0 : align256((size_t)h.n * sizeof(float)));
    kern = flood_kernel_ptr(GF2C_ALGO_MINSUM, 0, dcmax);
  }
  if (!kern) return set_error(GF2C_ERR_UNSUPPORTED, "no decode kernel for this code");
  if (tables_end + work_stride > kScratchBytes)
    return set_error(GF2C_ERR_UNSUPPORTED,
                     "code too large for the 64 MiB static scratch of gf2c_decode_batch_noalloc (needs " +
                         std::to_string((tables_end + work_stride) >> 20) + " MiB); use gf2c_decode_batch");

  // tables of this code (copied only when the resident code changes)
  if (S.resident != &h || S.resident_serial != h.serial) {
    DevCode d{};
    d.n = (int)h.n;
    d.m = (int)h.m;
    d.k = (int)h.k;
    d.ncg = (int)h.cg.size();
    d.nvg = (int)h.vg.size();
    d.vgs = h.vgs;
    d.e_slots = h.e_slots;
    d.max_dc = h.max_dc;
    d.max_dv = h.max_dv;
    d.words_k = (int)((h.k + 63) / 64);
    d.words_n = (int)((h.n + 63) / 64);
    d.words_m = (int)((h.m + 63) / 64);
    d.layered_ok = h.layered_ok;
    d.max_nchk = h.max_nchk;
    auto at = [&](int i) -> const void* { return parts[i].bytes ? (const void*)(S.base + parts[i].off) : nullptr; };
    d.cg = (const int4*)at(0);
    d.chk_cg = (const uint16_t*)at(1);
    d.slot_var = (const int*)at(2);
    d.slot_desc = (const uint32_t*)at(3);
    d.z = h.slot_desc.empty() ? 0 : h.z;
    d.vg = (const int2*)at(4);
    d.vg_slot = (const int*)at(5);
    d.sp_cg = (const int4*)at(6);
    d.sp_desc = (const int2*)at(7);
    d.sp_absent = (const uint32_t*)at(8);
    d.sp_cchunk = (const int2*)at(9);
    d.sp_ncchunk = (int)h.sp_cchunk.size();
    d.sp_vg = (const int2*)at(10);
    d.sp_ci = (const int*)at(11);
    d.sp_vchunk = (const int2*)at(12);
    d.sp_nvchunk = (int)h.sp_vchunk.size();
    d.sp_u2v = (const int*)at(13);
    for (auto& pt : parts)
      if (pt.bytes) GF2C_CUDA(cudaMemcpyAsync(S.base + pt.off, pt.src, pt.bytes, cudaMemcpyHostToDevice, st));
    S.dev = d;
    GF2C_CUDA(cudaMemcpyAsync(S.base + off_code, &S.dev, sizeof(DevCode), cudaMemcpyHostToDevice, st));
    S.resident = &h;
    S.resident_serial = h.serial;
    S.tables_end = tables_end;
  }

  // launch attributes and occupancy, set up again only when the kernel or its
  // shared memory changes (the first call on a device does it)
  if (S.kern != kern || S.kern_smem != smem) {
    GF2C_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem));
    if (occ <= 0) return set_error(GF2C_ERR_UNSUPPORTED, "decode kernel does not fit on an SM");
    if (!S.sms) GF2C_CUDA(cudaDeviceGetAttribute(&S.sms, cudaDevAttrMultiProcessorCount, dev));
    S.kern = kern;
    S.kern_smem = smem;
    S.kern_occ = occ;
  }
  // launch shape limited by the scratch left for workspaces
  const int64_t fit = work_stride ? (int64_t)((kScratchBytes - tables_end) / work_stride) : (int64_t)1 << 30;
  const int grid = (int)std::min<int64_t>(std::min<int64_t>((int64_t)S.sms * S.kern_occ, fit), frames);

  // the queue counter and the status word start at zero on every call
  GF2C_CUDA(cudaMemsetAsync(S.base, 0, 256, st));
  DecodeArgs a{};
  a.codes = (const DevCode*)(S.base + off_code);
  a.ncodes = 1;
  a.llr = llr;
  a.max_iter = max_iter;
  a.msg = msg_bits;
  a.iters = iterations;
  a.conv = converged;
  a.synd_ok = syndrome_ok;
  a.frames = frames;
  a.queue = (unsigned long long*)S.base;
  a.status = (int*)(S.base + 8);
  a.work = (char*)(S.base + tables_end);
  a.work_stride = (long long)work_stride;
  a.app_offset = (long long)c2v_bytes;
  a.smem_app_floats = smem_app;
  a.bitmap_words = bitmap_words;
  a.early_stop = 1;
  a.sf_msg16 = 0;
  a.sf_app_soff = (int)st_bytes;
  a.sf_llr_off = (long long)sf_llr_off;
  a.sf_st_off = (long long)sf_st_off;
  a.sf_app_off = (long long)sf_app_off;
  void* args[] = {(void*)&a};
  GF2C_CUDA(cudaLaunchKernel(kern, dim3(grid), dim3(threads), args, smem, st));
  return GF2C_OK;
}
