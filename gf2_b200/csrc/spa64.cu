// gf2cuda FP64 sum-product judge (sm_100a).
//
// The precision reference of the library's decoders: sum-product belief
// propagation 2 atanh(prod_{j != i} tanh(x_j / 2)) evaluated in FP64 with
// CUDA's double-precision tanh / atanh, messages and posteriors stored in FP64.
// It is the GPU counterpart of the CPU oracle's FP64 sum-product (the
// semantics of the reference's unused check_node_update_spa + Llr::boxplus_n,
// crates/gf2-coding/src/ldpc/core.rs:762-787 and llr.rs:210-215) and is used
// only as a judge: the FP32 / FP16 decoders' LLR deviation, hard-decision
// agreement and FER are stated against it.  FP64 is used nowhere else.
//
// Numerics (same definition as the CPU judge): extrinsic products by prefix /
// suffix products in slot order, |P| clamped to 1 - 2^-50 (|c2v| <= 35.4), a
// check with one edge sends 0.  Schedules: flooding (core.rs:909-924: all
// checks from the previous posteriors, then posterior = LLR + sum c2v in
// ascending original check order) and layered (row groups in order, v2c from
// the pre-layer posterior, posterior += c2v_new - c2v_old, a variable with
// several edges in one row group taking its deltas in ascending circulant
// shift).  The syndrome is tested after every iteration (core.rs:918-922).
//
// One CTA decodes one frame at a time (persistent, atomic frame queue), one
// thread per check of a row group; posteriors are kept in the u order of the
// check-state plan (identity for the first k bits), so codes need the
// structured row-group plan (DVB-T2 and QC codes).
#include "internal.h"

namespace gf2c {

namespace {

constexpr int kJudgeMaxDc = 32;

struct JudgeArgs {
  const DevCode* code;
  const float* llr;
  long long frames;
  int max_iter;
  int layered;
  uint64_t* msg;
  int32_t* iters;
  uint8_t* conv;
  uint8_t* synd_ok;
  double* beliefs;
  unsigned long long* queue;
  char* work;
  long long work_stride;
  long long app_off;
};

__device__ __forceinline__ int slot_u64(const int2 D, int t, int Z) { return D.x + t - (t >= D.y ? Z : 0); }

// Sum-product check node of check t of row group g: new messages written to
// c2v; for the layered schedule the posterior deltas are applied (after a
// barrier per repeated block) -- every thread of the CTA calls this.
__device__ void judge_row_group(const DevCode& C, int g, double* app, double* c2v, bool first, bool layered) {
  const int tid = threadIdx.x;
  const int4 G = C.cg[g];  // {chk_begin, nchk, dc, edge0}
  const int nchk = G.y, d = G.z;
  const int2* sd = C.sp_desc + C.sp_cg[g].w;
  const uint32_t sync = C.cg_sync[g];
  const bool act = tid < nchk;
  const int t = act ? tid : 0;
  const uint32_t absent = (t == 0) ? C.sp_absent[g] : 0u;
  int vv[kJudgeMaxDc];   // u-order variable of each slot (-1: no edge)
  int rs[kJudgeMaxDc];   // slots holding an edge, in slot order
  double x[kJudgeMaxDc], pre[kJudgeMaxDc], delta[kJudgeMaxDc];
  int nr = 0;
  if (act) {
    for (int i = 0; i < d; i++) {
      const bool real = !((absent >> i) & 1u);
      vv[i] = real ? slot_u64(sd[i], t, nchk) : -1;
      if (real) rs[nr++] = i;
    }
    // tanh(v2c / 2) of the edges, v2c = posterior - old message
    for (int j = 0; j < nr; j++) {
      const int i = rs[j];
      const double o = first ? 0.0 : c2v[G.w + i * nchk + t];
      x[j] = tanh(__dsub_rn(app[vv[i]], o) * 0.5);
      delta[j] = o;  // the old message, replaced by the delta below
    }
    // inclusive prefix products; the extrinsic product of edge j is
    // pre[j-1] * (x[j+1] * (x[j+2] * ...)), the suffix formed on the way back
    pre[0] = x[0];
    for (int j = 1; j < nr; j++) pre[j] = __dmul_rn(pre[j - 1], x[j]);
    const double pmax = 1.0 - 8.8817841970012523e-16;  // 1 - 2^-50
    double suf = 1.0;
    for (int j = nr - 1; j >= 0; j--) {
      double e = 0.0;
      if (nr > 1) {
        double q = (j == nr - 1) ? pre[nr - 2] : (j == 0 ? suf : __dmul_rn(pre[j - 1], suf));
        q = q > pmax ? pmax : (q < -pmax ? -pmax : q);
        e = 2.0 * atanh(q);
      }
      suf = (j == nr - 1) ? x[j] : __dmul_rn(x[j], suf);
      c2v[G.w + rs[j] * nchk + t] = e;
      delta[j] = __dsub_rn(e, delta[j]);
    }
  }
  if (!layered) return;
  if (sync == 0) {
    if (act)
      for (int j = 0; j < nr; j++) app[vv[rs[j]]] = __dadd_rn(app[vv[rs[j]]], delta[j]);
  } else {
    __syncthreads();  // every pre-layer posterior read
    int j = 0;
    for (int i = 0; i < d; i++) {
      if (act && j < nr && rs[j] == i) {
        app[vv[i]] = __dadd_rn(app[vv[i]], delta[j]);
        j++;
      }
      if ((sync >> i) & 1u) __syncthreads();  // the next slot may hold the same variable
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(1024, 1) spa64_judge_kernel(const JudgeArgs a) {
  extern __shared__ uint32_t bitmap[];
  __shared__ long long s_frame;
  __shared__ int s_unsat;
  const DevCode& C = *a.code;
  const int tid = threadIdx.x, NT = blockDim.x;
  const int n = C.n, m = C.m;
  char* work = a.work + (long long)blockIdx.x * a.work_stride;
  double* c2v = (double*)work;
  double* app = (double*)(work + a.app_off);
  const int* u2v = C.sp_u2v;
  for (;;) {
    if (tid == 0) s_frame = (long long)atomicAdd(a.queue, 1ull);
    __syncthreads();
    const long long f = s_frame;
    if (f >= a.frames) break;
    const float* llr = a.llr + f * (long long)n;
    for (int u = tid; u < n; u += NT) app[u] = (double)llr[u2v ? u2v[u] : u];
    __syncthreads();
    int it = 0, converged = 0;
    while (it < a.max_iter) {
      const bool first = it == 0;
      for (int g = 0; g < C.ncg; g++) judge_row_group(C, g, app, c2v, first, a.layered != 0);
      if (!a.layered) {
        __syncthreads();  // every message of the iteration written
        // posterior = LLR + sum of c2v in ascending original check order
        for (int u = tid; u < n; u += NT) {
          const int h = u / C.vgs, j = u - h * C.vgs;
          const int2 V = C.sp_vg[h];
          double acc = (double)llr[u2v ? u2v[u] : u];
          for (int i = 0; i < V.x; i++) {
            const int e = C.sp_ci[V.y + i * C.vgs + j];
            if (e < 0) break;
            const int cc = e & 0xffffff, slot = e >> 24;
            const int4 G = C.cg[C.chk_cg[cc]];
            acc = __dadd_rn(acc, c2v[G.w + slot * G.y + (cc - G.x)]);
          }
          app[u] = acc;
        }
      }
      ++it;
      // hard decisions and the syndrome
      __syncthreads();
      for (int base = 0; base < n; base += NT) {
        const int u = base + tid;
        const unsigned b = __ballot_sync(0xffffffffu, u < n && app[u < n ? u : 0] < 0.0);
        if ((tid & 31) == 0 && u < n) bitmap[u >> 5] = b;
      }
      if (tid == 0) s_unsat = 0;
      __syncthreads();
      int cnt = 0;
      for (int cc = tid; cc < m; cc += NT) {
        const int g = C.chk_cg[cc];
        const int4 G = C.sp_cg[g];
        const int t = cc - G.x;
        const uint32_t ab = t == 0 ? C.sp_absent[g] : 0u;
        uint32_t par = 0;
        for (int i = 0; i < G.z; i++) {
          const int u = slot_u64(C.sp_desc[G.w + i], t, G.y);
          if (!((ab >> i) & 1u)) par ^= (bitmap[u >> 5] >> (u & 31)) & 1u;
        }
        cnt += (int)par;
      }
      if (cnt) atomicAdd(&s_unsat, cnt);
      __syncthreads();
      const int unsat = s_unsat;
      __syncthreads();
      if (unsat == 0) {
        converged = 1;
        break;
      }
    }
    if (it == 0) {  // max_iter = 0: the all-zero word, syndrome of the zero word passes
      for (int w = tid; w < (n + 31) / 32; w += NT) bitmap[w] = 0u;
      __syncthreads();
    }
    if (a.msg) {
      uint64_t* mo = a.msg + f * (long long)C.words_k;
      const int wn = (n + 31) >> 5;
      for (int w = tid; w < C.words_k; w += NT) {
        const uint32_t lo = bitmap[2 * w];
        const uint32_t hi = (2 * w + 1 < wn) ? bitmap[2 * w + 1] : 0u;
        unsigned long long word = (unsigned long long)lo | ((unsigned long long)hi << 32);
        const int rem = C.k - 64 * w;
        if (rem < 64) word &= (1ull << rem) - 1ull;
        mo[w] = word;
      }
    }
    if (a.beliefs) {
      double* bo = a.beliefs + f * (long long)n;
      for (int u = tid; u < n; u += NT) bo[u2v ? u2v[u] : u] = it == 0 ? 0.0 : app[u];
    }
    if (tid == 0) {
      if (a.iters) a.iters[f] = it;
      if (a.conv) a.conv[f] = (uint8_t)converged;
      if (a.synd_ok) a.synd_ok[f] = (uint8_t)(converged || it == 0);
    }
    __syncthreads();
  }
}

struct JudgeWork {
  void* work = nullptr;
  size_t work_bytes = 0;
  void* queue = nullptr;
  void* dcode = nullptr;
  ~JudgeWork() {
    if (work) cudaFree(work);
    if (queue) cudaFree(queue);
    if (dcode) cudaFree(dcode);
  }
};

thread_local JudgeWork g_judge;

}  // namespace

}  // namespace gf2c

using namespace gf2c;

extern "C" int gf2c_judge_spa64(const gf2c_code* code, int32_t schedule, const float* llr, int64_t frames,
                                int32_t max_iter, uint64_t* msg_bits, int32_t* iterations, uint8_t* converged,
                                uint8_t* syndrome_ok, double* beliefs, void* stream) {
  if (!code || frames < 0 || max_iter < 0 || (frames > 0 && !llr) || (schedule != GF2C_SCHED_FLOODING &&
                                                                      schedule != GF2C_SCHED_LAYERED))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (frames == 0) return GF2C_OK;
  HostCode& h = *code->h;
  if (h.sp_desc.empty() || !h.layered_ok)
    return set_error(GF2C_ERR_UNSUPPORTED, "FP64 judge needs a DVB-T2 or QC code (row-group plan)");
  if (h.max_dc > kJudgeMaxDc || h.max_nchk > 1024)
    return set_error(GF2C_ERR_UNSUPPORTED, "FP64 judge: check degree above 32 or row group above 1024");
  int rc = upload_code(h);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  GF2C_CUDA(cudaGetDevice(&dev));
  GF2C_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long msg_bytes = ((long long)h.e_slots * 8 + 255) / 256 * 256;
  const long long stride = msg_bytes + ((long long)h.n * 8 + 255) / 256 * 256;
  const int grid = (int)std::min<int64_t>(frames, (int64_t)sms * 2);
  const size_t need = (size_t)stride * grid;
  JudgeWork& w = g_judge;
  if (w.work_bytes < need) {
    if (w.work) cudaFree(w.work);
    w.work = nullptr;
    w.work_bytes = 0;
    GF2C_CUDA(cudaMalloc(&w.work, need));
    w.work_bytes = need;
  }
  if (!w.queue) GF2C_CUDA(cudaMalloc(&w.queue, 64));
  if (!w.dcode) GF2C_CUDA(cudaMalloc(&w.dcode, sizeof(DevCode)));
  GF2C_CUDA(cudaMemcpyAsync(w.dcode, &h.dev, sizeof(DevCode), cudaMemcpyHostToDevice, st));
  GF2C_CUDA(cudaMemsetAsync(w.queue, 0, sizeof(unsigned long long), st));
  JudgeArgs a{};
  a.code = (const DevCode*)w.dcode;
  a.llr = llr;
  a.frames = frames;
  a.max_iter = max_iter;
  a.layered = schedule == GF2C_SCHED_LAYERED;
  a.msg = msg_bits;
  a.iters = iterations;
  a.conv = converged;
  a.synd_ok = syndrome_ok;
  a.beliefs = beliefs;
  a.queue = (unsigned long long*)w.queue;
  a.work = (char*)w.work;
  a.work_stride = stride;
  a.app_off = msg_bytes;
  const int threads = std::max(32, (h.max_nchk + 31) / 32 * 32);
  const size_t smem = (size_t)((h.n + 31) / 32) * 4;
  GF2C_CUDA(cudaFuncSetAttribute(spa64_judge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  spa64_judge_kernel<<<grid, threads, smem, st>>>(a);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}
