// gf2cuda C ABI implementation: argument validation, device workspace, host
// staging, launch shapes and CUDA-graph replay.  Every entry point returns a
// status code; nothing aborts.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>

#include "internal.h"

namespace gf2c {

static thread_local std::string g_error;

int set_error(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char* what) {
  g_error = std::string(what) + ": " + cudaGetErrorString(e);
  return GF2C_ERR_CUDA;
}

// Device buffer that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t need) {
    if (need <= bytes) return GF2C_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t sz = std::max(need, (size_t)256);
    cudaError_t e = cudaMalloc(&p, sz);
    if (e == cudaErrorMemoryAllocation) {  // not sticky: the context stays usable
      cudaGetLastError();
      p = nullptr;
      return set_error(GF2C_ERR_NOMEM, "out of device memory (" + std::to_string(sz) + " bytes)");
    }
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    bytes = sz;
    return GF2C_OK;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace gf2c

using namespace gf2c;

struct GraphKey {
  std::vector<uintptr_t> v;
  bool operator<(const GraphKey& o) const { return v < o.v; }
};

struct gf2c_decoder {
  std::vector<const gf2c_code*> codes;
  gf2c_decoder_opts opts{};
  int dev = 0;
  DevBuf d_codes;
  int max_n = 0, max_m = 0, max_words_k = 0, max_e_slots = 0, max_dc = 0, max_nchk = 0;
  int dcmax = 0, threads = 0, grid = 0, bitmap_words = 0, smem_app_floats = 0;
  int lay_dbuf_off = 0, lay_dbuf_floats = 0;
  int lay_stage_off = 0, lay_stage_bytes = 0;
  const void* kernel = nullptr;
  bool state_flood = false;  // check-state flooding min-sum kernel (state_flood.cu)
  int sf_app_soff = 0;
  long long sf_llr_off = 0, sf_st_off = 0, sf_app_off = 0;
  size_t smem = 0;
  long long work_stride = 0, app_offset = 0;
  DevBuf work, queue, status, alpha, beta;
  int nms_iters = 0, nms_L = 0;
  // staging for host-memory calls
  DevBuf s_llr, s_msg, s_it, s_cv, s_so, s_bel, s_off1, s_off2, s_cid, s_mit;
  int last_launches = 0;
  std::map<GraphKey, cudaGraphExec_t> graphs;
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // pipelined host-memory batches: a second decode stream with its own
  // workspace and queue, and a stream that issues the input copies; the
  // fallback call's high-priority stream for the fallback passes and the
  // output copies (each chunk's after its primary pass, event pev_prim)
  cudaStream_t pstream = nullptr, cstream = nullptr, fstream = nullptr;
  cudaEvent_t pev_fork = nullptr, pev_join = nullptr, pev_copy[2] = {nullptr, nullptr};
  cudaEvent_t pev_prim = nullptr, pev_fjoin = nullptr;
  DevBuf work2, queue2;
  // mixed batches: rank of each code in the frame order (longest codes first),
  // frame order buffer; host copy of the ranks and the per-chunk frame counts
  // of the pipelined host-memory path
  DevBuf d_rank, d_order, s_cnt;
  std::vector<int32_t> h_rank;
  // single-code batches, hardest frames first: per-frame keys and order (one pair per stream slot)
  DevBuf d_key[2], d_korder[2];
  // fallback decoding: the frames this decoder left failing (list and count)
  DevBuf fb_list, fb_count;
  ~gf2c_decoder() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    if (gstream) {
      cudaStreamSynchronize(gstream);
      cudaStreamDestroy(gstream);
    }
    for (cudaStream_t ps : {pstream, cstream, fstream})
      if (ps) {
        cudaStreamSynchronize(ps);
        cudaStreamDestroy(ps);
      }
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    for (cudaEvent_t e : {pev_fork, pev_join, pev_copy[0], pev_copy[1], pev_prim, pev_fjoin})
      if (e) cudaEventDestroy(e);
  }
};

extern "C" {

const char* gf2c_last_error(void) { return g_error.c_str(); }
const char* gf2c_version(void) { return "gf2cuda 0.1 (sm_100a)"; }

void gf2c_decoder_opts_default(gf2c_decoder_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->algorithm = GF2C_ALGO_MINSUM;
  o->schedule = GF2C_SCHED_FLOODING;
  o->msg_dtype = GF2C_MSG_F32;
  o->early_stop = 1;
}

double gf2c_sigma2_from_ebn0(double ebn0_db, double rate) {
  return 1.0 / (2.0 * rate * std::pow(10.0, ebn0_db / 10.0));
}

static int make_code(gf2c_code** out, std::unique_ptr<HostCode> h) {
  gf2c_code* c = new (std::nothrow) gf2c_code();
  if (!c) return set_error(GF2C_ERR_NOMEM, "out of host memory");
  c->h = std::move(h);
  *out = c;
  return GF2C_OK;
}

int gf2c_code_create_dvbt2(int32_t frame_size, int32_t rate, gf2c_code** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  auto h = std::make_unique<HostCode>();
  int rc = build_dvbt2(frame_size, rate, *h);
  if (rc) return rc;
  return make_code(out, std::move(h));
}

int gf2c_code_create_qc(const int32_t* base, int32_t mb, int32_t nb, int32_t z, gf2c_code** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  auto h = std::make_unique<HostCode>();
  int rc = build_qc(base, mb, nb, z, *h);
  if (rc) return rc;
  return make_code(out, std::move(h));
}

int gf2c_code_create_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count, gf2c_code** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  auto h = std::make_unique<HostCode>();
  int rc = build_edges(m, n, pairs, count, *h);
  if (rc) return rc;
  return make_code(out, std::move(h));
}

int gf2c_code_destroy(gf2c_code* code) {
  delete code;
  return GF2C_OK;
}

int gf2c_code_dims(const gf2c_code* code, int64_t* n, int64_t* m, int64_t* k, int64_t* nnz,
                   int32_t* layers) {
  if (!code) return set_error(GF2C_ERR_INVALID_ARG, "code is NULL");
  const HostCode& h = *code->h;
  if (n) *n = h.n;
  if (m) *m = h.m;
  if (k) *k = h.k;
  if (nnz) *nnz = (int64_t)h.row_idx.size();
  if (layers) *layers = h.layered_ok ? (int32_t)h.cg.size() : 0;
  return GF2C_OK;
}

int gf2c_code_csr(const gf2c_code* code, int64_t* indptr, int64_t* indices) {
  if (!code || !indptr || !indices) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  const HostCode& h = *code->h;
  std::memcpy(indptr, h.row_ptr.data(), sizeof(int64_t) * h.row_ptr.size());
  if (!h.row_idx.empty()) std::memcpy(indices, h.row_idx.data(), sizeof(int64_t) * h.row_idx.size());
  return GF2C_OK;
}

// ---------------------------------------------------------------------------
// helpers for host / device argument handling
// ---------------------------------------------------------------------------
static int check_mem(int32_t mem) {
  if (mem != GF2C_MEM_HOST && mem != GF2C_MEM_DEVICE)
    return set_error(GF2C_ERR_INVALID_ARG, "mem must be GF2C_MEM_HOST or GF2C_MEM_DEVICE");
  return GF2C_OK;
}

static int ensure_code_on_device(const gf2c_code* code) {
  return upload_code(*code->h);
}

// One DevCode on the device for single-code kernels (kept in the HostCode).
static int code_dev_struct(const gf2c_code* code, DevBuf& buf) {
  int rc = ensure_code_on_device(code);
  if (rc) return rc;
  if ((rc = buf.ensure(sizeof(DevCode)))) return rc;
  GF2C_CUDA(cudaMemcpy(buf.p, &code->h->dev, sizeof(DevCode), cudaMemcpyHostToDevice));
  return GF2C_OK;
}

struct CodeOps {
  DevBuf dcode, in, out, aux, aux2;
};
static thread_local CodeOps g_ops;

int gf2c_syndrome_batch(const gf2c_code* code, const uint64_t* cw_bits, int64_t frames,
                        uint64_t* synd_bits, int32_t* weight, int32_t mem, void* stream) {
  if (!code || frames < 0 || (frames > 0 && !cw_bits)) return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  int rc = check_mem(mem);
  if (rc || frames == 0) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = code_dev_struct(code, g_ops.dcode))) return rc;
  const DevCode& h = code->h->dev;
  if (mem == GF2C_MEM_DEVICE)
    return launch_syndrome((const DevCode*)g_ops.dcode.p, h, cw_bits, frames, synd_bits, weight, st);
  size_t bin = (size_t)frames * h.words_n * 8, bs = (size_t)frames * h.words_m * 8, bw = (size_t)frames * 4;
  if ((rc = g_ops.in.ensure(bin)) || (rc = g_ops.out.ensure(bs)) || (rc = g_ops.aux.ensure(bw))) return rc;
  GF2C_CUDA(cudaMemcpyAsync(g_ops.in.p, cw_bits, bin, cudaMemcpyHostToDevice, st));
  if ((rc = launch_syndrome((const DevCode*)g_ops.dcode.p, h, (const uint64_t*)g_ops.in.p, frames,
                            (uint64_t*)g_ops.out.p, (int32_t*)g_ops.aux.p, st)))
    return rc;
  if (synd_bits) GF2C_CUDA(cudaMemcpyAsync(synd_bits, g_ops.out.p, bs, cudaMemcpyDeviceToHost, st));
  if (weight) GF2C_CUDA(cudaMemcpyAsync(weight, g_ops.aux.p, bw, cudaMemcpyDeviceToHost, st));
  GF2C_CUDA(cudaStreamSynchronize(st));
  return GF2C_OK;
}

int gf2c_encode_batch(const gf2c_code* code, const uint64_t* msg_bits, int64_t frames, uint64_t* cw_bits,
                      int32_t mem, void* stream) {
  if (!code || frames < 0 || (frames > 0 && (!msg_bits || !cw_bits)))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  int rc = check_mem(mem);
  if (rc || frames == 0) return rc;
  if ((rc = prepare_encoder(*code->h))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = code_dev_struct(code, g_ops.dcode))) return rc;
  const DevCode& h = code->h->dev;
  if (mem == GF2C_MEM_DEVICE) return launch_encode((const DevCode*)g_ops.dcode.p, h, msg_bits, frames, cw_bits, st);
  size_t bin = (size_t)frames * h.words_k * 8, bout = (size_t)frames * h.words_n * 8;
  if ((rc = g_ops.in.ensure(bin)) || (rc = g_ops.out.ensure(bout))) return rc;
  GF2C_CUDA(cudaMemcpyAsync(g_ops.in.p, msg_bits, bin, cudaMemcpyHostToDevice, st));
  if ((rc = launch_encode((const DevCode*)g_ops.dcode.p, h, (const uint64_t*)g_ops.in.p, frames,
                          (uint64_t*)g_ops.out.p, st)))
    return rc;
  GF2C_CUDA(cudaMemcpyAsync(cw_bits, g_ops.out.p, bout, cudaMemcpyDeviceToHost, st));
  GF2C_CUDA(cudaStreamSynchronize(st));
  return GF2C_OK;
}

int gf2c_channel_awgn(const gf2c_code* code, uint64_t seed, uint64_t frame0, int64_t frames,
                      const double* sigma2, uint64_t* info_bits, uint64_t* cw_bits, float* llr,
                      int32_t mem, void* stream) {
  if (!code || frames < 0 || (frames > 0 && !sigma2)) return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  int rc = check_mem(mem);
  if (rc || frames == 0) return rc;
  if (mem == GF2C_MEM_HOST)
    for (int64_t f = 0; f < frames; f++)
      if (!(sigma2[f] > 0.0) || !std::isfinite(sigma2[f]))
        return set_error(GF2C_ERR_INVALID_ARG, "sigma2 must be positive and finite");
  if ((rc = prepare_encoder(*code->h))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = code_dev_struct(code, g_ops.dcode))) return rc;
  const DevCode& h = code->h->dev;
  if (mem == GF2C_MEM_DEVICE)
    return launch_channel((const DevCode*)g_ops.dcode.p, h, seed, frame0, frames, sigma2, info_bits, cw_bits,
                          llr, st);
  size_t bi = (size_t)frames * h.words_k * 8, bc = (size_t)frames * h.words_n * 8,
         bl = (size_t)frames * h.n * 4, bs = (size_t)frames * 8;
  if ((rc = g_ops.in.ensure(bs)) || (rc = g_ops.out.ensure(bl)) || (rc = g_ops.aux.ensure(bi)) ||
      (rc = g_ops.aux2.ensure(bc)))
    return rc;
  GF2C_CUDA(cudaMemcpyAsync(g_ops.in.p, sigma2, bs, cudaMemcpyHostToDevice, st));
  if ((rc = launch_channel((const DevCode*)g_ops.dcode.p, h, seed, frame0, frames, (const double*)g_ops.in.p,
                           info_bits ? (uint64_t*)g_ops.aux.p : nullptr,
                           cw_bits ? (uint64_t*)g_ops.aux2.p : nullptr, llr ? (float*)g_ops.out.p : nullptr, st)))
    return rc;
  if (info_bits) GF2C_CUDA(cudaMemcpyAsync(info_bits, g_ops.aux.p, bi, cudaMemcpyDeviceToHost, st));
  if (cw_bits) GF2C_CUDA(cudaMemcpyAsync(cw_bits, g_ops.aux2.p, bc, cudaMemcpyDeviceToHost, st));
  if (llr) GF2C_CUDA(cudaMemcpyAsync(llr, g_ops.out.p, bl, cudaMemcpyDeviceToHost, st));
  GF2C_CUDA(cudaStreamSynchronize(st));
  return GF2C_OK;
}

// ---------------------------------------------------------------------------
// decoder
// ---------------------------------------------------------------------------
static const int kSmemBudget = 200 * 1024;

int gf2c_decoder_create_multi(const gf2c_code* const* codes, int32_t ncodes, const gf2c_decoder_opts* opts,
                              gf2c_decoder** out) {
  if (!out || !codes || ncodes <= 0) return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  for (int i = 0; i < ncodes; i++)
    if (!codes[i]) return set_error(GF2C_ERR_INVALID_ARG, "NULL code handle");
  gf2c_decoder_opts o;
  if (opts) o = *opts;
  else gf2c_decoder_opts_default(&o);
  if (o.algorithm < 0 || o.algorithm > 3 || o.schedule < 0 || o.schedule > 1 || o.msg_dtype < 0 ||
      o.msg_dtype > 1 || o.threads_per_block < 0 || o.threads_per_block > 1024 || o.blocks_per_sm < 0 ||
      (o.threads_per_block % 32) != 0)
    return set_error(GF2C_ERR_INVALID_ARG, "invalid decoder options");
  std::unique_ptr<gf2c_decoder> d(new (std::nothrow) gf2c_decoder());
  if (!d) return set_error(GF2C_ERR_NOMEM, "out of host memory");
  d->opts = o;
  d->opts.nms_alpha = nullptr;
  d->opts.nms_beta = nullptr;
  GF2C_CUDA(cudaGetDevice(&d->dev));
  std::vector<DevCode> dc;
  for (int i = 0; i < ncodes; i++) {
    if (!codes[i]) return set_error(GF2C_ERR_INVALID_ARG, "NULL code handle");
    const HostCode& h = *codes[i]->h;
    if (o.schedule == GF2C_SCHED_LAYERED && (!h.layered_ok || h.sp_desc.empty()))
      return set_error(GF2C_ERR_UNSUPPORTED, "layered schedule needs a QC or DVB-T2 code with Z <= 1023");
    int rc = ensure_code_on_device(codes[i]);
    if (rc) return rc;
    d->codes.push_back(codes[i]);
    dc.push_back(h.dev);
    d->max_n = std::max(d->max_n, (int)h.n);
    d->max_m = std::max(d->max_m, (int)h.m);
    d->max_words_k = std::max(d->max_words_k, (int)((h.k + 63) / 64));
    d->max_e_slots = std::max(d->max_e_slots, h.e_slots);
    d->max_dc = std::max(d->max_dc, h.max_dc);
    d->max_nchk = std::max(d->max_nchk, h.max_nchk);
  }
  const bool layered = o.schedule == GF2C_SCHED_LAYERED;
  d->dcmax = layered ? layered_dcmax_bucket(d->max_dc) : decode_dcmax_bucket(d->max_dc);
  if (d->dcmax < 0)
    return set_error(GF2C_ERR_UNSUPPORTED, layered ? "layered schedule: check degree above 32"
                                                   : "check degree above 64");
  int rc = d->d_codes.ensure(sizeof(DevCode) * dc.size());
  if (rc) return rc;
  GF2C_CUDA(cudaMemcpy(d->d_codes.p, dc.data(), sizeof(DevCode) * dc.size(), cudaMemcpyHostToDevice));
  if (d->codes.size() > 1) {
    // mixed batches are decoded code by code: longest frames first, then by code index
    std::vector<int> by(d->codes.size());
    for (size_t i = 0; i < by.size(); i++) by[i] = (int)i;
    std::stable_sort(by.begin(), by.end(), [&](int x, int y) { return d->codes[x]->h->n > d->codes[y]->h->n; });
    std::vector<int32_t> rank(by.size());
    for (size_t r = 0; r < by.size(); r++) rank[by[r]] = (int32_t)r;
    if ((rc = d->d_rank.ensure(sizeof(int32_t) * rank.size()))) return rc;
    GF2C_CUDA(cudaMemcpy(d->d_rank.p, rank.data(), sizeof(int32_t) * rank.size(), cudaMemcpyHostToDevice));
    d->h_rank = rank;
  }

  // NMS weights
  if (o.algorithm == GF2C_ALGO_NMS) {
    if (!opts || !opts->nms_alpha || !opts->nms_beta || opts->nms_iters <= 0)
      return set_error(GF2C_ERR_INVALID_ARG, "NMS needs nms_alpha, nms_beta and nms_iters > 0");
    const HostCode& h0 = *codes[0]->h;
    d->nms_L = h0.layered_ok ? (int)h0.cg.size() : 1;
    d->nms_iters = opts->nms_iters;
    size_t nb = sizeof(float) * (size_t)d->nms_iters * d->nms_L;
    for (size_t i = 0; i < (size_t)d->nms_iters * d->nms_L; i++)
      if (!std::isfinite(opts->nms_alpha[i]) || !std::isfinite(opts->nms_beta[i]))
        return set_error(GF2C_ERR_INVALID_ARG, "NMS weights must be finite");
    if ((rc = d->alpha.ensure(nb)) || (rc = d->beta.ensure(nb))) return rc;
    GF2C_CUDA(cudaMemcpy(d->alpha.p, opts->nms_alpha, nb, cudaMemcpyHostToDevice));
    GF2C_CUDA(cudaMemcpy(d->beta.p, opts->nms_beta, nb, cudaMemcpyHostToDevice));
  }

  // Layered min-sum runs on the normalised / offset min-sum kernels with one
  // weight pair alpha = 1, beta = 0 (bit-identical messages: 1 * max(m - 0, 0) = m).
  if (o.schedule == GF2C_SCHED_LAYERED && o.algorithm == GF2C_ALGO_MINSUM) {
    const float one = 1.0f, zero = 0.0f;
    d->nms_L = 1;
    d->nms_iters = 1;
    if ((rc = d->alpha.ensure(sizeof(float))) || (rc = d->beta.ensure(sizeof(float)))) return rc;
    GF2C_CUDA(cudaMemcpy(d->alpha.p, &one, sizeof(float), cudaMemcpyHostToDevice));
    GF2C_CUDA(cudaMemcpy(d->beta.p, &zero, sizeof(float), cudaMemcpyHostToDevice));
  }

  // launch shape
  int sms = 148;
  GF2C_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->dev));
  int threads = o.threads_per_block;
  if (threads == 0) threads = layered ? ((d->max_nchk + 31) / 32) * 32 : 512;
  // Layered: one thread per check of a row group, or (several checks per
  // thread, more frames in flight per SM) 192 / 128 threads for one code with
  // FP16 messages and a fused-row algorithm, on the TMA-staged kernel.
  const bool multi = layered && threads < d->max_nchk;
  // a mixed batch: 192 threads for the SFU sum-product (the mixed kernel)
  const bool multi_mixed = multi && d->codes.size() > 1 && threads == 192 && o.algorithm == GF2C_ALGO_SPA_FAST;
  if (multi && !((threads == 192 || threads == 128) && (d->codes.size() == 1 || multi_mixed) &&
                 o.msg_dtype == GF2C_MSG_F16 && o.algorithm != GF2C_ALGO_SPA && d->max_nchk <= 384))
    return set_error(GF2C_ERR_INVALID_ARG,
                     "layered schedule needs threads_per_block >= row group size (or 192 / 128 threads for one "
                     "DVB-T2 code, FP16 messages, min-sum / NMS / SFU sum-product)");
  threads = std::max(threads, 32);
  d->threads = threads;
  d->bitmap_words = (d->max_n + 31) / 32;
  auto smem_of = [&](int app_floats) {
    return layered ? layered_smem_bytes(app_floats, d->bitmap_words)
                   : decode_smem_bytes(app_floats, d->bitmap_words);
  };
  // keep the APP of every code whose n fits in shared memory there
  d->smem_app_floats = 0;
  for (auto* c : d->codes)
    if (smem_of((int)c->h->n) <= (size_t)kSmemBudget) d->smem_app_floats = std::max(d->smem_app_floats, (int)c->h->n);
  // several checks per thread over a mixed batch: every posterior in the
  // workspace, so that the CTAs are small enough for four per SM
  if (multi_mixed) d->smem_app_floats = 0;
  d->smem = smem_of(d->smem_app_floats);
  if (layered && o.algorithm != GF2C_ALGO_SPA) {
    // row groups with repeated variables: deltas of every slot (fused row paths)
    int fl = 0;
    for (auto* c : d->codes)
      for (size_t g = 0; g < c->h->cg.size(); g++)
        if (c->h->cg_sync[g] != 0) fl = std::max(fl, c->h->cg[g].z * c->h->cg[g].y);
    if (fl > 0) {  // taken below where it costs no occupancy
      d->lay_dbuf_off = (int)((d->smem + 15) & ~(size_t)15);
      d->lay_dbuf_floats = fl;
    }
  }
  const size_t msg_bytes = o.msg_dtype == GF2C_MSG_F16 ? 2 : 4;
  // per-edge messages, or (layered min-sum family) one compressed state per check
  const long long c2v_bytes = (std::max((long long)d->max_e_slots * (long long)msg_bytes,
                                        (long long)d->max_m * (o.msg_dtype == GF2C_MSG_F16 ? 8 : 16)) +
                               255) / 256 * 256;
  d->app_offset = c2v_bytes;
  const bool need_gapp = d->max_n > d->smem_app_floats;
  d->work_stride = c2v_bytes + (need_gapp ? ((long long)d->max_n * 4 + 255) / 256 * 256 : 0);
  d->kernel = layered ? layered_kernel_ptr(o.algorithm, o.msg_dtype, d->dcmax, threads)
                      : flood_kernel_ptr(o.algorithm, o.msg_dtype, d->dcmax, threads);
  if (layered && threads <= 384) {
    // codes of different slot counts (a mixed batch): the kernel that runs each
    // frame with its own code's exact slot count, where one exists
    bool differ = false, dispatchable = true;
    for (auto* c : d->codes) {
      const int b = layered_dcmax_bucket(c->h->max_dc);
      differ = differ || b != d->dcmax;
      dispatchable = dispatchable && b > 0 && b <= 22;
    }
    const void* k = ((differ || multi_mixed) && dispatchable) ? layered_kernel_ptr(o.algorithm, o.msg_dtype, 0, threads)
                                                               : nullptr;
    if (k) d->kernel = k;
  }
  // Flooding min-sum / normalised-offset min-sum: the check-state kernel, with
  // the check states and posteriors in shared memory where they fit.
  const bool ms_family = o.algorithm == GF2C_ALGO_MINSUM || o.algorithm == GF2C_ALGO_NMS;
  const int sf_dc = state_dcmax_bucket(d->max_dc);
  if (!layered && ms_family && sf_dc > 0 && !std::getenv("GF2C_NO_STATE_FLOOD") &&
      (o.threads_per_block == 0 || o.threads_per_block == state_flood_threads())) {
    const size_t budget = 224 * 1024;
    const size_t st_bytes = (size_t)d->max_m * 16, app_bytes = (size_t)d->max_n * 4;
    bool any_perm = false;
    for (auto* c : d->codes) any_perm = any_perm || !c->h->sp_u2v.empty();
    // Either the whole frame state is on chip, or all of it is in the workspace:
    // keeping only part of it in shared memory (measured on normal 3/5 frames)
    // shrinks L1, which caches the workspace, by more than it saves in L2 traffic.
    const bool all_smem = st_bytes + app_bytes <= budget;
    d->sf_app_soff = (int)st_bytes;
    auto al = [](long long x) { return (x + 255) / 256 * 256; };
    long long off = 0;
    d->sf_llr_off = off;
    off += any_perm ? al(app_bytes) : 0;
    d->sf_st_off = off;
    off += all_smem ? 0 : al(st_bytes);
    d->sf_app_off = off;
    off += all_smem ? 0 : al(app_bytes);
    d->work_stride = off;
    d->smem = all_smem ? st_bytes + app_bytes : 0;
    d->kernel = state_flood_kernel_ptr(sf_dc, all_smem);
    d->dcmax = sf_dc;
    threads = state_flood_threads();
    d->threads = threads;
    d->state_flood = true;
  }
  if (!layered && !d->state_flood && threads > 512 && !d->kernel)
    return set_error(GF2C_ERR_INVALID_ARG,
                     "flooding schedule: threads_per_block above 512 needs a code of check degree <= 8");
  if (!d->kernel && !multi) return set_error(GF2C_ERR_UNSUPPORTED, "no decode kernel for this configuration");
  if (multi && d->lay_dbuf_floats > 0) {
    // several checks per thread: the delta buffer is required
    d->smem = (size_t)d->lay_dbuf_off + (size_t)d->lay_dbuf_floats * 4;
  } else if (d->lay_dbuf_floats > 0) {
    int optin = 0, occ0 = 0, occ1 = 0;
    GF2C_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->dev));
    const size_t with = (size_t)d->lay_dbuf_off + (size_t)d->lay_dbuf_floats * 4;
    if (with <= (size_t)optin) {
      GF2C_CUDA(cudaFuncSetAttribute(d->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)with));
      GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, d->kernel, threads, d->smem));
      GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, d->kernel, threads, with));
    }
    if (occ1 > 0 && occ1 >= occ0) {
      d->smem = with;
    } else {
      d->lay_dbuf_off = 0;
      d->lay_dbuf_floats = 0;
    }
  }
  // Layered decoding of one code with a fused-row algorithm: the old messages
  // of each row group are staged in shared memory by TMA bulk copies (a row
  // group's messages are one contiguous block, which must start and end on a
  // 16-byte boundary; three or more row groups), where this costs no occupancy.
  if (layered && d->codes.size() == 1 && o.algorithm != GF2C_ALGO_SPA && threads <= 384 &&
      !std::getenv("GF2C_NO_STAGE")) {
    const HostCode& h = *d->codes[0]->h;
    // the min-sum family keeps compressed check states and stages nothing (the
    // staged kernel then only needs its two mbarriers)
    const bool states = layered_state_mode(o.algorithm, d->dcmax, true);
    bool ok = states || h.cg.size() >= 3;
    size_t mx = 0;
    for (const int4& G : h.cg) {
      const size_t off = (size_t)G.w * msg_bytes, by = (size_t)G.z * G.y * msg_bytes;
      ok = ok && (states || (off % 16 == 0 && by % 16 == 0));
      if (!states) mx = std::max(mx, by);
    }
    const void* k = ok ? layered_kernel_ptr(o.algorithm, o.msg_dtype, d->dcmax, threads, true, o.blocks_per_sm)
                       : nullptr;
    int optin = 0, occ0 = 0, occ1 = 0;
    GF2C_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->dev));
    const size_t off = (d->smem + 15) & ~(size_t)15, with = off + 2 * mx + 16;
    if (k && with <= (size_t)optin) {
      if (d->kernel) {
        GF2C_CUDA(cudaFuncSetAttribute(d->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d->smem));
        GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, d->kernel, threads, d->smem));
      }
      GF2C_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)with));
      GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, k, threads, with));
      if (occ1 > 0 && (occ1 >= occ0 || !d->kernel || std::getenv("GF2C_FORCE_STAGE"))) {
        d->kernel = k;
        d->smem = with;
        d->lay_stage_off = (int)off;
        d->lay_stage_bytes = (int)mx;
      }
    }
  }
  if (!d->kernel)
    return set_error(GF2C_ERR_UNSUPPORTED, "no decode kernel for this configuration (several checks per thread "
                                          "need the staged kernel: 16-byte aligned row groups, >= 3 row groups)");
  GF2C_CUDA(cudaFuncSetAttribute(d->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d->smem));
  int occ = 0;
  GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, d->kernel, threads, d->smem));
  if (occ <= 0) return set_error(GF2C_ERR_UNSUPPORTED, "decode kernel does not fit on an SM with this shape");
  int bps = o.blocks_per_sm ? std::min(o.blocks_per_sm, occ) : occ;
  d->grid = sms * bps;
  if ((rc = d->work.ensure((size_t)d->work_stride * d->grid))) return rc;
  if ((rc = d->queue.ensure(64)) || (rc = d->status.ensure(64))) return rc;
  GF2C_CUDA(cudaMemset(d->status.p, 0, 64));
  *out = d.release();
  return GF2C_OK;
}

int gf2c_decoder_create(const gf2c_code* code, const gf2c_decoder_opts* opts, gf2c_decoder** out) {
  const gf2c_code* codes[1] = {code};
  return gf2c_decoder_create_multi(codes, 1, opts, out);
}

int gf2c_decoder_destroy(gf2c_decoder* dec) {
  delete dec;
  return GF2C_OK;
}

int gf2c_decoder_last_launches(const gf2c_decoder* dec, int32_t* launches) {
  if (!dec || !launches) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  *launches = dec->last_launches;
  return GF2C_OK;
}

// slot 1: the second workspace and queue of the pipelined host-memory path
static int launch_decoder(gf2c_decoder* d, DecodeArgs& a, int64_t frames, cudaStream_t st, int slot = 0) {
  a.codes = (const DevCode*)d->d_codes.p;
  a.ncodes = (int)d->codes.size();
  a.frames = frames;
  a.queue = (unsigned long long*)(slot ? d->queue2.p : d->queue.p);
  a.work = (char*)(slot ? d->work2.p : d->work.p);
  a.work_stride = d->work_stride;
  a.app_offset = d->app_offset;
  a.smem_app_floats = d->smem_app_floats;
  a.bitmap_words = d->bitmap_words;
  a.lay_dbuf_off = d->lay_dbuf_off;
  a.lay_dbuf_floats = d->lay_dbuf_floats;
  a.lay_stage_off = d->lay_stage_off;
  a.lay_stage_bytes = d->lay_stage_bytes;
  a.alpha = (const float*)d->alpha.p;
  a.beta = (const float*)d->beta.p;
  a.nms_iters = (d->opts.algorithm == GF2C_ALGO_NMS ||
                 (d->opts.algorithm == GF2C_ALGO_MINSUM && d->opts.schedule == GF2C_SCHED_LAYERED))
                    ? d->nms_iters
                    : 0;
  a.nms_L = d->nms_L;
  a.early_stop = d->opts.early_stop;
  a.status = (int*)d->status.p;
  a.sf_app_soff = d->sf_app_soff;
  a.sf_msg16 = d->opts.msg_dtype == GF2C_MSG_F16;
  a.sf_llr_off = d->sf_llr_off;
  a.sf_st_off = d->sf_st_off;
  a.sf_app_off = d->sf_app_off;
  GF2C_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(unsigned long long), st));
  int grid = (int)std::min<int64_t>(d->grid, frames);
  d->last_launches = 1;
  void* args[] = {(void*)&a};
  GF2C_CUDA(cudaLaunchKernel(d->kernel, dim3(grid), dim3(d->threads), args, d->smem, st));
  return GF2C_OK;
}

// Single-code batches of more frames than CTAs are decoded hardest frames first
// (ascending sum of |LLR|), so that the last frames the persistent kernel
// takes are short ones and the SMs finish together.  Per-frame results do not
// depend on the order.  Skipped above kKeyOrderMax frames, and while `st` is
// being captured into a graph if the buffers would have to grow.  Returns the
// number of kernels launched (0 or 2) in `launches`.
static int key_order(gf2c_decoder* d, DecodeArgs& a, int64_t frames, cudaStream_t st, int slot, int& launches) {
  launches = 0;
  if (d->codes.size() != 1 || frames <= d->grid || frames > kKeyOrderMax) return GF2C_OK;
  DevBuf& kb = d->d_key[slot];
  DevBuf& ob = d->d_korder[slot];
  if (kb.bytes < (size_t)frames * 4 || ob.bytes < (size_t)frames * 8) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return GF2C_OK;
    }
    int rc;
    if ((rc = kb.ensure((size_t)frames * 4)) || (rc = ob.ensure((size_t)frames * 8))) return rc;
  }
  GF2C_CUDA(launch_key_order(a.llr, (int)d->codes[0]->h->n, frames, (float*)kb.p, (int64_t*)ob.p, st));
  a.order = (const int64_t*)ob.p;
  launches = 2;
  return GF2C_OK;
}

static int check_status(gf2c_decoder* d, cudaStream_t st) {
  int h = 0;
  GF2C_CUDA(cudaMemcpyAsync(&h, d->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  GF2C_CUDA(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(d->status.p, 0, sizeof(int), st);
    if (h == 2) return set_error(GF2C_ERR_KERNEL, "a staged message copy did not complete in time");
    return set_error(GF2C_ERR_INVALID_ARG, "a frame referenced a code id outside the decoder's codes");
  }
  return GF2C_OK;
}

// Chunk sizes of the pipelined host-memory paths.  Mixed batches: one wave of
// frames first (the copy that nothing overlaps is short), then doubling up to
// an eighth of the batch.  Single-code batches: chunks of one size, the larger
// of one wave and a 64th of the batch, so that the copy of the first chunk and
// the decode of the last one (what the copies cannot overlap) are short, and
// each chunk's copy takes about as long as the previous chunk's decode when
// the two run at about the same speed (the copy stream then stays busy from
// the first copy to the last).  A remainder below one wave joins the last
// chunk.
static int64_t chunk_frames(int64_t want, int64_t left, int64_t wave) {
  const int64_t nf = std::min(want, left);
  return (left - nf < wave) ? left : nf;
}
static int64_t chunk_cap(int64_t frames, int64_t wave) { return std::max(wave, (frames + 7) / 8); }
static int64_t even_chunk(int64_t frames, int64_t wave) { return std::max(wave, (frames + 63) / 64); }

// The second decode stream, its workspace and queue, and the copy stream of
// the pipelined host-memory path (made on first use; false where they cannot
// be had, and the call then runs unpipelined).
static bool pipeline_ready(gf2c_decoder* d) {
  for (cudaStream_t* ps : {&d->pstream, &d->cstream})
    if (!*ps && cudaStreamCreateWithFlags(ps, cudaStreamNonBlocking) != cudaSuccess) {
      *ps = nullptr;
      cudaGetLastError();
      return false;
    }
  for (cudaEvent_t* e : {&d->pev_fork, &d->pev_join, &d->pev_copy[0], &d->pev_copy[1]})
    if (!*e && cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) {
      *e = nullptr;
      cudaGetLastError();
      return false;
    }
  if (d->work2.ensure((size_t)d->work_stride * d->grid) != GF2C_OK || d->queue2.ensure(64) != GF2C_OK) {
    cudaGetLastError();  // an allocation failure: the call runs unpipelined
    return false;
  }
  return true;
}

int gf2c_decode_batch(gf2c_decoder* dec, const float* llr, int64_t frames, int32_t max_iter, uint64_t* msg_bits,
                      int32_t* iterations, uint8_t* converged, uint8_t* syndrome_ok, float* beliefs, int32_t mem,
                      void* stream) {
  if (!dec || frames < 0 || max_iter < 0 || (frames > 0 && !llr))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  int rc = check_mem(mem);
  if (rc || frames == 0) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const HostCode& h = *dec->codes[0]->h;
  DecodeArgs a{};
  a.max_iter = max_iter;
  if (mem == GF2C_MEM_DEVICE) {
    a.llr = llr;
    a.msg = msg_bits;
    a.iters = iterations;
    a.conv = converged;
    a.synd_ok = syndrome_ok;
    a.beliefs = beliefs;
    int extra = 0;
    if ((rc = key_order(dec, a, frames, st, 0, extra))) return rc;
    if ((rc = launch_decoder(dec, a, frames, st))) return rc;
    dec->last_launches += extra;
    return GF2C_OK;
  }
  const int wk = (int)((h.k + 63) / 64);
  size_t bl = (size_t)frames * h.n * 4, bm = (size_t)frames * wk * 8;
  if ((rc = dec->s_llr.ensure(bl)) || (rc = dec->s_msg.ensure(bm)) || (rc = dec->s_it.ensure(frames * 4)) ||
      (rc = dec->s_cv.ensure(frames)) || (rc = dec->s_so.ensure(frames)))
    return rc;
  if (beliefs && (rc = dec->s_bel.ensure(bl))) return rc;
  // Large batches: chunks of frames alternating between the caller's stream and
  // a second stream, each stream running decode and copy out of its chunks in
  // order, while a copy stream brings the chunks in back to back (the staging
  // buffer holds the whole batch, so no copy waits for a decode).  A chunk's
  // decode waits for its own copy only and starts on the SMs that the previous
  // chunk's last frames leave free (each stream has its own workspace and
  // frame queue).  Only the last chunk is decoded hardest frames first: the
  // ordering kernels of the others would wait for those SMs, which the next
  // chunk's decode fills anyway.
  const int64_t chunk = std::max<int64_t>(dec->grid, (frames + 7) / 8);
  if (frames >= 2 * chunk && bl >= ((size_t)64 << 20) && pipeline_ready(dec)) {
    GF2C_CUDA(cudaEventRecord(dec->pev_fork, st));
    GF2C_CUDA(cudaStreamWaitEvent(dec->pstream, dec->pev_fork, 0));
    GF2C_CUDA(cudaStreamWaitEvent(dec->cstream, dec->pev_fork, 0));
    int chunks = 0, launches = 0;
    const int64_t csz = even_chunk(frames, dec->grid);
    for (int64_t f0 = 0, nf = 0; f0 < frames; f0 += nf, chunks++) {
      nf = chunk_frames(csz, frames - f0, dec->grid);
      const int slot = chunks & 1;
      cudaStream_t s = slot ? dec->pstream : st;
      const size_t ln = (size_t)nf * h.n * 4, lo = (size_t)f0 * h.n * 4;
      const size_t mn = (size_t)nf * wk * 8, mo = (size_t)f0 * wk * 8;
      // input copies back to back on the copy stream (the staging buffer holds
      // the whole batch), each chunk's decode waiting for its own copy only
      GF2C_CUDA(cudaMemcpyAsync((char*)dec->s_llr.p + lo, (const char*)llr + lo, ln, cudaMemcpyHostToDevice,
                                dec->cstream));
      GF2C_CUDA(cudaEventRecord(dec->pev_copy[slot], dec->cstream));
      GF2C_CUDA(cudaStreamWaitEvent(s, dec->pev_copy[slot], 0));
      DecodeArgs b = a;
      b.llr = (const float*)((char*)dec->s_llr.p + lo);
      b.msg = msg_bits ? (uint64_t*)((char*)dec->s_msg.p + mo) : nullptr;
      b.iters = (int32_t*)dec->s_it.p + f0;
      b.conv = (uint8_t*)dec->s_cv.p + f0;
      b.synd_ok = (uint8_t*)dec->s_so.p + f0;
      b.beliefs = beliefs ? (float*)((char*)dec->s_bel.p + lo) : nullptr;
      int extra = 0;
      if (f0 + nf == frames && (rc = key_order(dec, b, nf, s, slot, extra))) return rc;
      if ((rc = launch_decoder(dec, b, nf, s, slot))) return rc;
      launches += 1 + extra;
      if (msg_bits)
        GF2C_CUDA(cudaMemcpyAsync((char*)msg_bits + mo, (char*)dec->s_msg.p + mo, mn, cudaMemcpyDeviceToHost, s));
      if (iterations)
        GF2C_CUDA(cudaMemcpyAsync(iterations + f0, (int32_t*)dec->s_it.p + f0, nf * 4, cudaMemcpyDeviceToHost, s));
      if (converged)
        GF2C_CUDA(cudaMemcpyAsync(converged + f0, (uint8_t*)dec->s_cv.p + f0, nf, cudaMemcpyDeviceToHost, s));
      if (syndrome_ok)
        GF2C_CUDA(cudaMemcpyAsync(syndrome_ok + f0, (uint8_t*)dec->s_so.p + f0, nf, cudaMemcpyDeviceToHost, s));
      if (beliefs)
        GF2C_CUDA(cudaMemcpyAsync((char*)beliefs + lo, (char*)dec->s_bel.p + lo, ln, cudaMemcpyDeviceToHost, s));
    }
    GF2C_CUDA(cudaEventRecord(dec->pev_join, dec->pstream));
    GF2C_CUDA(cudaStreamWaitEvent(st, dec->pev_join, 0));
    dec->last_launches = launches;
    return check_status(dec, st);
  }
  GF2C_CUDA(cudaMemcpyAsync(dec->s_llr.p, llr, bl, cudaMemcpyHostToDevice, st));
  a.llr = (const float*)dec->s_llr.p;
  a.msg = msg_bits ? (uint64_t*)dec->s_msg.p : nullptr;
  a.iters = (int32_t*)dec->s_it.p;
  a.conv = (uint8_t*)dec->s_cv.p;
  a.synd_ok = (uint8_t*)dec->s_so.p;
  a.beliefs = beliefs ? (float*)dec->s_bel.p : nullptr;
  int extra = 0;
  if ((rc = key_order(dec, a, frames, st, 0, extra))) return rc;
  if ((rc = launch_decoder(dec, a, frames, st))) return rc;
  dec->last_launches += extra;
  if (msg_bits) GF2C_CUDA(cudaMemcpyAsync(msg_bits, dec->s_msg.p, bm, cudaMemcpyDeviceToHost, st));
  if (iterations) GF2C_CUDA(cudaMemcpyAsync(iterations, dec->s_it.p, frames * 4, cudaMemcpyDeviceToHost, st));
  if (converged) GF2C_CUDA(cudaMemcpyAsync(converged, dec->s_cv.p, frames, cudaMemcpyDeviceToHost, st));
  if (syndrome_ok) GF2C_CUDA(cudaMemcpyAsync(syndrome_ok, dec->s_so.p, frames, cudaMemcpyDeviceToHost, st));
  if (beliefs) GF2C_CUDA(cudaMemcpyAsync(beliefs, dec->s_bel.p, bl, cudaMemcpyDeviceToHost, st));
  return check_status(dec, st);
}

// The primary pass over `frames` frames whose arrays `a` points at, on stream
// `st` (slot: workspace and queue of the pipelined host path); `ordered`:
// hardest frames first (key_order).
static int primary_pass(gf2c_decoder* primary, DecodeArgs a, int64_t frames, int32_t max_iter_primary,
                        cudaStream_t st, int slot, int& launches, bool ordered = true) {
  int rc, extra = 0;
  a.max_iter = max_iter_primary;
  if (ordered && (rc = key_order(primary, a, frames, st, slot, extra))) return rc;
  if ((rc = launch_decoder(primary, a, frames, st, slot))) return rc;
  launches += 1 + extra;
  return GF2C_OK;
}
// The frames the primary pass left failing, listed on the device (the list
// goes to `list`, its length to *cnt), and the fallback decoder on them (the
// count read on the device), on stream `st`.
static int fallback_pass(gf2c_decoder* fallback, DecodeArgs a, int64_t frames, int32_t max_iter_primary,
                         int32_t max_iter_fallback, int64_t* list, long long* cnt, cudaStream_t st, int slot,
                         int& launches) {
  GF2C_CUDA(launch_failed_list(a.synd_ok, frames, list, cnt, st));
  a.max_iter = max_iter_fallback;
  a.order = list;
  a.frames_dev = cnt;
  a.iters_add = max_iter_primary;
  int rc = launch_decoder(fallback, a, frames, st, slot);
  if (rc) return rc;
  launches += 2;
  return GF2C_OK;
}
// Both passes on one stream.
static int fallback_passes(gf2c_decoder* primary, gf2c_decoder* fallback, DecodeArgs a, int64_t frames,
                           int32_t max_iter_primary, int32_t max_iter_fallback, int64_t* list, long long* cnt,
                           cudaStream_t st, int slot, int& launches) {
  int rc;
  launches = 0;
  if ((rc = primary_pass(primary, a, frames, max_iter_primary, st, slot, launches))) return rc;
  return fallback_pass(fallback, a, frames, max_iter_primary, max_iter_fallback, list, cnt, st, slot, launches);
}

// The fallback call's stream for the fallback passes of a pipelined host batch
// (the highest priority, so that the few frames of a fallback pass get SMs as
// soon as the primary passes free them) and its events; false where they
// cannot be had.
static bool fallback_stream_ready(gf2c_decoder* d) {
  if (!d->fstream) {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&d->fstream, cudaStreamNonBlocking, greatest) != cudaSuccess) {
      d->fstream = nullptr;
      cudaGetLastError();
      return false;
    }
  }
  for (cudaEvent_t* e : {&d->pev_prim, &d->pev_fjoin})
    if (!*e && cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) {
      *e = nullptr;
      cudaGetLastError();
      return false;
    }
  return true;
}

int gf2c_decode_batch_fallback(gf2c_decoder* primary, gf2c_decoder* fallback, const float* llr, int64_t frames,
                               int32_t max_iter_primary, int32_t max_iter_fallback, uint64_t* msg_bits,
                               int32_t* iterations, uint8_t* converged, uint8_t* syndrome_ok,
                               int64_t* fallback_count, int32_t mem, void* stream) {
  if (!primary || !fallback || frames < 0 || max_iter_primary < 0 || max_iter_fallback <= 0 || (frames > 0 && !llr))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  int rc = check_mem(mem);
  if (rc) return rc;
  if (primary->codes.size() != 1 || fallback->codes.size() != 1 ||
      primary->codes[0]->h->serial != fallback->codes[0]->h->serial)
    return set_error(GF2C_ERR_INVALID_ARG, "both decoders must decode the same single code");
  if (fallback->opts.schedule != GF2C_SCHED_LAYERED)
    return set_error(GF2C_ERR_UNSUPPORTED, "the fallback decoder must use the layered schedule");
  if (frames == 0) {
    if (fallback_count && mem == GF2C_MEM_HOST) *fallback_count = 0;
    return GF2C_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int launches = 0;
  if (mem == GF2C_MEM_DEVICE) {
    uint8_t* so = syndrome_ok;
    if (!so) {
      if ((rc = primary->s_so.ensure((size_t)frames))) return rc;
      so = (uint8_t*)primary->s_so.p;
    }
    if ((rc = primary->fb_list.ensure((size_t)frames * 8)) || (rc = primary->fb_count.ensure(64))) return rc;
    DecodeArgs a{};
    a.llr = llr;
    a.msg = msg_bits;
    a.iters = iterations;
    a.conv = converged;
    a.synd_ok = so;
    long long* cnt = (long long*)primary->fb_count.p;
    if ((rc = fallback_passes(primary, fallback, a, frames, max_iter_primary, max_iter_fallback,
                              (int64_t*)primary->fb_list.p, cnt, st, 0, launches)))
      return rc;
    if (fallback_count)
      GF2C_CUDA(cudaMemcpyAsync(fallback_count, cnt, sizeof(long long), cudaMemcpyDeviceToDevice, st));
    primary->last_launches = launches;
    return GF2C_OK;
  }
  // Host memory: the batch is staged in the primary decoder's buffers.  Large
  // batches go in chunks alternating between the caller's stream and a second
  // stream, as in gf2c_decode_batch, with the input copies issued back to back
  // on a copy stream, and only the last chunk decoded hardest frames first.
  // The fallback passes and output copies run on a third stream, one per group
  // of chunks (about eight groups), each after its chunks' primary passes
  // only, so that the primary passes follow one another without waiting for
  // the fallback passes (a few frames of up to max_iter_fallback iterations
  // each: a pass lasts about as long whatever its frame count, so fewer passes
  // finish sooner).  The fallback passes share the fallback decoder's first
  // workspace, one after another on that stream; every group has its own list
  // and count.  When the two decoders are one, each chunk's passes stay on its
  // own stream and workspace.
  const HostCode& h = *primary->codes[0]->h;
  const int wk = (int)((h.k + 63) / 64);
  const size_t bl = (size_t)frames * h.n * 4, bm = (size_t)frames * wk * 8;
  if ((rc = primary->s_llr.ensure(bl)) || (rc = primary->s_msg.ensure(bm)) ||
      (rc = primary->s_it.ensure((size_t)frames * 4)) || (rc = primary->s_cv.ensure((size_t)frames)) ||
      (rc = primary->s_so.ensure((size_t)frames)) || (rc = primary->fb_list.ensure((size_t)frames * 8)) ||
      (rc = primary->fb_count.ensure(64 * 8)))
    return rc;
  const int64_t wave = std::max(primary->grid, fallback->grid);
  const bool pipe = frames >= 3 * wave && bl >= ((size_t)64 << 20) && pipeline_ready(primary) &&
                    (fallback == primary || fallback_stream_ready(primary));
  const bool fsplit = pipe && fallback != primary;
  if (pipe) {
    GF2C_CUDA(cudaEventRecord(primary->pev_fork, st));
    GF2C_CUDA(cudaStreamWaitEvent(primary->pstream, primary->pev_fork, 0));
    GF2C_CUDA(cudaStreamWaitEvent(primary->cstream, primary->pev_fork, 0));
  }
  int chunks = 0, groups = 0;
  const int64_t csz = pipe ? even_chunk(frames, wave) : frames;
  const int gsz = fsplit ? (int)std::max<int64_t>(1, (frames / csz + 7) / 8) : 1;  // chunks per group
  for (int64_t f0 = 0, nf = 0, g0 = 0; f0 < frames; f0 += nf, chunks++) {
    nf = (chunks == 63) ? frames - f0 : chunk_frames(csz, frames - f0, wave);
    const int slot = pipe ? (chunks & 1) : 0;
    cudaStream_t s = slot ? primary->pstream : st;
    const size_t ln = (size_t)nf * h.n * 4, lo = (size_t)f0 * h.n * 4;
    const size_t mo = (size_t)f0 * wk * 8;
    // input copies back to back on the copy stream, each chunk's passes
    // waiting for its own copy only
    if (pipe) {
      GF2C_CUDA(cudaMemcpyAsync((char*)primary->s_llr.p + lo, (const char*)llr + lo, ln, cudaMemcpyHostToDevice,
                                primary->cstream));
      GF2C_CUDA(cudaEventRecord(primary->pev_copy[slot], primary->cstream));
      GF2C_CUDA(cudaStreamWaitEvent(s, primary->pev_copy[slot], 0));
    } else {
      GF2C_CUDA(cudaMemcpyAsync((char*)primary->s_llr.p + lo, (const char*)llr + lo, ln, cudaMemcpyHostToDevice, s));
    }
    DecodeArgs a{};
    a.llr = (const float*)((char*)primary->s_llr.p + lo);
    a.msg = msg_bits ? (uint64_t*)((char*)primary->s_msg.p + mo) : nullptr;
    a.iters = (int32_t*)primary->s_it.p + f0;
    a.conv = (uint8_t*)primary->s_cv.p + f0;
    a.synd_ok = (uint8_t*)primary->s_so.p + f0;
    if ((rc = primary_pass(primary, a, nf, max_iter_primary, s, slot, launches, f0 + nf == frames))) return rc;
    if (fsplit) {
      GF2C_CUDA(cudaEventRecord(primary->pev_prim, s));
      GF2C_CUDA(cudaStreamWaitEvent(primary->fstream, primary->pev_prim, 0));
      s = primary->fstream;
    }
    if (f0 + nf < frames && (chunks + 1) % gsz != 0) continue;
    // the group [g0, f0 + nf): fallback pass, then its outputs
    const int64_t gn = f0 + nf - g0;
    const size_t gmn = (size_t)gn * wk * 8, gmo = (size_t)g0 * wk * 8;
    DecodeArgs ga = a;
    ga.llr = (const float*)((char*)primary->s_llr.p + (size_t)g0 * h.n * 4);
    ga.msg = msg_bits ? (uint64_t*)((char*)primary->s_msg.p + gmo) : nullptr;
    ga.iters = (int32_t*)primary->s_it.p + g0;
    ga.conv = (uint8_t*)primary->s_cv.p + g0;
    ga.synd_ok = (uint8_t*)primary->s_so.p + g0;
    if ((rc = fallback_pass(fallback, ga, gn, max_iter_primary, max_iter_fallback, (int64_t*)primary->fb_list.p + g0,
                            (long long*)primary->fb_count.p + groups, s, fsplit ? 0 : slot, launches)))
      return rc;
    if (msg_bits)
      GF2C_CUDA(cudaMemcpyAsync((char*)msg_bits + gmo, (char*)primary->s_msg.p + gmo, gmn, cudaMemcpyDeviceToHost, s));
    if (iterations)
      GF2C_CUDA(cudaMemcpyAsync(iterations + g0, (int32_t*)primary->s_it.p + g0, gn * 4, cudaMemcpyDeviceToHost, s));
    if (converged)
      GF2C_CUDA(cudaMemcpyAsync(converged + g0, (uint8_t*)primary->s_cv.p + g0, gn, cudaMemcpyDeviceToHost, s));
    if (syndrome_ok)
      GF2C_CUDA(cudaMemcpyAsync(syndrome_ok + g0, (uint8_t*)primary->s_so.p + g0, gn, cudaMemcpyDeviceToHost, s));
    groups++;
    g0 = f0 + nf;
  }
  if (pipe) {
    GF2C_CUDA(cudaEventRecord(primary->pev_join, primary->pstream));
    GF2C_CUDA(cudaStreamWaitEvent(st, primary->pev_join, 0));
  }
  if (fsplit) {
    GF2C_CUDA(cudaEventRecord(primary->pev_fjoin, primary->fstream));
    GF2C_CUDA(cudaStreamWaitEvent(st, primary->pev_fjoin, 0));
  }
  long long counts[64] = {0};
  GF2C_CUDA(cudaMemcpyAsync(counts, primary->fb_count.p, sizeof(long long) * groups, cudaMemcpyDeviceToHost, st));
  primary->last_launches = launches;
  if ((rc = check_status(primary, st)) || (rc = check_status(fallback, st))) return rc;
  if (fallback_count) {
    long long total = 0;
    for (int c = 0; c < groups; c++) total += counts[c];
    *fallback_count = total;
  }
  return GF2C_OK;
}

int gf2c_decode_mixed(gf2c_decoder* dec, const float* llr, const int64_t* llr_offset, const int32_t* code_id,
                      const int32_t* max_iter, int64_t frames, uint64_t* msg_bits, const int64_t* msg_offset,
                      int32_t* iterations, uint8_t* converged, uint8_t* syndrome_ok, int32_t use_graph,
                      int32_t mem, void* stream) {
  if (!dec || frames < 0 || (frames > 0 && (!llr || !llr_offset || !code_id || !max_iter)))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (msg_bits && !msg_offset) return set_error(GF2C_ERR_INVALID_ARG, "msg_bits needs msg_offset");
  int rc = check_mem(mem);
  if (rc || frames == 0) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  DecodeArgs a{};
  // Frames of a mixed batch are taken code by code (the ordering kernel runs
  // before the decode, in the same stream or graph).  A larger order buffer
  // invalidates the graphs that captured the old one.
  const bool ordered = dec->codes.size() > 1;
  if (ordered) {
    void* before = dec->d_order.p;
    if ((rc = dec->d_order.ensure((size_t)frames * 8))) return rc;
    if (dec->d_order.p != before && !dec->graphs.empty()) {
      if (dec->gstream) GF2C_CUDA(cudaStreamSynchronize(dec->gstream));
      for (auto& kv : dec->graphs) cudaGraphExecDestroy(kv.second);
      dec->graphs.clear();
    }
    a.order = (const int64_t*)dec->d_order.p;
  }
  auto order_then_decode = [&](cudaStream_t s) -> int {
    if (ordered)
      GF2C_CUDA(launch_mixed_order(a.code_id, frames, (const int32_t*)dec->d_rank.p, (int)dec->codes.size(),
                                   (int64_t*)dec->d_order.p, s));
    int r = launch_decoder(dec, a, frames, s);
    if (!r && ordered) dec->last_launches = 2;
    return r;
  };
  if (mem == GF2C_MEM_DEVICE) {
    a.llr = llr;
    a.llr_off = llr_offset;
    a.code_id = code_id;
    a.max_iter_arr = max_iter;
    a.msg = msg_bits;
    a.msg_off = msg_offset;
    a.iters = iterations;
    a.conv = converged;
    a.synd_ok = syndrome_ok;
    if (!use_graph) return order_then_decode(st);
    GraphKey key;
    key.v = {(uintptr_t)llr, (uintptr_t)llr_offset, (uintptr_t)code_id, (uintptr_t)max_iter,
             (uintptr_t)msg_bits, (uintptr_t)msg_offset, (uintptr_t)iterations, (uintptr_t)converged,
             (uintptr_t)syndrome_ok, (uintptr_t)frames};
    // Graphs are captured and replayed on the decoder's own stream, ordered
    // after / before the caller's stream with events (the legacy default
    // stream cannot be captured).
    if (!dec->gstream) {
      GF2C_CUDA(cudaStreamCreateWithFlags(&dec->gstream, cudaStreamNonBlocking));
      GF2C_CUDA(cudaEventCreateWithFlags(&dec->ev_in, cudaEventDisableTiming));
      GF2C_CUDA(cudaEventCreateWithFlags(&dec->ev_out, cudaEventDisableTiming));
    }
    cudaStream_t gs = dec->gstream;
    auto it = dec->graphs.find(key);
    if (it == dec->graphs.end()) {
      cudaGraph_t g;
      GF2C_CUDA(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
      rc = order_then_decode(gs);
      cudaError_t e = cudaStreamEndCapture(gs, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
      it = dec->graphs.emplace(key, ex).first;
    }
    GF2C_CUDA(cudaEventRecord(dec->ev_in, st));
    GF2C_CUDA(cudaStreamWaitEvent(gs, dec->ev_in, 0));
    GF2C_CUDA(cudaGraphLaunch(it->second, gs));
    GF2C_CUDA(cudaEventRecord(dec->ev_out, gs));
    GF2C_CUDA(cudaStreamWaitEvent(st, dec->ev_out, 0));
    dec->last_launches = ordered ? 2 : 1;
    return GF2C_OK;
  }
  // host memory: validate ids and offsets, stage everything
  int64_t llr_total = 0, msg_total = 0;
  for (int64_t f = 0; f < frames; f++) {
    int c = code_id[f];
    if (c < 0 || c >= (int)dec->codes.size()) return set_error(GF2C_ERR_INVALID_ARG, "code_id out of range");
    if (max_iter[f] < 0 || llr_offset[f] < 0 || (msg_bits && msg_offset[f] < 0))
      return set_error(GF2C_ERR_INVALID_ARG, "negative offset or max_iter");
    const HostCode& h = *dec->codes[c]->h;
    llr_total = std::max<int64_t>(llr_total, llr_offset[f] + h.n);
    if (msg_bits) msg_total = std::max<int64_t>(msg_total, msg_offset[f] + (h.k + 63) / 64);
  }
  if ((rc = dec->s_llr.ensure(llr_total * 4)) || (rc = dec->s_msg.ensure(std::max<int64_t>(msg_total, 1) * 8)) ||
      (rc = dec->s_it.ensure(frames * 4)) || (rc = dec->s_cv.ensure(frames)) || (rc = dec->s_so.ensure(frames)) ||
      (rc = dec->s_off1.ensure(frames * 8)) || (rc = dec->s_off2.ensure(frames * 8)) ||
      (rc = dec->s_cid.ensure(frames * 4)) || (rc = dec->s_mit.ensure(frames * 4)))
    return rc;
  // Large batches: chunks of frames in memory order, each chunk's LLRs brought
  // in by the copy stream while earlier chunks decode on two streams (as in
  // gf2c_decode_batch).  The frame order of a chunk (code by code, longest
  // codes first, then by frame index, the ordering kernel's rule) is made on
  // the host; the persistent kernel takes the chunk's frames from it.
  const int64_t wave = dec->grid;
  if (ordered && frames >= 3 * wave && (size_t)llr_total * 4 >= ((size_t)64 << 20) && pipeline_ready(dec) &&
      dec->s_cnt.ensure(64 * 8) == GF2C_OK) {
    std::vector<int64_t> mem((size_t)frames), ord((size_t)frames);
    for (int64_t f = 0; f < frames; f++) mem[f] = f;
    std::stable_sort(mem.begin(), mem.end(), [&](int64_t x, int64_t y) { return llr_offset[x] < llr_offset[y]; });
    std::vector<long long> cnt;
    std::vector<std::pair<int64_t, int64_t>> copy;  // LLR element range each chunk brings in
    const int64_t cap = chunk_cap(frames, wave);
    int64_t copied = 0;
    for (int64_t p0 = 0, nf = 0, want = wave; p0 < frames; p0 += nf, want = std::min(2 * want, cap)) {
      nf = (cnt.size() == 63) ? frames - p0 : chunk_frames(want, frames - p0, wave);
      int64_t hi = 0;
      for (int64_t p = p0; p < p0 + nf; p++) hi = std::max<int64_t>(hi, llr_offset[mem[p]] + dec->codes[code_id[mem[p]]]->h->n);
      const int64_t lo = std::max<int64_t>(llr_offset[mem[p0]], copied);
      copy.emplace_back(lo, std::max(hi, lo));
      copied = std::max(copied, hi);
      std::copy(mem.begin() + p0, mem.begin() + p0 + nf, ord.begin() + p0);
      std::stable_sort(ord.begin() + p0, ord.begin() + p0 + nf, [&](int64_t x, int64_t y) {
        const int rx = dec->h_rank[code_id[x]], ry = dec->h_rank[code_id[y]];
        return rx != ry ? rx < ry : x < y;
      });
      cnt.push_back(nf);
    }
    GF2C_CUDA(cudaEventRecord(dec->pev_fork, st));
    GF2C_CUDA(cudaStreamWaitEvent(dec->pstream, dec->pev_fork, 0));
    GF2C_CUDA(cudaStreamWaitEvent(dec->cstream, dec->pev_fork, 0));
    cudaStream_t cs = dec->cstream;
    GF2C_CUDA(cudaMemcpyAsync(dec->d_order.p, ord.data(), frames * 8, cudaMemcpyHostToDevice, cs));
    GF2C_CUDA(cudaMemcpyAsync(dec->s_cnt.p, cnt.data(), cnt.size() * 8, cudaMemcpyHostToDevice, cs));
    GF2C_CUDA(cudaMemcpyAsync(dec->s_off1.p, llr_offset, frames * 8, cudaMemcpyHostToDevice, cs));
    if (msg_bits) GF2C_CUDA(cudaMemcpyAsync(dec->s_off2.p, msg_offset, frames * 8, cudaMemcpyHostToDevice, cs));
    GF2C_CUDA(cudaMemcpyAsync(dec->s_cid.p, code_id, frames * 4, cudaMemcpyHostToDevice, cs));
    GF2C_CUDA(cudaMemcpyAsync(dec->s_mit.p, max_iter, frames * 4, cudaMemcpyHostToDevice, cs));
    a.llr = (const float*)dec->s_llr.p;
    a.llr_off = (const int64_t*)dec->s_off1.p;
    a.code_id = (const int32_t*)dec->s_cid.p;
    a.max_iter_arr = (const int32_t*)dec->s_mit.p;
    a.msg = msg_bits ? (uint64_t*)dec->s_msg.p : nullptr;
    a.msg_off = msg_bits ? (const int64_t*)dec->s_off2.p : nullptr;
    a.iters = (int32_t*)dec->s_it.p;
    a.conv = (uint8_t*)dec->s_cv.p;
    a.synd_ok = (uint8_t*)dec->s_so.p;
    int launches = 0;
    for (size_t c = 0, p0 = 0; c < cnt.size(); p0 += (size_t)cnt[c], c++) {
      const int slot = (int)(c & 1);
      cudaStream_t s = slot ? dec->pstream : st;
      const int64_t lo = copy[c].first, n = copy[c].second - copy[c].first;
      if (n > 0)
        GF2C_CUDA(cudaMemcpyAsync((float*)dec->s_llr.p + lo, llr + lo, (size_t)n * 4, cudaMemcpyHostToDevice, cs));
      GF2C_CUDA(cudaEventRecord(dec->pev_copy[slot], cs));
      GF2C_CUDA(cudaStreamWaitEvent(s, dec->pev_copy[slot], 0));
      DecodeArgs b = a;
      b.order = (const int64_t*)dec->d_order.p + p0;
      b.frames_dev = (const long long*)dec->s_cnt.p + c;
      if ((rc = launch_decoder(dec, b, frames, s, slot))) return rc;
      launches++;
    }
    GF2C_CUDA(cudaEventRecord(dec->pev_join, dec->pstream));
    GF2C_CUDA(cudaStreamWaitEvent(st, dec->pev_join, 0));
    dec->last_launches = launches;
    if (msg_bits) GF2C_CUDA(cudaMemcpyAsync(msg_bits, dec->s_msg.p, msg_total * 8, cudaMemcpyDeviceToHost, st));
    if (iterations) GF2C_CUDA(cudaMemcpyAsync(iterations, dec->s_it.p, frames * 4, cudaMemcpyDeviceToHost, st));
    if (converged) GF2C_CUDA(cudaMemcpyAsync(converged, dec->s_cv.p, frames, cudaMemcpyDeviceToHost, st));
    if (syndrome_ok) GF2C_CUDA(cudaMemcpyAsync(syndrome_ok, dec->s_so.p, frames, cudaMemcpyDeviceToHost, st));
    return check_status(dec, st);
  }
  GF2C_CUDA(cudaMemcpyAsync(dec->s_llr.p, llr, llr_total * 4, cudaMemcpyHostToDevice, st));
  GF2C_CUDA(cudaMemcpyAsync(dec->s_off1.p, llr_offset, frames * 8, cudaMemcpyHostToDevice, st));
  if (msg_bits) GF2C_CUDA(cudaMemcpyAsync(dec->s_off2.p, msg_offset, frames * 8, cudaMemcpyHostToDevice, st));
  GF2C_CUDA(cudaMemcpyAsync(dec->s_cid.p, code_id, frames * 4, cudaMemcpyHostToDevice, st));
  GF2C_CUDA(cudaMemcpyAsync(dec->s_mit.p, max_iter, frames * 4, cudaMemcpyHostToDevice, st));
  a.llr = (const float*)dec->s_llr.p;
  a.llr_off = (const int64_t*)dec->s_off1.p;
  a.code_id = (const int32_t*)dec->s_cid.p;
  a.max_iter_arr = (const int32_t*)dec->s_mit.p;
  a.msg = msg_bits ? (uint64_t*)dec->s_msg.p : nullptr;
  a.msg_off = msg_bits ? (const int64_t*)dec->s_off2.p : nullptr;
  a.iters = (int32_t*)dec->s_it.p;
  a.conv = (uint8_t*)dec->s_cv.p;
  a.synd_ok = (uint8_t*)dec->s_so.p;
  if ((rc = order_then_decode(st))) return rc;
  if (msg_bits) GF2C_CUDA(cudaMemcpyAsync(msg_bits, dec->s_msg.p, msg_total * 8, cudaMemcpyDeviceToHost, st));
  if (iterations) GF2C_CUDA(cudaMemcpyAsync(iterations, dec->s_it.p, frames * 4, cudaMemcpyDeviceToHost, st));
  if (converged) GF2C_CUDA(cudaMemcpyAsync(converged, dec->s_cv.p, frames, cudaMemcpyDeviceToHost, st));
  if (syndrome_ok) GF2C_CUDA(cudaMemcpyAsync(syndrome_ok, dec->s_so.p, frames, cudaMemcpyDeviceToHost, st));
  return check_status(dec, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// learned normalised / offset min-sum trainer
// ---------------------------------------------------------------------------
struct gf2c_nms_trainer {
  const gf2c_code* code = nullptr;
  int T = 0, L = 1;
  int schedule = GF2C_SCHED_FLOODING;
  int64_t max_frames = 0;
  int grid = 0;
  long long work_stride = 0;
  DevBuf dcode, X, B, work, pf;  // pf: per-frame gradients and loss, [frames][2 T L + 1]
};

extern "C" {

int gf2c_nms_trainer_create(const gf2c_code* code, int32_t iterations, int64_t max_frames, gf2c_nms_trainer** out) {
  if (!code || !out || iterations <= 0 || iterations > 64 || max_frames <= 0)
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  *out = nullptr;
  const HostCode& h = *code->h;
  if (h.max_dc > 32) return set_error(GF2C_ERR_UNSUPPORTED, "learned decoder: check degree above 32");
  std::unique_ptr<gf2c_nms_trainer> tr(new (std::nothrow) gf2c_nms_trainer());
  if (!tr) return set_error(GF2C_ERR_NOMEM, "out of host memory");
  tr->code = code;
  tr->T = iterations;
  tr->L = h.layered_ok ? (int)h.cg.size() : 1;
  tr->max_frames = max_frames;
  int rc = code_dev_struct(code, tr->dcode);
  if (rc) return rc;
  const size_t E = (size_t)h.e_slots;
  if ((rc = tr->X.ensure(sizeof(float) * E * iterations * (size_t)max_frames))) return rc;
  if ((rc = tr->B.ensure(sizeof(float) * (size_t)h.n * (size_t)max_frames))) return rc;
  int dev = 0, sms = 148;
  GF2C_CUDA(cudaGetDevice(&dev));
  GF2C_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  tr->grid = (int)std::min<int64_t>(max_frames, (int64_t)sms * 4);
  tr->work_stride = (long long)(((E + 63) & ~(size_t)63) + (((size_t)h.n + 63) & ~(size_t)63) + 2 * (size_t)h.m + 64) * 4;
  if ((rc = tr->work.ensure((size_t)tr->work_stride * tr->grid))) return rc;
  if ((rc = tr->pf.ensure(sizeof(float) * (size_t)max_frames * (2 * (size_t)iterations * tr->L + 1)))) return rc;
  *out = tr.release();
  return GF2C_OK;
}

int gf2c_nms_trainer_destroy(gf2c_nms_trainer* tr) {
  delete tr;
  return GF2C_OK;
}

int gf2c_nms_trainer_layers(const gf2c_nms_trainer* tr, int32_t* layers) {
  if (!tr || !layers) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  *layers = tr->L;
  return GF2C_OK;
}

int gf2c_nms_trainer_set_schedule(gf2c_nms_trainer* tr, int32_t schedule) {
  if (!tr || (schedule != GF2C_SCHED_FLOODING && schedule != GF2C_SCHED_LAYERED))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  const HostCode& h = *tr->code->h;
  if (schedule == GF2C_SCHED_LAYERED && (!h.layered_ok || h.max_nchk > 1024))
    return set_error(GF2C_ERR_UNSUPPORTED, "layered training needs a QC or DVB-T2 code with Z <= 1024");
  tr->schedule = schedule;
  return GF2C_OK;
}

int gf2c_nms_loss_grad(gf2c_nms_trainer* tr, const float* llr, const uint64_t* cw_bits, int64_t frames,
                       const float* alpha, const float* beta, float* grad_alpha, float* grad_beta, float* loss,
                       float* soft_out, void* stream) {
  if (!tr || frames <= 0 || frames > tr->max_frames || !llr || !cw_bits || !alpha || !beta || !grad_alpha ||
      !grad_beta || !loss)
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments (frames must be in [1, max_frames])");
  cudaStream_t st = (cudaStream_t)stream;
  const DevCode& h = tr->code->h->dev;
  const int grid = (int)std::min<int64_t>(tr->grid, frames);
  float* B = soft_out ? soft_out : (float*)tr->B.p;
  if (tr->schedule == GF2C_SCHED_LAYERED)
    return launch_nms_layered((const DevCode*)tr->dcode.p, h, tr->T, tr->L, llr, cw_bits, frames, alpha, beta,
                              (float*)tr->X.p, B, (char*)tr->work.p, tr->work_stride, grid, (float*)tr->pf.p,
                              grad_alpha, grad_beta, loss, st);
  int rc = launch_nms_forward((const DevCode*)tr->dcode.p, h, tr->T, tr->L, llr, cw_bits, frames, alpha, beta,
                              (float*)tr->X.p, B, (char*)tr->work.p, tr->work_stride, grid, (float*)tr->pf.p, st);
  if (rc) return rc;
  return launch_nms_backward((const DevCode*)tr->dcode.p, h, tr->T, tr->L, llr, cw_bits, frames, alpha, beta,
                             (const float*)tr->X.p, B, (char*)tr->work.p, tr->work_stride, grid, (float*)tr->pf.p,
                             grad_alpha, grad_beta, loss, st);
}

int gf2c_count_errors(const uint64_t* ref_bits, const uint64_t* test_bits, int64_t frames, int32_t words,
                      int32_t* bit_errors, uint64_t* totals, void* stream) {
  if (frames < 0 || words <= 0 || (frames > 0 && (!ref_bits || !test_bits || !totals)))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  return launch_count_errors(ref_bits, test_bits, frames, words, bit_errors, (unsigned long long*)totals,
                             (cudaStream_t)stream);
}

int gf2c_adam_step(float* params, const float* grads, float* m, float* v, int64_t count, float lr, float beta1,
                   float beta2, float eps, int32_t step, float lo, float hi, void* stream) {
  if (!params || !grads || !m || !v || count <= 0 || count > (1 << 30) || step < 1 || !(lo <= hi))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  return launch_adam(params, grads, m, v, (int)count, lr, beta1, beta2, eps, step, lo, hi, (cudaStream_t)stream);
}

}  // extern "C"
