// gf2cuda internal declarations: host code graph, device layout, kernel args.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gf2cuda.h"

namespace gf2c {

// ---------------------------------------------------------------------------
// Device-side description of one code ("check groups" x "slots").
//
// Check nodes are grouped into check groups (CG).  For QC / DVB-T2 codes a CG
// is one row group of Z checks (the layer of the layered schedule); for other
// codes a CG is a run of up to 256 consecutive checks.  Inside a CG every check
// has the same number of slots dc (shorter rows are padded with var = -1), and
// the c2v message of slot i of check t lives at edge slot edge0 + i*nchk + t,
// so a warp of consecutive checks touches consecutive message addresses.
//
// Variable nodes are grouped into var groups (VG) of vgs consecutive variables;
// vg_slot lists, for slot i of variable j, the edge slot of its i-th edge in
// ascending ORIGINAL check order (the reference's summation order), -1 = pad.
// ---------------------------------------------------------------------------
struct DevCode {
  int n, m, k;
  int ncg, nvg, vgs;
  int e_slots;
  int max_dc, max_dv;
  int words_k, words_n, words_m;   // ceil(x/64)
  int layered_ok;                  // CGs are layers usable by the layered schedule
  int lay_bucket;                  // slot count of the layered kernel that fits this code exactly
  int max_nchk;                    // largest CG
  const int4* cg;                  // {chk_begin, nchk, dc, edge0}
  const uint32_t* cg_sync;         // layered: bit i = barrier after slot i (dup variables)
  const int* slot_var;             // [e_slots]
  const uint16_t* chk_cg;          // [m] flattened check -> CG
  const int2* vg;                  // {dv, vedge0}
  const int* vg_slot;              // VG-major, [vg][i][j]
  const int* vg_chk;               // same layout: flattened check index of the edge
  const int* vg_ci;                // same layout: flattened check | slot << 24
  // QC / DVB-T2 codes: slot i of check group g is described by slot_desc[edge0/Z + i]
  // (all Z checks of a row group share it), packed as base | shift_or_q << 20 | type << 30:
  //   type 0 circulant:   var = base + (t + shift) mod Z
  //   type 1 staircase sub-diagonal: var = base + q t - 1, absent for (row group 0, t 0)
  //   type 2 staircase diagonal:     var = base + q t
  const uint32_t* slot_desc;       // nullptr for codes without the QC structure
  const int* cg_ninfo;             // per CG: number of circulant slots (the rest are staircase)
  int z;                           // circulant size of slot_desc codes
  // Check-state flooding kernel (state_flood.cu).  Variables are stored in a
  // "u order": the identity, except for DVB-T2 codes whose parity bit
  // k + a + q t is stored at k + a Z + t, which makes every slot of every row
  // group a contiguous (rotated) run of Z posteriors.
  const int4* sp_cg;               // per CG {chk_begin, nchk, dc, desc offset (structured) | edge0}
  const int2* sp_desc;             // u-order slot descriptors {start, wrap}: check t reads variable
                                   // start + t - (t >= wrap ? nchk : 0) (nullptr: u order is the
                                   // identity and slot_var is used)
  const uint32_t* sp_absent;       // per CG: slots without an edge at check t = 0 (staircase corner)
  const int2* sp_cchunk;           // check chunks {CG, first check in CG}: 32 checks of one CG
  int sp_ncchunk;
  const int2* sp_vg;               // per u-order var group of vgs variables {dv, offset into sp_ci}
  const int* sp_ci;                // [offset + i * vgs + j]: flattened check | slot << 24 of edge i,
                                   // ascending original check index; -1 = pad
  const int2* sp_vchunk;           // var chunks {var group, first j}: 32 variables of one group
  int sp_nvchunk;
  const int* sp_u2v;               // natural index of u-order variable u (nullptr: identity)
  const int* csr_ptr;              // natural order H (m + 1)
  const int* csr_idx;              // (nnz)
  // encoder
  int enc_kind;                    // 0 = DVB-T2 accumulator, 1 = dense generator
  const uint64_t* enc_p;           // kind 1: k rows of words_m words (parity j of row i)
  const int* enc_msg_cols;         // kind 1: k message columns
  const int* enc_par_cols;         // kind 1: m parity columns
  int enc_q;                       // kind 0: row groups (m / 360)
  const int* enc_rg_ptr;           // kind 0: q + 1 offsets into enc_rg_ent
  const int* enc_rg_ent;           // kind 0: info block b << 16 | rotation tau, per row group
};

uint64_t next_code_serial();

// Host-side code (reference-exact sparse structure + device layout plan).
struct HostCode {
  uint64_t serial = next_code_serial();    // unique per code object in the process
  int64_t n = 0, m = 0, k = 0;
  std::vector<int64_t> row_ptr, row_idx;   // CSR, columns ascending (sparse.rs:166-203)
  std::vector<int64_t> col_ptr, col_idx;   // CSC, rows ascending (sparse.rs:297-328)
  std::vector<int64_t> col_edge;           // CSC slot -> CSR edge
  int kind = 0;                            // 0 edges, 1 QC, 2 DVB-T2
  int z = 0, q = 0;
  int dvb_index = -1;
  std::vector<int32_t> qc_base;            // QC: mb x nb
  int mb = 0, nb = 0;

  // layout plan
  std::vector<int4> cg;
  std::vector<uint32_t> cg_sync;
  std::vector<int> slot_var;
  std::vector<uint16_t> chk_cg;
  std::vector<int2> vg;
  std::vector<int> vg_slot;
  std::vector<int> vg_chk;
  std::vector<int> vg_ci;
  std::vector<uint32_t> slot_desc;         // QC / DVB-T2 slot descriptors (see DevCode)
  std::vector<int> cg_ninfo;               // circulant slots per CG
  int vgs = 0, max_dc = 0, max_dv = 0, e_slots = 0, layered_ok = 0, max_nchk = 0;
  std::vector<int64_t> cg_checks;          // original check of each flattened check
  // check-state flooding plan (see DevCode)
  std::vector<int4> sp_cg;
  std::vector<int2> sp_desc;
  std::vector<uint32_t> sp_absent;
  std::vector<int2> sp_cchunk, sp_vchunk, sp_vg;
  std::vector<int> sp_ci, sp_u2v;

  // encoder (generic)
  int enc_kind = 0;
  bool enc_ready = false;
  int enc_status = GF2C_OK;
  std::vector<uint64_t> enc_p;
  std::vector<int> enc_msg_cols, enc_par_cols;
  std::vector<int> enc_rg_ptr, enc_rg_ent;  // DVB-T2: per row group a, (block, rotation) of its info addresses

  // device copy (lazily uploaded per device)
  std::mutex dev_mu;
  int dev_id = -1;
  DevCode dev{};
  std::vector<void*> dev_allocs;
  ~HostCode();
};

struct KernelShape {
  int threads = 0;
  int blocks_per_sm = 0;
};

}  // namespace gf2c

struct gf2c_code {
  std::unique_ptr<gf2c::HostCode> h;
};

namespace gf2c {

// error helpers
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
#define GF2C_CUDA(call)                                        \
  do {                                                          \
    cudaError_t _e = (call);                                    \
    if (_e != cudaSuccess) return ::gf2c::cuda_error(_e, #call); \
  } while (0)

// host code construction (code_host.cpp)
int build_dvbt2(int frame, int rate, HostCode& c);
int build_qc(const int32_t* base, int mb, int nb, int z, HostCode& c);
int build_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count, HostCode& c);
void plan_state(HostCode& c);  // the check-state flooding plan (after the CG / VG plan)
int prepare_encoder(HostCode& c);
int upload_code(HostCode& c);  // uploads the device layout on the current device

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------
struct DecodeArgs {
  const DevCode* codes;            // device array of ncodes
  int ncodes;
  const float* llr;
  const int64_t* llr_off;          // nullable: frame f at f * n
  const int32_t* code_id;          // nullable: code 0
  const int64_t* order;            // nullable: the queue's q-th frame is order[q] (mixed batches grouped by code)
  const int32_t* max_iter_arr;     // nullable: max_iter for all
  int max_iter;
  uint64_t* msg;
  const int64_t* msg_off;          // nullable: frame f at f * words_k
  int32_t* iters;
  uint8_t* conv;
  uint8_t* synd_ok;
  float* beliefs;                  // nullable
  long long frames;
  const long long* frames_dev;     // nullable: number of queue entries (order[0..*frames_dev)) in device
                                   // memory; frames then only bounds the frame indices
  int iters_add;                   // added to every reported iteration count
  unsigned long long* queue;       // work counter, zero at launch
  char* work;                      // per-CTA workspace
  long long work_stride;           // bytes per CTA
  long long app_offset;            // offset of the global APP inside a CTA workspace
  int smem_app_floats;             // APP kept in shared memory when n <= this
  int bitmap_words;                // 32-bit words of the hard-decision bitmap
  int lay_dbuf_off, lay_dbuf_floats;  // layered fused rows: shared-memory buffer of slots x checks
  int lay_stage_off, lay_stage_bytes; // layered, TMA-staged messages: two buffers of one row group's
                                      // messages, then two mbarriers (byte offset in dynamic smem)
  const float* alpha;              // NMS weights [nms_iters][nms_L]
  const float* beta;
  int nms_iters;
  int nms_L;
  int early_stop;
  int* status;                     // kernel-side error flag
  // check-state flooding kernel: byte offset of the posteriors in shared memory
  // (frame state on chip) and the offsets in the CTA workspace of the u-order
  // LLRs, the check states and the posteriors (frame state in the workspace)
  int sf_msg16;
  int sf_app_soff;
  long long sf_llr_off, sf_st_off, sf_app_off;
};

const void* flood_kernel_ptr(int algo, int msg16, int dcmax, int threads = 512);
// Frame order of a mixed batch (one CTA): frames grouped by rank_of[code id],
// ascending rank, ids outside [0, ncodes) last; ascending frame index within a group.
cudaError_t launch_mixed_order(const int32_t* code_id, int64_t frames, const int32_t* rank_of, int ncodes,
                               int64_t* order, cudaStream_t st);
// Frame order of a single-code batch, hardest frames first: ascending sum of
// |LLR| per frame (ties by frame index).  frames <= kKeyOrderMax; key: frames floats.
constexpr int kKeyOrderMax = 16384;
cudaError_t launch_key_order(const float* llr, int n, int64_t frames, float* key, int64_t* order, cudaStream_t st);
// Frames whose syndrome check failed (syndrome_ok[f] == 0), ascending, into
// list; their number into *count (one CTA, device memory only).
cudaError_t launch_failed_list(const uint8_t* syndrome_ok, int64_t frames, int64_t* list, long long* count,
                               cudaStream_t st);
int state_dcmax_bucket(int max_dc);
int state_flood_threads();
const void* state_flood_kernel_ptr(int dcmax, bool all_smem);
int decode_dcmax_bucket(int max_dc);
int layered_dcmax_bucket(int max_dc);
// bps: requested CTAs per SM (0 = any); 192 threads with 5 or more picks the 64-register build
const void* layered_kernel_ptr(int algo, int msg16, int dcmax, int maxt, bool stage = false, int bps = 0);
size_t layered_smem_bytes(int smem_app_floats, int bitmap_words);
// Layered min-sum / normalised-offset min-sum on the single-code (staged)
// kernels with the fused row paths: one compressed state per check (8 bytes
// for binary16 messages, 16 for FP32) replaces the per-edge messages, and
// nothing is staged in shared memory.
__host__ __device__ constexpr bool layered_state_mode(int algo, int dcmax, bool staged) {
  return (algo == GF2C_ALGO_MINSUM || algo == GF2C_ALGO_NMS) && staged && dcmax > 0 && dcmax <= 22;
}
size_t decode_smem_bytes(int smem_app_floats, int bitmap_words);

int launch_nms_forward(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                       long long frames, const float* alpha, const float* beta, float* X, float* B, char* work,
                       long long work_stride, int grid, float* pf, cudaStream_t st);
int launch_nms_backward(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                        long long frames, const float* alpha, const float* beta, const float* X, const float* B,
                        char* work, long long work_stride, int grid, float* pf, float* ga, float* gb,
                        float* loss, cudaStream_t st);
int launch_nms_layered(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                       long long frames, const float* alpha, const float* beta, float* X, float* B, char* work,
                       long long work_stride, int grid, float* pf, float* ga, float* gb, float* loss,
                       cudaStream_t st);
int launch_count_errors(const uint64_t* a, const uint64_t* b, long long frames, int words, int32_t* per_frame,
                        unsigned long long* totals, cudaStream_t st);
int launch_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2, float eps,
                int step, float lo, float hi, cudaStream_t st);

int launch_syndrome(const DevCode* dcode, const DevCode& hcode, const uint64_t* cw, long long frames,
                    uint64_t* synd, int32_t* weight, cudaStream_t st);
int launch_encode(const DevCode* dcode, const DevCode& hcode, const uint64_t* msg, long long frames,
                  uint64_t* cw, cudaStream_t st);
int launch_channel(const DevCode* dcode, const DevCode& hcode, uint64_t seed, uint64_t frame0,
                   long long frames, const double* sigma2, uint64_t* info, uint64_t* cw, float* llr,
                   cudaStream_t st);

}  // namespace gf2c
