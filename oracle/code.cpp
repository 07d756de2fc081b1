// CPU oracle: LDPC code construction (test infrastructure only).
//
// Restates, from erankavija/gf2:
//   * DvbParams::for_code            crates/gf2-coding/src/ldpc/dvb_t2/params.rs:56-85
//   * build_dvb_edges                crates/gf2-coding/src/ldpc/dvb_t2/builder.rs:74-118
//   * SpBitMatrix::from_coo          crates/gf2-core/src/sparse.rs:166-203 (sort + XOR dedup)
//   * SpBitMatrix::transpose         crates/gf2-core/src/sparse.rs:297-328 (stable CSC)
//   * QuasiCyclicLdpc::to_edges      crates/gf2-coding/src/ldpc/core.rs:578-605
//   * CirculantMatrix::to_edges      crates/gf2-coding/src/ldpc/core.rs:436-447
//   * LdpcCode::{k, syndrome}        crates/gf2-coding/src/ldpc/core.rs:116-138
#include "oracle_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "../gf2_b200/csrc/dvbt2_tables.h"

static thread_local std::string g_err;
void or_set_error(const std::string& s) { g_err = s; }
extern "C" const char* or_last_error(void) { return g_err.c_str(); }

static void finish_code(or_code* c, const std::vector<std::pair<int64_t, int64_t>>& edges) {
  // from_coo: collect per row, sort, keep columns with odd multiplicity.
  std::vector<std::vector<int64_t>> per_row(c->m);
  for (auto& e : edges) per_row[e.first].push_back(e.second);
  c->row_ptr.assign(1, 0);
  c->row_idx.clear();
  for (auto& row : per_row) {
    std::sort(row.begin(), row.end());
    size_t i = 0;
    while (i < row.size()) {
      size_t cnt = 1;
      while (i + cnt < row.size() && row[i + cnt] == row[i]) cnt++;
      if (cnt & 1) c->row_idx.push_back(row[i]);
      i += cnt;
    }
    c->row_ptr.push_back((int64_t)c->row_idx.size());
  }
  // transpose: stable scatter by row -> CSC with ascending check index.
  std::vector<int64_t> cnt(c->n + 1, 0);
  for (int64_t v : c->row_idx) cnt[v + 1]++;
  c->col_ptr.assign(c->n + 1, 0);
  for (int64_t v = 0; v < c->n; v++) c->col_ptr[v + 1] = c->col_ptr[v] + cnt[v + 1];
  c->col_idx.assign(c->row_idx.size(), 0);
  c->col_edge.assign(c->row_idx.size(), 0);
  std::vector<int64_t> next(c->col_ptr.begin(), c->col_ptr.end() - 1);
  for (int64_t r = 0; r < c->m; r++)
    for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) {
      int64_t v = c->row_idx[e];
      c->col_idx[next[v]] = r;
      c->col_edge[next[v]] = e;  // CSC slot -> CSR edge id
      next[v]++;
    }
  c->k = c->n > c->m ? c->n - c->m : 0;
  c->slot_order.resize(c->row_idx.size());
  for (int64_t r = 0; r < c->m; r++)
    for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++)
      c->slot_order[e] = (int32_t)(e - c->row_ptr[r]);
}

extern "C" or_code* or_code_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count) {
  if (m < 0 || n < 0) { or_set_error("negative dimensions"); return nullptr; }
  std::vector<std::pair<int64_t, int64_t>> edges;
  edges.reserve(count);
  for (int64_t i = 0; i < count; i++) {
    int64_t r = pairs[2 * i], col = pairs[2 * i + 1];
    if (r < 0 || r >= m || col < 0 || col >= n) {
      or_set_error("edge index out of bounds");
      return nullptr;
    }
    edges.push_back({r, col});
  }
  or_code* c = new or_code();
  c->m = m;
  c->n = n;
  finish_code(c, edges);
  c->edge_key.assign(c->row_idx.size(), 0);
  return c;
}

extern "C" or_code* or_code_qc(const int32_t* base, int mb, int nb, int z) {
  if (mb <= 0 || nb <= 0) { or_set_error("base matrix must be non-empty"); return nullptr; }
  if (z <= 0) { or_set_error("expansion factor must be positive"); return nullptr; }
  std::vector<std::pair<int64_t, int64_t>> edges;
  for (int r = 0; r < mb; r++)
    for (int cb = 0; cb < nb; cb++) {
      int s = base[r * nb + cb];
      if (s == -1) continue;
      if (s < 0 || s >= z) { or_set_error("shift must be -1 or in [0, Z)"); return nullptr; }
      for (int i = 0; i < z; i++)
        edges.push_back({(int64_t)r * z + i, (int64_t)cb * z + (i + s) % z});
    }
  or_code* c = new or_code();
  c->m = (int64_t)mb * z;
  c->n = (int64_t)nb * z;
  finish_code(c, edges);
  c->layers = mb;
  c->check_layer.resize(c->m);
  for (int64_t r = 0; r < c->m; r++) c->check_layer[r] = (int32_t)(r / z);
  c->edge_key.assign(c->row_idx.size(), 0);
  return c;
}

extern "C" or_code* or_code_dvbt2(int frame, int rate) {
  if (frame < 0 || frame > 1 || rate < 0 || rate > 5) {
    or_set_error("DVB-T2 frame must be 0/1 and rate 0..5");
    return nullptr;
  }
  const gf2_dvbt2_table_t& t = gf2_dvbt2_tables[frame * 6 + rate];
  const int64_t n = t.n, k = t.k, m = n - k, q = t.q, z = 360;
  std::vector<std::pair<int64_t, int64_t>> edges;
  for (int b = 0; b < t.rows; b++)
    for (int a = t.row_ptr[b]; a < t.row_ptr[b + 1]; a++) {
      int64_t x = t.addr[a];
      for (int64_t j = 0; j < z; j++) edges.push_back({(x + j * q) % m, b * z + j});
    }
  for (int64_t p = 0; p < m; p++) {
    edges.push_back({p, k + p});
    if (p > 0) edges.push_back({p, k + p - 1});
  }
  or_code* c = new or_code();
  c->m = m;
  c->n = n;
  finish_code(c, edges);
  c->dvb_q = (int)q;
  c->layers = (int)q;
  c->check_layer.resize(m);
  for (int64_t p = 0; p < m; p++) c->check_layer[p] = (int32_t)(p % q);
  // Ordering key of an info edge inside its layer: the circulant shift
  // s = (p div q - j) mod 360; repeated variables of one layer add their
  // deltas in ascending s (the library's layered-schedule rule).
  c->edge_key.assign(c->row_idx.size(), 0);
  for (int64_t p = 0; p < m; p++)
    for (int64_t e = c->row_ptr[p]; e < c->row_ptr[p + 1]; e++) {
      int64_t v = c->row_idx[e];
      if (v < k) c->edge_key[e] = (((p / q) - (v % z)) % z + z) % z;
    }
  // Slot order of a check in the library: its circulants sorted by (info block,
  // shift), then the staircase sub-diagonal and diagonal.  It fixes the
  // association order of the sum-product extrinsic products.
  for (int64_t p = 0; p < m; p++) {
    int64_t b = c->row_ptr[p], d = c->row_ptr[p + 1] - b;
    std::vector<int32_t> ord(d);
    for (int64_t j = 0; j < d; j++) ord[j] = (int32_t)j;
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) {
      int64_t vx = c->row_idx[b + x], vy = c->row_idx[b + y];
      int64_t bx = vx < k ? vx / z : (int64_t)1 << 40, by = vy < k ? vy / z : (int64_t)1 << 40;
      if (bx != by) return bx < by;
      return c->edge_key[b + x] < c->edge_key[b + y];
    });
    for (int64_t j = 0; j < d; j++) c->slot_order[b + j] = ord[j];
  }
  return c;
}

extern "C" void or_code_free(or_code* c) { delete c; }

extern "C" void or_code_dims(const or_code* c, int64_t* o) {
  o[0] = c->n;
  o[1] = c->m;
  o[2] = c->k;
  o[3] = (int64_t)c->row_idx.size();
}

extern "C" void or_code_csr(const or_code* c, int64_t* indptr, int64_t* indices) {
  std::memcpy(indptr, c->row_ptr.data(), sizeof(int64_t) * c->row_ptr.size());
  std::memcpy(indices, c->row_idx.data(), sizeof(int64_t) * c->row_idx.size());
}

extern "C" void or_code_csc(const or_code* c, int64_t* indptr, int64_t* indices) {
  std::memcpy(indptr, c->col_ptr.data(), sizeof(int64_t) * c->col_ptr.size());
  std::memcpy(indices, c->col_idx.data(), sizeof(int64_t) * c->col_idx.size());
}

extern "C" int or_code_layers(const or_code* c) { return c->layers; }

extern "C" void or_code_check_layer(const or_code* c, int32_t* layer) {
  for (int64_t r = 0; r < c->m; r++) layer[r] = c->layers ? c->check_layer[r] : 0;
}

// SpBitMatrix::matvec (sparse.rs:367-381): XOR of the row's bits.
extern "C" int64_t or_syndrome(const or_code* c, const uint8_t* cw, uint8_t* synd) {
  int64_t w = 0;
  for (int64_t r = 0; r < c->m; r++) {
    uint8_t acc = 0;
    for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) acc ^= (cw[c->row_idx[e]] & 1);
    if (synd) synd[r] = acc;
    w += acc;
  }
  return w;
}
