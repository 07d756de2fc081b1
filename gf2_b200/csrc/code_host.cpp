// gf2cuda host side: building the parity-check matrix exactly as the reference
// does, and planning its device layout.
//
// Sparse structure (the reference's, so that neighbour orders match):
//   LdpcCode::from_edges -> SpBitMatrixDual::from_coo      ldpc/core.rs:96-104
//   SpBitMatrix::from_coo: rows sorted, odd multiplicity kept  gf2-core/src/sparse.rs:166-203
//   SpBitMatrix::transpose: stable, CSC rows ascending         gf2-core/src/sparse.rs:297-328
//   build_dvb_edges: (x + j q) mod m, staircase p / p-1       ldpc/dvb_t2/builder.rs:74-118
//   QuasiCyclicLdpc::to_edges: row i -> col (i + s) mod Z     ldpc/core.rs:436-447, 578-605
#include <algorithm>
#include <atomic>
#include <cstring>

#include "dvbt2_tables.h"
#include "internal.h"

namespace gf2c {

static void finish_sparse(HostCode& c, std::vector<std::vector<int64_t>>& per_row) {
  c.row_ptr.assign(1, 0);
  c.row_idx.clear();
  for (auto& row : per_row) {
    std::sort(row.begin(), row.end());
    size_t i = 0;
    while (i < row.size()) {
      size_t cnt = 1;
      while (i + cnt < row.size() && row[i + cnt] == row[i]) cnt++;
      if (cnt & 1) c.row_idx.push_back(row[i]);
      i += cnt;
    }
    c.row_ptr.push_back((int64_t)c.row_idx.size());
  }
  std::vector<int64_t> cnt(c.n + 1, 0);
  for (int64_t v : c.row_idx) cnt[v + 1]++;
  c.col_ptr.assign(c.n + 1, 0);
  for (int64_t v = 0; v < c.n; v++) c.col_ptr[v + 1] = c.col_ptr[v] + cnt[v + 1];
  c.col_idx.assign(c.row_idx.size(), 0);
  c.col_edge.assign(c.row_idx.size(), 0);
  std::vector<int64_t> next(c.col_ptr.begin(), c.col_ptr.end() - 1);
  for (int64_t r = 0; r < c.m; r++)
    for (int64_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; e++) {
      int64_t v = c.row_idx[e];
      c.col_idx[next[v]] = r;
      c.col_edge[next[v]] = e;
      next[v]++;
    }
  c.k = c.n > c.m ? c.n - c.m : 0;
}

uint64_t next_code_serial() {
  static std::atomic<uint64_t> counter{0};
  return ++counter;
}

static uint32_t pack_desc(int type, int base, int shift_or_q) {
  return (uint32_t)base | ((uint32_t)shift_or_q << 20) | ((uint32_t)type << 30);
}

// Edge of (check, var) in CSR, -1 if absent.
static int64_t find_edge(const HostCode& c, int64_t p, int64_t v) {
  auto b = c.row_idx.begin() + c.row_ptr[p], e = c.row_idx.begin() + c.row_ptr[p + 1];
  auto it = std::lower_bound(b, e, v);
  if (it == e || *it != v) return -1;
  return it - c.row_idx.begin();
}

// Builds the VG tables and validates the CG plan against the CSR.  Returns
// false if the plan does not cover every edge exactly once.
static bool finish_plan(HostCode& c) {
  const int64_t E = (int64_t)c.row_idx.size();
  std::vector<int> edge_slot(E, -1);
  int64_t flat = 0;
  for (size_t g = 0; g < c.cg.size(); g++) {
    int4 G = c.cg[g];
    for (int t = 0; t < G.y; t++, flat++) {
      int64_t p = c.cg_checks[flat];
      int real = 0;
      for (int i = 0; i < G.z; i++) {
        int s = G.w + i * G.y + t;
        int v = c.slot_var[s];
        if (v < 0) continue;
        int64_t e = find_edge(c, p, v);
        if (e < 0 || edge_slot[e] >= 0) return false;
        edge_slot[e] = s;
        real++;
      }
      if (real != c.row_ptr[p + 1] - c.row_ptr[p]) return false;
    }
  }
  if (flat != c.m) return false;
  c.chk_cg.assign(c.m, 0);
  flat = 0;
  for (size_t g = 0; g < c.cg.size(); g++)
    for (int t = 0; t < c.cg[g].y; t++) c.chk_cg[flat++] = (uint16_t)g;
  c.max_dc = 0;
  c.max_nchk = 0;
  for (auto& G : c.cg) {
    c.max_dc = std::max(c.max_dc, G.z);
    c.max_nchk = std::max(c.max_nchk, G.y);
  }
  // variable groups
  int nvg = (int)((c.n + c.vgs - 1) / c.vgs);
  c.vg.assign(nvg, int2{0, 0});
  c.vg_slot.clear();
  c.vg_chk.clear();
  c.vg_ci.clear();
  std::vector<int> slot_cc(c.e_slots, -1), slot_i(c.e_slots, -1);
  for (size_t g = 0; g < c.cg.size(); g++) {
    int4 G = c.cg[g];
    for (int i = 0; i < G.z; i++)
      for (int t = 0; t < G.y; t++) {
        slot_cc[(size_t)G.w + (size_t)i * G.y + t] = G.x + t;
        slot_i[(size_t)G.w + (size_t)i * G.y + t] = i;
      }
  }
  c.max_dv = 0;
  for (int h = 0; h < nvg; h++) {
    int dv = 0;
    for (int j = 0; j < c.vgs; j++) {
      int64_t v = (int64_t)h * c.vgs + j;
      if (v >= c.n) break;
      dv = std::max(dv, (int)(c.col_ptr[v + 1] - c.col_ptr[v]));
    }
    c.vg[h] = int2{dv, (int)c.vg_slot.size()};
    size_t base = c.vg_slot.size();
    c.vg_slot.resize(base + (size_t)dv * c.vgs, -1);
    c.vg_chk.resize(base + (size_t)dv * c.vgs, -1);
    c.vg_ci.resize(base + (size_t)dv * c.vgs, -1);
    for (int j = 0; j < c.vgs; j++) {
      int64_t v = (int64_t)h * c.vgs + j;
      if (v >= c.n) break;
      int i = 0;
      for (int64_t s = c.col_ptr[v]; s < c.col_ptr[v + 1]; s++, i++) {
        const int sl = edge_slot[c.col_edge[s]];
        c.vg_slot[base + (size_t)i * c.vgs + j] = sl;
        c.vg_chk[base + (size_t)i * c.vgs + j] = slot_cc[sl];
        c.vg_ci[base + (size_t)i * c.vgs + j] = slot_cc[sl] | (slot_i[sl] << 24);
      }
    }
    c.max_dv = std::max(c.max_dv, dv);
  }
  return true;
}

// Check-state flooding plan.  DVB-T2 parity bits are stored transposed (u order,
// see DevCode); every other code keeps the natural order.  For codes with slot
// descriptors each (CG, slot) is refitted in u order as base + (t + shift) mod Z
// with an optional missing t = 0 (the staircase corner); if any slot does not
// fit, the plan falls back to the natural order and the slot table.  A slot
// with shift s is stored as {start = base + s, wrap = Z - s}; the variable of a
// missing t = 0 entry is start itself (a valid index, masked by sp_absent).
void plan_state(HostCode& c) {
  const int64_t n = c.n;
  std::vector<int> u_of(n), v_of(n);
  for (int64_t v = 0; v < n; v++) u_of[v] = (int)v;
  if (c.kind == 2) {
    const int64_t k = c.k, q = c.q, Z = c.z;
    for (int64_t p = 0; p < c.m; p++) u_of[k + p] = (int)(k + (p % q) * Z + p / q);
  }
  c.sp_desc.clear();
  c.sp_absent.clear();
  c.sp_cg.clear();
  bool structured = !c.slot_desc.empty() && n < (1 << 30);
  for (size_t g = 0; g < c.cg.size() && structured; g++) {
    const int4 G = c.cg[g];
    const int Z = G.y;
    if (G.z > 32) structured = false;
    uint32_t absent = 0;
    for (int i = 0; i < G.z && structured; i++) {
      std::vector<int> u(Z);
      int base = INT32_MAX, t1 = -1;
      for (int t = 0; t < Z; t++) {
        const int v = c.slot_var[(size_t)G.w + (size_t)i * Z + t];
        u[t] = v < 0 ? -1 : u_of[v];
        if (u[t] >= 0) {
          base = std::min(base, u[t]);
          if (t1 < 0) t1 = t;
        } else if (t > 0) {
          structured = false;
        }
      }
      if (!structured || t1 < 0) {
        structured = false;
        break;
      }
      const int sh = (int)((((int64_t)u[t1] - base - t1) % Z + Z) % Z);
      if ((int64_t)base + Z > n) structured = false;  // every start + t must be a valid index
      for (int t = 0; t < Z && structured; t++)
        if (u[t] >= 0 && u[t] != base + (t + sh) % Z) structured = false;
      c.sp_desc.push_back(int2{base + sh, Z - sh});
      if (u[0] < 0) absent |= 1u << i;
    }
    c.sp_absent.push_back(absent);
  }
  if (!structured) {
    c.sp_desc.clear();
    c.sp_absent.clear();
    for (int64_t v = 0; v < n; v++) u_of[v] = (int)v;
  }
  bool identity = true;
  for (int64_t v = 0; v < n; v++) {
    v_of[u_of[v]] = (int)v;
    identity = identity && u_of[v] == v;
  }
  c.sp_u2v.clear();
  if (!identity) c.sp_u2v = v_of;
  int desc_off = 0;
  c.sp_cchunk.clear();
  for (size_t g = 0; g < c.cg.size(); g++) {
    const int4 G = c.cg[g];
    c.sp_cg.push_back(int4{G.x, G.y, G.z, structured ? desc_off : G.w});
    desc_off += G.z;
    for (int t0 = 0; t0 < G.y; t0 += 32) c.sp_cchunk.push_back(int2{(int)g, t0});
  }
  // u-order var groups of vgs variables; edge lists copied from the natural ones
  const int vgs = c.vgs;
  const int nvg = (int)((n + vgs - 1) / vgs);
  std::vector<int2> vg2(nvg, int2{0, 0});
  c.sp_ci.clear();
  c.sp_vchunk.clear();
  for (int h = 0; h < nvg; h++) {
    int dv = 0;
    for (int j = 0; j < vgs && (int64_t)h * vgs + j < n; j++) {
      const int v = v_of[(size_t)h * vgs + j];
      dv = std::max(dv, (int)(c.col_ptr[v + 1] - c.col_ptr[v]));
    }
    const size_t off = c.sp_ci.size();
    vg2[h] = int2{dv, (int)off};
    c.sp_ci.resize(off + (size_t)dv * vgs, -1);
    for (int j = 0; j < vgs && (int64_t)h * vgs + j < n; j++) {
      const int v = v_of[(size_t)h * vgs + j];
      const int hv = v / vgs, jv = v - hv * vgs;
      const int2 V = c.vg[hv];
      const int deg = (int)(c.col_ptr[v + 1] - c.col_ptr[v]);
      for (int i = 0; i < deg; i++) c.sp_ci[off + (size_t)i * vgs + j] = c.vg_ci[(size_t)V.y + (size_t)i * vgs + jv];
    }
    for (int j0 = 0; j0 < vgs && (int64_t)h * vgs + j0 < n; j0 += 32) c.sp_vchunk.push_back(int2{h, j0});
  }
  c.sp_vg = vg2;
}

// Generic plan: CGs of up to 256 consecutive checks, slots in CSR order.
static void plan_generic(HostCode& c) {
  c.cg.clear();
  c.cg_sync.clear();
  c.slot_var.clear();
  c.cg_checks.clear();
  const int G = 256;
  int edge0 = 0;
  for (int64_t r0 = 0; r0 < c.m; r0 += G) {
    int nchk = (int)std::min<int64_t>(G, c.m - r0);
    int dc = 0;
    for (int t = 0; t < nchk; t++) dc = std::max(dc, (int)(c.row_ptr[r0 + t + 1] - c.row_ptr[r0 + t]));
    c.cg.push_back(int4{(int)r0, nchk, dc, edge0});
    c.cg_sync.push_back(0);
    c.slot_var.resize((size_t)edge0 + (size_t)dc * nchk, -1);
    for (int t = 0; t < nchk; t++) {
      int64_t r = r0 + t;
      c.cg_checks.push_back(r);
      int i = 0;
      for (int64_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; e++, i++)
        c.slot_var[(size_t)edge0 + (size_t)i * nchk + t] = (int)c.row_idx[e];
    }
    edge0 += dc * nchk;
  }
  c.e_slots = edge0;
  c.vgs = 256;
  c.layered_ok = 0;
  finish_plan(c);
}

int build_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count, HostCode& c) {
  if (m < 0 || n < 0 || count < 0 || (count > 0 && !pairs))
    return set_error(GF2C_ERR_INVALID_ARG, "invalid dimensions or pairs");
  if (n > (int64_t)1 << 30 || m > 65535LL * 256 || count > (int64_t)1 << 31)
    return set_error(GF2C_ERR_UNSUPPORTED, "code too large");
  c.m = m;
  c.n = n;
  std::vector<std::vector<int64_t>> per_row(m);
  for (int64_t i = 0; i < count; i++) {
    int64_t r = pairs[2 * i], col = pairs[2 * i + 1];
    if (r < 0 || r >= m || col < 0 || col >= n)
      return set_error(GF2C_ERR_INVALID_ARG, "edge index out of bounds");
    per_row[r].push_back(col);
  }
  finish_sparse(c, per_row);
  c.kind = 0;
  plan_generic(c);
  plan_state(c);
  return GF2C_OK;
}

int build_qc(const int32_t* base, int mb, int nb, int z, HostCode& c) {
  if (!base || mb <= 0 || nb <= 0) return set_error(GF2C_ERR_INVALID_ARG, "base matrix must be non-empty");
  if (z <= 0) return set_error(GF2C_ERR_INVALID_ARG, "expansion factor must be positive");
  if ((int64_t)mb * z > 65535LL * 256 || (int64_t)nb * z > (int64_t)1 << 30)
    return set_error(GF2C_ERR_UNSUPPORTED, "code too large");
  c.m = (int64_t)mb * z;
  c.n = (int64_t)nb * z;
  std::vector<std::vector<int64_t>> per_row(c.m);
  for (int r = 0; r < mb; r++)
    for (int cb = 0; cb < nb; cb++) {
      int s = base[r * nb + cb];
      if (s == -1) continue;
      if (s < 0 || s >= z) return set_error(GF2C_ERR_INVALID_ARG, "shift must be -1 or in [0, Z)");
      for (int i = 0; i < z; i++) per_row[(int64_t)r * z + i].push_back((int64_t)cb * z + (i + s) % z);
    }
  finish_sparse(c, per_row);
  c.kind = 1;
  c.z = z;
  c.mb = mb;
  c.nb = nb;
  c.qc_base.assign(base, base + (size_t)mb * nb);
  // QC plan: one CG per base row, slots in ascending base column.
  c.cg.clear();
  c.cg_sync.clear();
  c.slot_var.clear();
  c.cg_checks.clear();
  int edge0 = 0;
  for (int r = 0; r < mb; r++) {
    std::vector<std::pair<int, int>> circ;
    for (int cb = 0; cb < nb; cb++)
      if (base[r * nb + cb] >= 0) circ.push_back({cb, base[r * nb + cb]});
    int dc = (int)circ.size();
    c.cg.push_back(int4{r * z, z, dc, edge0});
    c.cg_sync.push_back(0);
    for (int i = 0; i < dc; i++) c.slot_desc.push_back(pack_desc(0, circ[i].first * z, circ[i].second));
    c.cg_ninfo.push_back(dc);
    c.slot_var.resize((size_t)edge0 + (size_t)dc * z, -1);
    for (int t = 0; t < z; t++) {
      c.cg_checks.push_back((int64_t)r * z + t);
      for (int i = 0; i < dc; i++)
        c.slot_var[(size_t)edge0 + (size_t)i * z + t] = circ[i].first * z + (t + circ[i].second) % z;
    }
    edge0 += dc * z;
  }
  c.e_slots = edge0;
  c.vgs = z <= 1024 ? z : 256;
  c.layered_ok = (z <= 1023 && c.n < (1 << 20)) ? 1 : 0;
  if (!c.layered_ok) c.slot_desc.clear();
  if (!finish_plan(c)) {
    c.slot_desc.clear();
    plan_generic(c);
  }
  plan_state(c);
  return GF2C_OK;
}

int build_dvbt2(int frame, int rate, HostCode& c) {
  if (frame < 0 || frame > 1 || rate < 0 || rate > 5)
    return set_error(GF2C_ERR_INVALID_ARG, "DVB-T2 frame size must be 0/1 and rate 0..5");
  const gf2_dvbt2_table_t& T = gf2_dvbt2_tables[frame * 6 + rate];
  const int64_t n = T.n, k = T.k, m = n - k, q = T.q, Z = 360;
  c.m = m;
  c.n = n;
  std::vector<std::vector<int64_t>> per_row(m);
  for (int b = 0; b < T.rows; b++)
    for (int a = T.row_ptr[b]; a < T.row_ptr[b + 1]; a++) {
      int64_t x = T.addr[a];
      for (int64_t j = 0; j < Z; j++) per_row[(x + j * q) % m].push_back(b * Z + j);
    }
  for (int64_t p = 0; p < m; p++) {
    per_row[p].push_back(k + p);
    if (p > 0) per_row[p].push_back(k + p - 1);
  }
  finish_sparse(c, per_row);
  c.kind = 2;
  c.z = (int)Z;
  c.q = (int)q;
  // encoder lists: address x of block b lies in row group x mod q and rotates
  // the block's 360 bits by x div q; repeated addresses cancel (XOR)
  {
    std::vector<std::vector<int>> rg(q);
    for (int b = 0; b < T.rows; b++) {
      std::vector<int64_t> xs(T.addr + T.row_ptr[b], T.addr + T.row_ptr[b + 1]);
      std::sort(xs.begin(), xs.end());
      for (size_t i = 0; i < xs.size();) {
        size_t j = i;
        while (j < xs.size() && xs[j] == xs[i]) j++;
        if ((j - i) & 1) rg[xs[i] % q].push_back((b << 16) | (int)(xs[i] / q));
        i = j;
      }
    }
    c.enc_rg_ptr.assign(1, 0);
    c.enc_rg_ent.clear();
    for (const auto& v : rg) {
      c.enc_rg_ent.insert(c.enc_rg_ent.end(), v.begin(), v.end());
      c.enc_rg_ptr.push_back((int)c.enc_rg_ent.size());
    }
  }
  c.dvb_index = frame * 6 + rate;
  // Row group a = checks p = a + q t (t = 0..359).  An address x lies in row
  // group x mod q and, for info block b, links check t to bit b*360 + (t - x div q) mod 360:
  // one 360x360 circulant.  Slots: circulants sorted by (block, shift), then the
  // staircase sub-diagonal (k + p - 1, absent for p = 0) and diagonal (k + p).
  c.cg.clear();
  c.cg_sync.clear();
  c.slot_var.clear();
  c.cg_checks.clear();
  std::vector<std::vector<std::pair<int, int>>> circ(q);
  for (int b = 0; b < T.rows; b++)
    for (int a = T.row_ptr[b]; a < T.row_ptr[b + 1]; a++) {
      int x = T.addr[a];
      circ[x % q].push_back({b, x / (int)q});
    }
  int edge0 = 0;
  for (int a = 0; a < q; a++) {
    auto& cl = circ[a];
    std::sort(cl.begin(), cl.end());
    int ninfo = (int)cl.size();
    int dc = ninfo + 2;
    c.cg.push_back(int4{(int)(a * Z), (int)Z, dc, edge0});
    uint32_t sync = 0;
    for (int i = 0; i + 1 < ninfo; i++)
      if (cl[i].first == cl[i + 1].first) sync |= 1u << i;
    c.cg_sync.push_back(sync);
    for (int i = 0; i < ninfo; i++)
      c.slot_desc.push_back(pack_desc(0, cl[i].first * (int)Z, (int)((Z - cl[i].second) % Z)));
    c.slot_desc.push_back(pack_desc(1, (int)(k + a), (int)q));
    c.slot_desc.push_back(pack_desc(2, (int)(k + a), (int)q));
    c.cg_ninfo.push_back(ninfo);
    c.slot_var.resize((size_t)edge0 + (size_t)dc * Z, -1);
    for (int t = 0; t < Z; t++) {
      int64_t p = a + q * t;
      c.cg_checks.push_back(p);
      for (int i = 0; i < ninfo; i++)
        c.slot_var[(size_t)edge0 + (size_t)i * Z + t] =
            (int)(cl[i].first * Z + ((t - cl[i].second) % Z + Z) % Z);
      c.slot_var[(size_t)edge0 + (size_t)ninfo * Z + t] = p > 0 ? (int)(k + p - 1) : -1;
      c.slot_var[(size_t)edge0 + (size_t)(ninfo + 1) * Z + t] = (int)(k + p);
    }
    edge0 += dc * (int)Z;
  }
  c.e_slots = edge0;
  c.vgs = (int)Z;
  c.layered_ok = 1;
  if (!finish_plan(c)) {
    c.slot_desc.clear();
    plan_generic(c);
  }
  // cross-check the descriptors against the slot table
  for (size_t g = 0; g < c.cg.size() && !c.slot_desc.empty(); g++) {
    const int4 G = c.cg[g];
    for (int i = 0; i < G.z; i++) {
      const uint32_t D = c.slot_desc[G.w / G.y + i];
      const int type = (int)(D >> 30), sh = (int)((D >> 20) & 1023u), base = (int)(D & 0xFFFFFu);
      for (int t = 0; t < G.y; t++) {
        int v;
        if (type == 0) v = base + (t + sh) % G.y;
        else if (type == 1) v = (g == 0 && t == 0) ? -1 : base + sh * t - 1;
        else v = base + sh * t;
        if (v != c.slot_var[(size_t)G.w + (size_t)i * G.y + t])
          return set_error(GF2C_ERR_KERNEL, "internal: DVB-T2 slot descriptor mismatch");
      }
    }
  }
  plan_state(c);
  return GF2C_OK;
}

// Right-to-left pivot search (RuEncodingMatrices::compute_generator_matrix with
// rref(h, pivot_from_right = true), richardson_urbanke.rs:158-243 and
// gf2-core/src/alg/rref.rs:67-130): parity columns = greedy right-most basis of
// the column space, message columns = the rest in ascending order, and
// P[i][j] = reduced H[pivot row of parity column j][message column i].
int prepare_encoder(HostCode& c) {
  if (c.enc_ready) return c.enc_status;
  c.enc_ready = true;
  if (c.kind == 2) {
    c.enc_kind = 0;
    c.enc_status = GF2C_OK;
    return GF2C_OK;
  }
  c.enc_kind = 1;
  const int64_t m = c.m, n = c.n;
  if (m == 0 || n == 0 || m >= n) {
    c.enc_status = set_error(GF2C_ERR_INVALID_ARG, "encoding needs 0 < m < n");
    return c.enc_status;
  }
  const int64_t W = (n + 63) / 64;
  if ((double)m * (double)W * 8.0 > 4e9) {
    c.enc_status = set_error(GF2C_ERR_UNSUPPORTED, "generic encoder: matrix too large");
    return c.enc_status;
  }
  std::vector<uint64_t> rows((size_t)m * W, 0);
  for (int64_t r = 0; r < m; r++)
    for (int64_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; e++)
      rows[(size_t)r * W + (c.row_idx[e] >> 6)] |= 1ull << (c.row_idx[e] & 63);
  std::vector<char> used(m, 0), is_piv(n, 0);
  std::vector<int64_t> piv_row;
  c.enc_par_cols.clear();
  for (int64_t col = n - 1; col >= 0 && (int64_t)piv_row.size() < m; col--) {
    int64_t pr = -1;
    for (int64_t r = 0; r < m; r++)
      if (!used[r] && ((rows[(size_t)r * W + (col >> 6)] >> (col & 63)) & 1)) {
        pr = r;
        break;
      }
    if (pr < 0) continue;
    used[pr] = 1;
    const uint64_t* src = &rows[(size_t)pr * W];
    for (int64_t r = 0; r < m; r++)
      if (r != pr && ((rows[(size_t)r * W + (col >> 6)] >> (col & 63)) & 1)) {
        uint64_t* dst = &rows[(size_t)r * W];
        for (int64_t w = 0; w < W; w++) dst[w] ^= src[w];
      }
    c.enc_par_cols.push_back((int)col);
    piv_row.push_back(pr);
    is_piv[col] = 1;
  }
  if ((int64_t)piv_row.size() != m) {
    c.enc_status = set_error(GF2C_ERR_RANK, "parity-check matrix is rank deficient");
    return c.enc_status;
  }
  c.enc_msg_cols.clear();
  for (int64_t col = 0; col < n; col++)
    if (!is_piv[col]) c.enc_msg_cols.push_back((int)col);
  const int64_t Wm = (m + 63) / 64;
  c.enc_p.assign((size_t)c.k * Wm, 0);
  for (int64_t i = 0; i < c.k; i++) {
    int64_t col = c.enc_msg_cols[i];
    for (int64_t j = 0; j < m; j++)
      if ((rows[(size_t)piv_row[j] * W + (col >> 6)] >> (col & 63)) & 1)
        c.enc_p[(size_t)i * Wm + (j >> 6)] |= 1ull << (j & 63);
  }
  c.enc_status = GF2C_OK;
  return GF2C_OK;
}

template <class T>
static int dev_copy(HostCode& c, const std::vector<T>& v, const T** out) {
  if (v.empty()) {
    *out = nullptr;
    return GF2C_OK;
  }
  void* p = nullptr;
  GF2C_CUDA(cudaMalloc(&p, sizeof(T) * v.size()));
  c.dev_allocs.push_back(p);
  GF2C_CUDA(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  *out = (const T*)p;
  return GF2C_OK;
}

int upload_code(HostCode& c) {
  std::lock_guard<std::mutex> lock(c.dev_mu);
  int dev = 0;
  GF2C_CUDA(cudaGetDevice(&dev));
  bool need_enc = c.enc_ready && c.enc_status == GF2C_OK && c.enc_kind == 1 && !c.dev.enc_p;
  if (c.dev_id == dev && !need_enc) return GF2C_OK;
  if (c.dev_id != dev) {
    if (c.dev_id >= 0) return set_error(GF2C_ERR_UNSUPPORTED, "code already bound to another device");
    DevCode d{};
    d.n = (int)c.n;
    d.m = (int)c.m;
    d.k = (int)c.k;
    d.ncg = (int)c.cg.size();
    d.nvg = (int)c.vg.size();
    d.vgs = c.vgs;
    d.e_slots = c.e_slots;
    d.max_dc = c.max_dc;
    d.max_dv = c.max_dv;
    d.words_k = (int)((c.k + 63) / 64);
    d.words_n = (int)((c.n + 63) / 64);
    d.words_m = (int)((c.m + 63) / 64);
    d.layered_ok = c.layered_ok;
    d.lay_bucket = layered_dcmax_bucket(c.max_dc);
    d.max_nchk = c.max_nchk;
    int rc;
    if ((rc = dev_copy(c, c.cg, &d.cg))) return rc;
    if ((rc = dev_copy(c, c.cg_sync, &d.cg_sync))) return rc;
    if ((rc = dev_copy(c, c.slot_var, &d.slot_var))) return rc;
    if ((rc = dev_copy(c, c.chk_cg, &d.chk_cg))) return rc;
    if ((rc = dev_copy(c, c.vg, &d.vg))) return rc;
    if ((rc = dev_copy(c, c.vg_slot, &d.vg_slot))) return rc;
    if ((rc = dev_copy(c, c.vg_chk, &d.vg_chk))) return rc;
    if ((rc = dev_copy(c, c.vg_ci, &d.vg_ci))) return rc;
    if ((rc = dev_copy(c, c.slot_desc, &d.slot_desc))) return rc;
    if ((rc = dev_copy(c, c.slot_desc.empty() ? std::vector<int>() : c.cg_ninfo, &d.cg_ninfo))) return rc;
    d.z = c.slot_desc.empty() ? 0 : c.z;
    if ((rc = dev_copy(c, c.sp_cg, &d.sp_cg))) return rc;
    if ((rc = dev_copy(c, c.sp_desc, &d.sp_desc))) return rc;
    if ((rc = dev_copy(c, c.sp_absent, &d.sp_absent))) return rc;
    if ((rc = dev_copy(c, c.sp_cchunk, &d.sp_cchunk))) return rc;
    if ((rc = dev_copy(c, c.sp_vg, &d.sp_vg))) return rc;
    if ((rc = dev_copy(c, c.sp_ci, &d.sp_ci))) return rc;
    if ((rc = dev_copy(c, c.sp_vchunk, &d.sp_vchunk))) return rc;
    if ((rc = dev_copy(c, c.sp_u2v, &d.sp_u2v))) return rc;
    d.sp_ncchunk = (int)c.sp_cchunk.size();
    d.sp_nvchunk = (int)c.sp_vchunk.size();
    std::vector<int> rp(c.row_ptr.begin(), c.row_ptr.end()), ri(c.row_idx.begin(), c.row_idx.end());
    if ((rc = dev_copy(c, rp, &d.csr_ptr))) return rc;
    if ((rc = dev_copy(c, ri, &d.csr_idx))) return rc;
    d.enc_kind = c.kind == 2 ? 0 : 1;
    if (c.kind == 2) {
      d.enc_q = c.q;
      if ((rc = dev_copy(c, c.enc_rg_ptr, &d.enc_rg_ptr))) return rc;
      if ((rc = dev_copy(c, c.enc_rg_ent, &d.enc_rg_ent))) return rc;
    }
    c.dev = d;
    c.dev_id = dev;
  }
  if (need_enc) {
    int rc;
    if ((rc = dev_copy(c, c.enc_p, &c.dev.enc_p))) return rc;
    if ((rc = dev_copy(c, c.enc_msg_cols, &c.dev.enc_msg_cols))) return rc;
    if ((rc = dev_copy(c, c.enc_par_cols, &c.dev.enc_par_cols))) return rc;
  }
  return GF2C_OK;
}

HostCode::~HostCode() {
  for (void* p : dev_allocs) cudaFree(p);
}

}  // namespace gf2c
