// gf2cuda host I/O: the gf2 binary / text / hex file formats and the LDPC
// encoder cache (crates/gf2-core/src/io, crates/gf2-coding/src/ldpc/encoding/cache.rs).
//
// Binary files ("GF2DATA", io/format.rs:1-16, io/header.rs:6-82):
//   32-byte header: magic "GF2DATA\0", u16 version (1), u8 type tag
//   (1 BitVec, 2 BitMatrix, 3 SpBitMatrix, 4 SpBitMatrixDual), u8 flags,
//   8 reserved bytes, u32 metadata length, u64 payload length (little endian);
//   then compact JSON metadata (serde_json field order of the metadata struct);
//   then the payload:
//     BitVec        words, u64 LE                                  (io/bitvec.rs)
//     BitMatrix     rows x ceil(cols/64) words, row-major, u64 LE  (io/matrix.rs)
//     SpBitMatrix   nnz (row, col) pairs in CSR order, u32 LE      (io/sparse.rs)
//     SpBitMatrixDual  row offsets, column indices, column offsets, row indices, u32 LE
// Text / hex files and the format detection follow io/formats.rs.
//
// Encoder cache (cache.rs:304-438, 461-502): one BitMatrix file per code,
// "n{n}_k{k}_h{hash:x}.gf2", holding the dense parity part P (k x r, row i =
// the parity bits of message bit i) of the systematic form [message | parity]
// with the message in columns [0, k).  The hash is Rust's DefaultHasher
// (SipHash-1-3 with zero keys) over rows, cols, nnz of H and the first 100
// (row, col) edges in CSR order, every value fed as 8 little-endian bytes.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "internal.h"

using namespace gf2c;

namespace {

const char kMagic[8] = {'G', 'F', '2', 'D', 'A', 'T', 'A', '\0'};
constexpr int kHeader = 32;

// ---------------------------------------------------------------------------
// SipHash-1-3 (Aumasson & Bernstein's SipHash with one compression and three
// finalisation rounds)
// ---------------------------------------------------------------------------
inline uint64_t rotl(uint64_t x, int b) { return (x << b) | (x >> (64 - b)); }

struct Sip13 {
  uint64_t v0, v1, v2, v3, tail = 0;
  uint64_t total = 0;
  int ntail = 0;
  Sip13(uint64_t k0, uint64_t k1) {
    v0 = k0 ^ 0x736f6d6570736575ull;
    v1 = k1 ^ 0x646f72616e646f6dull;
    v2 = k0 ^ 0x6c7967656e657261ull;
    v3 = k1 ^ 0x7465646279746573ull;
  }
  void round() {
    v0 += v1; v1 = rotl(v1, 13); v1 ^= v0; v0 = rotl(v0, 32);
    v2 += v3; v3 = rotl(v3, 16); v3 ^= v2;
    v0 += v3; v3 = rotl(v3, 21); v3 ^= v0;
    v2 += v1; v1 = rotl(v1, 17); v1 ^= v2; v2 = rotl(v2, 32);
  }
  void block(uint64_t m) {
    v3 ^= m;
    round();
    v0 ^= m;
  }
  void write(const uint8_t* p, size_t len) {
    total += len;
    for (size_t i = 0; i < len; i++) {
      tail |= (uint64_t)p[i] << (8 * ntail);
      if (++ntail == 8) {
        block(tail);
        tail = 0;
        ntail = 0;
      }
    }
  }
  void write_u64(uint64_t x) {
    uint8_t b[8];
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(x >> (8 * i));
    write(b, 8);
  }
  uint64_t finish() {
    Sip13 s = *this;
    s.block(((s.total & 0xff) << 56) | s.tail);
    s.v2 ^= 0xff;
    s.round();
    s.round();
    s.round();
    return s.v0 ^ s.v1 ^ s.v2 ^ s.v3;
  }
};

// ---------------------------------------------------------------------------
// byte helpers
// ---------------------------------------------------------------------------
void put_le(std::string& out, uint64_t v, int bytes) {
  for (int i = 0; i < bytes; i++) out.push_back((char)(uint8_t)(v >> (8 * i)));
}
uint64_t get_le(const std::string& s, size_t off, int bytes) {
  uint64_t v = 0;
  for (int i = 0; i < bytes; i++) v |= (uint64_t)(uint8_t)s[off + i] << (8 * i);
  return v;
}

int read_file(const char* path, std::string& out) {
  if (!path) return set_error(GF2C_ERR_INVALID_ARG, "path is NULL");
  std::ifstream f(path, std::ios::binary);
  if (!f) return set_error(GF2C_ERR_INVALID_ARG, std::string("cannot open ") + path);
  std::ostringstream ss;
  ss << f.rdbuf();
  out = ss.str();
  return GF2C_OK;
}

int write_file(const char* path, const std::string& data) {
  if (!path) return set_error(GF2C_ERR_INVALID_ARG, "path is NULL");
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return set_error(GF2C_ERR_INVALID_ARG, std::string("cannot create ") + path);
  f.write(data.data(), (std::streamsize)data.size());
  if (!f) return set_error(GF2C_ERR_INVALID_ARG, std::string("write failed: ") + path);
  return GF2C_OK;
}

std::string binary_file(int tag, const std::string& meta, const std::string& payload) {
  std::string out(kMagic, 8);
  put_le(out, 1, 2);          // version
  out.push_back((char)tag);   // type tag
  out.push_back(0);           // flags
  out.append(8, '\0');        // reserved
  put_le(out, meta.size(), 4);
  put_le(out, payload.size(), 8);
  out += meta;
  out += payload;
  return out;
}

// A parsed binary file: tag, metadata fields, payload.
struct Parsed {
  int tag = 0;
  std::string meta;
  std::string payload;
};

int parse_binary(const std::string& s, Parsed& p) {
  if (s.size() < (size_t)kHeader || std::memcmp(s.data(), kMagic, 8) != 0)
    return set_error(GF2C_ERR_INVALID_ARG, "invalid magic bytes (not a GF2DATA file)");
  const uint64_t version = get_le(s, 8, 2);
  if (version != 1) return set_error(GF2C_ERR_UNSUPPORTED, "unsupported GF2DATA version " + std::to_string(version));
  p.tag = (uint8_t)s[10];
  if (p.tag < 1 || p.tag > 4) return set_error(GF2C_ERR_INVALID_ARG, "unknown type tag " + std::to_string(p.tag));
  const uint64_t ml = get_le(s, 20, 4), dl = get_le(s, 24, 8);
  if ((uint64_t)s.size() < (uint64_t)kHeader + ml + dl) return set_error(GF2C_ERR_INVALID_ARG, "truncated GF2DATA file");
  p.meta = s.substr(kHeader, ml);
  p.payload = s.substr(kHeader + ml, dl);
  return GF2C_OK;
}

// Metadata value of `key` (a JSON number or string) in a flat JSON object.
bool meta_value(const std::string& meta, const char* key, std::string& out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t pos = 0;
  while ((pos = meta.find(k, pos)) != std::string::npos) {
    size_t i = pos + k.size();
    while (i < meta.size() && std::isspace((unsigned char)meta[i])) i++;
    if (i < meta.size() && meta[i] == ':') {
      i++;
      while (i < meta.size() && std::isspace((unsigned char)meta[i])) i++;
      if (i < meta.size() && meta[i] == '"') {
        const size_t e = meta.find('"', i + 1);
        if (e == std::string::npos) return false;
        out = meta.substr(i + 1, e - i - 1);
        return true;
      }
      size_t e = i;
      while (e < meta.size() && (std::isdigit((unsigned char)meta[e]) || meta[e] == '-')) e++;
      if (e == i) return false;
      out = meta.substr(i, e - i);
      return true;
    }
    pos += k.size();
  }
  return false;
}

int meta_int(const std::string& meta, const char* key, int64_t& v) {
  std::string s;
  if (!meta_value(meta, key, s)) return set_error(GF2C_ERR_INVALID_ARG, std::string("metadata lacks ") + key);
  v = std::stoll(s);
  if (v < 0) return set_error(GF2C_ERR_INVALID_ARG, std::string("negative ") + key);
  return GF2C_OK;
}

int check_type(const Parsed& p, int tag, const char* name) {
  if (p.tag != tag) return set_error(GF2C_ERR_INVALID_ARG, std::string("expected ") + name + " type tag, got " + std::to_string(p.tag));
  std::string t;
  if (!meta_value(p.meta, "type", t) || t != name)
    return set_error(GF2C_ERR_INVALID_ARG, std::string("expected ") + name + " metadata type");
  return GF2C_OK;
}

// SerializationFormat::detect (io/formats.rs): 0 binary, 1 text, 2 hex, -1 unknown.
int detect_format(const std::string& b) {
  if (b.empty()) return -1;
  if (b.size() >= 8 && std::memcmp(b.data(), kMagic, 8) == 0) return 0;
  auto text_byte = [](unsigned char c) { return std::isdigit(c) || c == '\n' || c == '\r' || c == ' ' || c == '\t'; };
  if (b.size() < 8) {
    for (unsigned char c : b)
      if (!text_byte(c)) return -1;
    return 1;
  }
  const size_t nl = b.find('\n');
  if (nl != std::string::npos && nl + 1 < b.size()) {
    const size_t s2 = nl + 1;
    size_t e2 = b.find('\n', s2);
    if (e2 == std::string::npos) e2 = b.size();
    bool hexletter = false, allhex = true, only01 = true;
    for (size_t i = s2; i < e2; i++) {
      const unsigned char c = b[i];
      if ((c >= 'A' && c <= 'F') || (c >= 'a' && c <= 'f')) hexletter = true;
      if (!std::isxdigit(c)) allhex = false;
      if (c != '0' && c != '1') only01 = false;
    }
    if (hexletter) return 2;
    const size_t l2 = e2 - s2;
    if (l2 >= 16 && l2 % 16 == 0 && allhex && !only01) return 2;
  }
  const size_t lim = std::min<size_t>(b.size(), 100);
  size_t zo = 0;
  bool valid = true;
  for (size_t i = 0; i < lim; i++) {
    const unsigned char c = b[i];
    if (c == '0' || c == '1') zo++;
    if (!(c == '0' || c == '1' || text_byte(c))) valid = false;
  }
  if (zo > 0 && zo * 100 >= lim * 70 && valid) return 1;
  if (std::isdigit((unsigned char)b[0])) {
    size_t e = b.find('\n');
    if (e == std::string::npos) e = b.size();
    bool dims = true;
    for (size_t i = 0; i < e; i++) {
      const unsigned char c = b[i];
      if (!(std::isdigit(c) || c == ' ' || c == '\t')) dims = false;
    }
    if (dims) return 1;
  }
  return -1;
}

std::vector<std::string> lines_of(const std::string& s) {
  std::vector<std::string> out;
  size_t i = 0;
  while (i < s.size()) {
    size_t e = s.find('\n', i);
    if (e == std::string::npos) e = s.size();
    std::string l = s.substr(i, e - i);
    while (!l.empty() && (l.back() == '\r' || l.back() == ' ' || l.back() == '\t')) l.pop_back();
    size_t b = 0;
    while (b < l.size() && (l[b] == ' ' || l[b] == '\t')) b++;
    out.push_back(l.substr(b));
    i = e + 1;
  }
  return out;
}

std::vector<int64_t> ints_of(const std::string& l) {
  std::vector<int64_t> v;
  std::istringstream is(l);
  std::string tok;
  while (is >> tok) {
    for (char c : tok)
      if (!std::isdigit((unsigned char)c)) return {};
    v.push_back(std::stoll(tok));
  }
  return v;
}

bool parse_hex_word(const std::string& s, uint64_t& w) {
  if (s.size() != 16) return false;
  w = 0;
  for (char c : s) {
    int d;
    if (c >= '0' && c <= '9') d = c - '0';
    else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else return false;
    w = (w << 4) | (uint64_t)d;
  }
  return true;
}

std::string hex_word(uint64_t w) {
  char buf[17];
  std::snprintf(buf, sizeof buf, "%016llX", (unsigned long long)w);
  return std::string(buf, 16);
}

inline int64_t words_of(int64_t bits) { return bits == 0 ? 0 : (bits + 63) / 64; }
inline bool bit_of(const uint64_t* w, int64_t i) { return (w[i >> 6] >> (i & 63)) & 1; }

// ---------------------------------------------------------------------------
// BitVec / BitMatrix
// ---------------------------------------------------------------------------
int read_bitvec_any(const std::string& s, std::vector<uint64_t>& words, int64_t& len) {
  const int fmt = detect_format(s);
  if (fmt < 0) return set_error(GF2C_ERR_INVALID_ARG, "unable to detect file format");
  if (fmt == 0) {
    Parsed p;
    int rc;
    if ((rc = parse_binary(s, p)) || (rc = check_type(p, 1, "BitVec")) || (rc = meta_int(p.meta, "len_bits", len))) return rc;
    const int64_t W = words_of(len);
    if ((int64_t)p.payload.size() != W * 8) return set_error(GF2C_ERR_INVALID_ARG, "BitVec data length mismatch");
    words.assign(W, 0);
    for (int64_t i = 0; i < W; i++) words[i] = get_le(p.payload, 8 * i, 8);
    if (len & 63) words[W - 1] &= (1ull << (len & 63)) - 1ull;
    return GF2C_OK;
  }
  const auto L = lines_of(s);
  if (L.empty()) return set_error(GF2C_ERR_INVALID_ARG, "empty BitVec file");
  const auto d = ints_of(L[0]);
  if (d.size() != 1) return set_error(GF2C_ERR_INVALID_ARG, "BitVec text/hex must start with the length");
  len = d[0];
  const int64_t W = words_of(len);
  words.assign(W, 0);
  if (fmt == 1) {
    int64_t i = 0;
    for (size_t li = 1; li < L.size() && i < len; li++)
      for (char c : L[li]) {
        if (c != '0' && c != '1') return set_error(GF2C_ERR_INVALID_ARG, "invalid bit character");
        if (i >= len) break;
        if (c == '1') words[i >> 6] |= 1ull << (i & 63);
        i++;
      }
    if (i != len) return set_error(GF2C_ERR_INVALID_ARG, "BitVec text has fewer bits than its length");
  } else {
    for (int64_t w = 0; w < W; w++) {
      if ((size_t)(w + 1) >= L.size() || !parse_hex_word(L[w + 1], words[w]))
        return set_error(GF2C_ERR_INVALID_ARG, "invalid BitVec hex word");
    }
    if (len & 63) words[W - 1] &= (1ull << (len & 63)) - 1ull;
  }
  return GF2C_OK;
}

int read_bitmatrix_fmt(const std::string& s, int fmt, std::vector<uint64_t>& words, int64_t& rows, int64_t& cols) {
  if (fmt < 0) fmt = detect_format(s);
  if (fmt < 0) return set_error(GF2C_ERR_INVALID_ARG, "unable to detect file format");
  if (fmt == 0) {
    Parsed p;
    int rc;
    if ((rc = parse_binary(s, p)) || (rc = check_type(p, 2, "BitMatrix")) || (rc = meta_int(p.meta, "rows", rows)) ||
        (rc = meta_int(p.meta, "cols", cols)))
      return rc;
    const int64_t S = words_of(cols);
    if ((int64_t)p.payload.size() != rows * S * 8) return set_error(GF2C_ERR_INVALID_ARG, "BitMatrix data length mismatch");
    words.assign((size_t)(rows * S), 0);
    for (int64_t i = 0; i < rows * S; i++) words[i] = get_le(p.payload, 8 * i, 8);
    if (cols & 63)
      for (int64_t r = 0; r < rows; r++) words[r * S + S - 1] &= (1ull << (cols & 63)) - 1ull;
    return GF2C_OK;
  }
  const auto L = lines_of(s);
  if (L.empty()) return set_error(GF2C_ERR_INVALID_ARG, "empty BitMatrix file");
  const auto d = ints_of(L[0]);
  if (d.size() != 2) return set_error(GF2C_ERR_INVALID_ARG, "BitMatrix text/hex must start with 'rows cols'");
  rows = d[0];
  cols = d[1];
  const int64_t S = words_of(cols);
  words.assign((size_t)(rows * S), 0);
  for (int64_t r = 0; r < rows; r++) {
    if ((size_t)(r + 1) >= L.size()) return set_error(GF2C_ERR_INVALID_ARG, "BitMatrix file has too few rows");
    const std::string& l = L[r + 1];
    if (fmt == 1) {
      if ((int64_t)l.size() != cols) return set_error(GF2C_ERR_INVALID_ARG, "BitMatrix text row has the wrong length");
      for (int64_t c = 0; c < cols; c++) {
        if (l[c] != '0' && l[c] != '1') return set_error(GF2C_ERR_INVALID_ARG, "invalid bit character");
        if (l[c] == '1') words[r * S + (c >> 6)] |= 1ull << (c & 63);
      }
    } else {
      if ((int64_t)l.size() != S * 16) return set_error(GF2C_ERR_INVALID_ARG, "BitMatrix hex row has the wrong length");
      for (int64_t w = 0; w < S; w++)
        if (!parse_hex_word(l.substr(16 * w, 16), words[r * S + w]))
          return set_error(GF2C_ERR_INVALID_ARG, "invalid BitMatrix hex word");
      if (cols & 63) words[r * S + S - 1] &= (1ull << (cols & 63)) - 1ull;
    }
  }
  return GF2C_OK;
}

// ---------------------------------------------------------------------------
// sparse matrices
// ---------------------------------------------------------------------------
// CSR of a COO list, rows sorted and duplicates removed (SpBitMatrix::from_coo_deduplicated).
int csr_dedup(int64_t rows, int64_t cols, const std::vector<std::pair<int64_t, int64_t>>& e, std::vector<int64_t>& ptr,
              std::vector<int64_t>& idx) {
  std::vector<std::vector<int64_t>> per(rows);
  for (const auto& x : e) {
    if (x.first < 0 || x.first >= rows || x.second < 0 || x.second >= cols)
      return set_error(GF2C_ERR_INVALID_ARG, "edge out of bounds");
    per[x.first].push_back(x.second);
  }
  ptr.assign(1, 0);
  idx.clear();
  for (auto& r : per) {
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    idx.insert(idx.end(), r.begin(), r.end());
    ptr.push_back((int64_t)idx.size());
  }
  return GF2C_OK;
}

int read_sparse_any(const std::string& s, int fmt, int64_t& rows, int64_t& cols, std::vector<int64_t>& ptr,
                    std::vector<int64_t>& idx, int& tag_out) {
  if (fmt < 0) fmt = detect_format(s);
  if (fmt == 2) return set_error(GF2C_ERR_INVALID_ARG, "hex format not supported for sparse matrices");
  if (fmt < 0) return set_error(GF2C_ERR_INVALID_ARG, "unable to detect file format");
  if (fmt == 0) {
    Parsed p;
    int rc = parse_binary(s, p);
    if (rc) return rc;
    tag_out = p.tag;
    int64_t nnz;
    if (p.tag == 3) {
      std::string f;
      if ((rc = check_type(p, 3, "SpBitMatrix")) || (rc = meta_int(p.meta, "rows", rows)) ||
          (rc = meta_int(p.meta, "cols", cols)) || (rc = meta_int(p.meta, "nnz", nnz)))
        return rc;
      if (!meta_value(p.meta, "format", f) || f != "coo") return set_error(GF2C_ERR_INVALID_ARG, "expected COO format");
      if ((int64_t)p.payload.size() != nnz * 8) return set_error(GF2C_ERR_INVALID_ARG, "SpBitMatrix data length mismatch");
      std::vector<std::pair<int64_t, int64_t>> e(nnz);
      for (int64_t i = 0; i < nnz; i++) e[i] = {(int64_t)get_le(p.payload, 8 * i, 4), (int64_t)get_le(p.payload, 8 * i + 4, 4)};
      return csr_dedup(rows, cols, e, ptr, idx);
    }
    if (p.tag == 4) {
      if ((rc = check_type(p, 4, "SpBitMatrixDual")) || (rc = meta_int(p.meta, "rows", rows)) ||
          (rc = meta_int(p.meta, "cols", cols)) || (rc = meta_int(p.meta, "nnz", nnz)))
        return rc;
      if ((int64_t)p.payload.size() != (rows + 1 + nnz + cols + 1 + nnz) * 4)
        return set_error(GF2C_ERR_INVALID_ARG, "SpBitMatrixDual data length mismatch");
      ptr.resize(rows + 1);
      idx.resize(nnz);
      for (int64_t i = 0; i <= rows; i++) ptr[i] = (int64_t)get_le(p.payload, 4 * i, 4);
      for (int64_t i = 0; i < nnz; i++) idx[i] = (int64_t)get_le(p.payload, 4 * (rows + 1 + i), 4);
      if (ptr[0] != 0 || ptr[rows] != nnz) return set_error(GF2C_ERR_INVALID_ARG, "SpBitMatrixDual row offsets are invalid");
      for (int64_t r = 0; r < rows; r++) {
        if (ptr[r + 1] < ptr[r]) return set_error(GF2C_ERR_INVALID_ARG, "SpBitMatrixDual row offsets are invalid");
        for (int64_t e = ptr[r]; e < ptr[r + 1]; e++)
          if (idx[e] < 0 || idx[e] >= cols || (e > ptr[r] && idx[e] <= idx[e - 1]))
            return set_error(GF2C_ERR_INVALID_ARG, "SpBitMatrixDual columns are not sorted / in range");
      }
      return GF2C_OK;
    }
    return set_error(GF2C_ERR_INVALID_ARG, "expected a sparse matrix type tag");
  }
  const auto L = lines_of(s);
  if (L.empty()) return set_error(GF2C_ERR_INVALID_ARG, "empty sparse matrix file");
  const auto d = ints_of(L[0]);
  if (d.size() != 3) return set_error(GF2C_ERR_INVALID_ARG, "sparse text must start with 'rows cols nnz'");
  rows = d[0];
  cols = d[1];
  std::vector<std::pair<int64_t, int64_t>> e;
  for (size_t li = 1; li < L.size() && (int64_t)e.size() < d[2]; li++) {
    if (L[li].empty()) continue;
    const auto rc = ints_of(L[li]);
    if (rc.size() != 2) return set_error(GF2C_ERR_INVALID_ARG, "invalid edge line");
    e.push_back({rc[0], rc[1]});
  }
  if ((int64_t)e.size() != d[2]) return set_error(GF2C_ERR_INVALID_ARG, "sparse text has fewer edges than nnz");
  tag_out = 3;
  return csr_dedup(rows, cols, e, ptr, idx);
}

std::string sparse_text(int64_t rows, int64_t cols, const int64_t* ptr, const int64_t* idx) {
  std::string out = std::to_string(rows) + " " + std::to_string(cols) + " " + std::to_string(ptr[rows]) + "\n";
  for (int64_t r = 0; r < rows; r++)
    for (int64_t e = ptr[r]; e < ptr[r + 1]; e++) out += std::to_string(r) + " " + std::to_string(idx[e]) + "\n";
  return out;
}

int check_csr(int64_t rows, int64_t cols, const int64_t* ptr, const int64_t* idx) {
  if (rows < 0 || cols < 0 || !ptr || (ptr[rows] > 0 && !idx)) return set_error(GF2C_ERR_INVALID_ARG, "bad CSR arguments");
  if (ptr[0] != 0) return set_error(GF2C_ERR_INVALID_ARG, "CSR row offsets must start at 0");
  for (int64_t r = 0; r < rows; r++) {
    if (ptr[r + 1] < ptr[r]) return set_error(GF2C_ERR_INVALID_ARG, "CSR row offsets must not decrease");
    for (int64_t e = ptr[r]; e < ptr[r + 1]; e++)
      if (idx[e] < 0 || idx[e] >= cols || (e > ptr[r] && idx[e] <= idx[e - 1]))
        return set_error(GF2C_ERR_INVALID_ARG, "CSR columns must be ascending and in range");
  }
  if (rows > 0xffffffffLL || cols > 0xffffffffLL || ptr[rows] > 0xffffffffLL)
    return set_error(GF2C_ERR_UNSUPPORTED, "sparse files store u32 indices");
  return GF2C_OK;
}

}  // namespace

extern "C" {

int gf2c_siphash13(const void* data, int64_t len, uint64_t k0, uint64_t k1, uint64_t* out) {
  if (!out || len < 0 || (len > 0 && !data)) return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  Sip13 h(k0, k1);
  h.write((const uint8_t*)data, (size_t)len);
  *out = h.finish();
  return GF2C_OK;
}

int gf2c_io_probe(const char* path, int32_t* type_tag, int32_t* format, int64_t* dims3) {
  std::string s;
  int rc = read_file(path, s);
  if (rc) return rc;
  const int fmt = detect_format(s);
  if (format) *format = fmt;
  if (fmt < 0) return set_error(GF2C_ERR_INVALID_ARG, "unable to detect file format");
  int64_t d[3] = {0, 0, 0};
  int tag = 0;
  if (fmt == 0) {
    Parsed p;
    if ((rc = parse_binary(s, p))) return rc;
    tag = p.tag;
    if (tag == 1) {
      if ((rc = meta_int(p.meta, "len_bits", d[0]))) return rc;
    } else {
      if ((rc = meta_int(p.meta, "rows", d[0])) || (rc = meta_int(p.meta, "cols", d[1]))) return rc;
      if (tag >= 3 && (rc = meta_int(p.meta, "nnz", d[2]))) return rc;
    }
  } else {
    const auto L = lines_of(s);
    const auto v = L.empty() ? std::vector<int64_t>() : ints_of(L[0]);
    if (v.empty() || v.size() > 3) return set_error(GF2C_ERR_INVALID_ARG, "unrecognised text header");
    tag = v.size() == 1 ? 1 : v.size() == 2 ? 2 : 3;
    for (size_t i = 0; i < v.size(); i++) d[i] = v[i];
  }
  if (type_tag) *type_tag = tag;
  if (dims3) std::memcpy(dims3, d, sizeof d);
  return GF2C_OK;
}

int gf2c_io_write_bitvec(const char* path, const uint64_t* words, int64_t len_bits, int32_t format) {
  if (len_bits < 0 || (len_bits > 0 && !words) || format < 0 || format > 2)
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  const int64_t W = words_of(len_bits);
  std::vector<uint64_t> w(words, words + W);
  if (len_bits & 63) w[W - 1] &= (1ull << (len_bits & 63)) - 1ull;
  std::string out;
  if (format == 0) {
    const std::string meta = "{\"type\":\"BitVec\",\"len_bits\":" + std::to_string(len_bits) + ",\"version\":1}";
    std::string payload;
    for (uint64_t x : w) put_le(payload, x, 8);
    out = binary_file(1, meta, payload);
  } else if (format == 1) {
    out = std::to_string(len_bits) + "\n";
    for (int64_t c = 0; c < len_bits; c += 80) {
      for (int64_t i = c; i < std::min<int64_t>(len_bits, c + 80); i++) out.push_back(bit_of(w.data(), i) ? '1' : '0');
      out.push_back('\n');
    }
  } else {
    out = std::to_string(len_bits) + "\n";
    for (uint64_t x : w) out += hex_word(x) + "\n";
  }
  return write_file(path, out);
}

int gf2c_io_read_bitvec(const char* path, uint64_t* words, int64_t cap_words, int64_t* len_bits) {
  std::string s;
  int rc = read_file(path, s);
  if (rc) return rc;
  std::vector<uint64_t> w;
  int64_t len = 0;
  if ((rc = read_bitvec_any(s, w, len))) return rc;
  if (len_bits) *len_bits = len;
  if (words) {
    if ((int64_t)w.size() > cap_words) return set_error(GF2C_ERR_INVALID_ARG, "output buffer too small");
    std::memcpy(words, w.data(), w.size() * 8);
  }
  return GF2C_OK;
}

int gf2c_io_write_bitmatrix(const char* path, const uint64_t* words, int64_t rows, int64_t cols, int32_t format) {
  if (rows < 0 || cols < 0 || (rows * words_of(cols) > 0 && !words) || format < 0 || format > 2)
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  const int64_t S = words_of(cols);
  const uint64_t tail = (cols & 63) ? (1ull << (cols & 63)) - 1ull : ~0ull;
  auto word = [&](int64_t r, int64_t w) { return w == S - 1 ? words[r * S + w] & tail : words[r * S + w]; };
  std::string out;
  if (format == 0) {
    const std::string meta = "{\"type\":\"BitMatrix\",\"rows\":" + std::to_string(rows) + ",\"cols\":" +
                             std::to_string(cols) + ",\"version\":1}";
    std::string payload;
    payload.reserve((size_t)(rows * S * 8));
    for (int64_t r = 0; r < rows; r++)
      for (int64_t w = 0; w < S; w++) put_le(payload, word(r, w), 8);
    out = binary_file(2, meta, payload);
  } else {
    out = std::to_string(rows) + " " + std::to_string(cols) + "\n";
    for (int64_t r = 0; r < rows; r++) {
      if (format == 1)
        for (int64_t c = 0; c < cols; c++) out.push_back(((words[r * S + (c >> 6)] >> (c & 63)) & 1) ? '1' : '0');
      else
        for (int64_t w = 0; w < S; w++) out += hex_word(word(r, w));
      out.push_back('\n');
    }
  }
  return write_file(path, out);
}

int gf2c_io_read_bitmatrix(const char* path, int32_t format, uint64_t* words, int64_t cap_words, int64_t* rows,
                           int64_t* cols) {
  if (format < -1 || format > 2) return set_error(GF2C_ERR_INVALID_ARG, "bad format");
  std::string s;
  int rc = read_file(path, s);
  if (rc) return rc;
  std::vector<uint64_t> w;
  int64_t r = 0, c = 0;
  if ((rc = read_bitmatrix_fmt(s, format, w, r, c))) return rc;
  if (rows) *rows = r;
  if (cols) *cols = c;
  if (words) {
    if ((int64_t)w.size() > cap_words) return set_error(GF2C_ERR_INVALID_ARG, "output buffer too small");
    std::memcpy(words, w.data(), w.size() * 8);
  }
  return GF2C_OK;
}

int gf2c_io_write_sparse(const char* path, int32_t type_tag, int64_t rows, int64_t cols, const int64_t* row_ptr,
                         const int64_t* col_idx, int32_t format) {
  if ((type_tag != 3 && type_tag != 4) || (format != 0 && format != 1))
    return set_error(GF2C_ERR_INVALID_ARG, "sparse files: type 3 or 4, binary or text format");
  int rc = check_csr(rows, cols, row_ptr, col_idx);
  if (rc) return rc;
  if (format == 1) return write_file(path, sparse_text(rows, cols, row_ptr, col_idx));
  const int64_t nnz = row_ptr[rows];
  std::string payload, meta;
  if (type_tag == 3) {
    meta = "{\"type\":\"SpBitMatrix\",\"rows\":" + std::to_string(rows) + ",\"cols\":" + std::to_string(cols) +
           ",\"nnz\":" + std::to_string(nnz) + ",\"format\":\"coo\",\"version\":1}";
    for (int64_t r = 0; r < rows; r++)
      for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; e++) {
        put_le(payload, (uint64_t)r, 4);
        put_le(payload, (uint64_t)col_idx[e], 4);
      }
  } else {
    meta = "{\"type\":\"SpBitMatrixDual\",\"rows\":" + std::to_string(rows) + ",\"cols\":" + std::to_string(cols) +
           ",\"nnz\":" + std::to_string(nnz) + ",\"version\":1}";
    // CSC with rows ascending (the stable transpose)
    std::vector<int64_t> cptr(cols + 1, 0), cidx(nnz);
    for (int64_t e = 0; e < nnz; e++) cptr[col_idx[e] + 1]++;
    for (int64_t c = 0; c < cols; c++) cptr[c + 1] += cptr[c];
    std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1);
    for (int64_t r = 0; r < rows; r++)
      for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; e++) cidx[fill[col_idx[e]]++] = r;
    for (int64_t i = 0; i <= rows; i++) put_le(payload, (uint64_t)row_ptr[i], 4);
    for (int64_t i = 0; i < nnz; i++) put_le(payload, (uint64_t)col_idx[i], 4);
    for (int64_t i = 0; i <= cols; i++) put_le(payload, (uint64_t)cptr[i], 4);
    for (int64_t i = 0; i < nnz; i++) put_le(payload, (uint64_t)cidx[i], 4);
  }
  return write_file(path, binary_file(type_tag, meta, payload));
}

int gf2c_io_read_sparse(const char* path, int32_t format, int64_t* rows, int64_t* cols, int64_t* nnz,
                        int64_t* row_ptr, int64_t* col_idx, int64_t cap_nnz) {
  if (format < -1 || format > 2) return set_error(GF2C_ERR_INVALID_ARG, "bad format");
  std::string s;
  int rc = read_file(path, s);
  if (rc) return rc;
  int64_t r = 0, c = 0;
  std::vector<int64_t> ptr, idx;
  int tag = 0;
  if ((rc = read_sparse_any(s, format, r, c, ptr, idx, tag))) return rc;
  if (rows) *rows = r;
  if (cols) *cols = c;
  if (nnz) *nnz = (int64_t)idx.size();
  if (row_ptr) std::memcpy(row_ptr, ptr.data(), ptr.size() * 8);
  if (col_idx) {
    if ((int64_t)idx.size() > cap_nnz) return set_error(GF2C_ERR_INVALID_ARG, "output buffer too small");
    std::memcpy(col_idx, idx.data(), idx.size() * 8);
  }
  return GF2C_OK;
}

int gf2c_code_create_file(const char* path, gf2c_code** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  std::string s;
  int rc = read_file(path, s);
  if (rc) return rc;
  int64_t r = 0, c = 0;
  std::vector<int64_t> ptr, idx;
  int tag = 0;
  if ((rc = read_sparse_any(s, -1, r, c, ptr, idx, tag))) return rc;
  std::vector<int64_t> pairs;
  pairs.reserve(2 * idx.size());
  for (int64_t row = 0; row < r; row++)
    for (int64_t e = ptr[row]; e < ptr[row + 1]; e++) {
      pairs.push_back(row);
      pairs.push_back(idx[e]);
    }
  return gf2c_code_create_edges(r, c, pairs.data(), (int64_t)idx.size(), out);
}

int gf2c_io_write_code(const char* path, const gf2c_code* code, int32_t type_tag, int32_t format) {
  if (!code) return set_error(GF2C_ERR_INVALID_ARG, "code is NULL");
  const HostCode& h = *code->h;
  return gf2c_io_write_sparse(path, type_tag, h.m, h.n, h.row_ptr.data(), h.row_idx.data(), format);
}

int gf2c_code_cache_hash(const gf2c_code* code, uint64_t* hash) {
  if (!code || !hash) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  const HostCode& h = *code->h;
  Sip13 s(0, 0);
  s.write_u64((uint64_t)h.m);
  s.write_u64((uint64_t)h.n);
  s.write_u64((uint64_t)h.row_idx.size());
  int count = 0;
  for (int64_t r = 0; r < h.m && count < 100; r++)
    for (int64_t e = h.row_ptr[r]; e < h.row_ptr[r + 1] && count < 100; e++, count++) {
      s.write_u64((uint64_t)r);
      s.write_u64((uint64_t)h.row_idx[e]);
    }
  *hash = s.finish();
  return GF2C_OK;
}

int gf2c_code_parity_part(const gf2c_code* code, uint64_t* words) {
  if (!code || !words) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  HostCode& h = *code->h;
  const int64_t k = h.k, r = h.n - h.k, S = words_of(r);
  std::memset(words, 0, (size_t)(k * S * 8));
  if (h.kind == 2) {
    // DVB-T2: the parity of message bit i is the prefix XOR, over the staircase,
    // of the indicator of the checks of column i
    if (h.m != r) return set_error(GF2C_ERR_KERNEL, "internal: DVB-T2 parity length");
    for (int64_t i = 0; i < k; i++) {
      uint64_t* row = words + i * S;
      for (int64_t e = h.col_ptr[i]; e < h.col_ptr[i + 1]; e++) row[h.col_idx[e] >> 6] ^= 1ull << (h.col_idx[e] & 63);
      uint64_t carry = 0;
      for (int64_t w = 0; w < S; w++) {
        uint64_t x = row[w];
        x ^= x << 1;
        x ^= x << 2;
        x ^= x << 4;
        x ^= x << 8;
        x ^= x << 16;
        x ^= x << 32;
        x ^= carry;
        row[w] = x;
        carry = (x >> 63) ? ~0ull : 0ull;
      }
      if (r & 63) row[S - 1] &= (1ull << (r & 63)) - 1ull;
    }
    return GF2C_OK;
  }
  int rc = prepare_encoder(h);
  if (rc) return rc;
  for (int64_t i = 0; i < k; i++)
    if (h.enc_msg_cols[i] != i)
      return set_error(GF2C_ERR_UNSUPPORTED, "the code's systematic form does not put the message in columns [0, k)");
  const int64_t Wm = (h.m + 63) / 64;
  for (int64_t j = 0; j < (int64_t)h.enc_par_cols.size(); j++) {
    const int64_t q = h.enc_par_cols[j] - k;  // parity bit index of pivot j
    for (int64_t i = 0; i < k; i++)
      if ((h.enc_p[(size_t)i * Wm + (j >> 6)] >> (j & 63)) & 1) words[i * S + (q >> 6)] |= 1ull << (q & 63);
  }
  return GF2C_OK;
}

}  // extern "C"
