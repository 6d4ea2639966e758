// Text loader: a LOAD ... USING (sep) AS (...) source parsed on the device
// (CudaSet::LoadBigFile, cm.cu:1852-2080, with the functors of cm.h:341-660). The file's
// records are its newline-terminated lines; each line's requested fields are cut at the
// separator (a double quote toggles a quoted span in which the separator does not cut;
// the quote characters stay in the field, NUL bytes are dropped) into a 23-byte slot,
// and each slot is parsed as the reference parses it: integers (gpu_atoll), decimals at a
// fixed number of fraction digits (gpu_atold) and yyyy-mm-dd dates (gpu_date), a column
// being a date column when its first record's slot has '-' at offset 4.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"

namespace {
constexpr int kT = 256;
constexpr uint32_t kSlot = 23;         // the reference's numeric field slot (max_len)
constexpr uint32_t kMaxTextCols = 32;  // columns of one LOAD
constexpr uint32_t kChunk = 1024;      // bytes a thread scans for newlines

struct TextArgs {
  const char* text;
  uint64_t n;
  char sep;
  uint32_t ncols;
  uint32_t field[kMaxTextCols];  // 0-based field of declared column i (the i-th smallest)
  uint32_t kind[kMaxTextCols];   // 0 integer, 1 decimal, 2 date, 3 fixed-width text
  uint32_t scale[kMaxTextCols];  // decimal: digits after the point; text: the width
  void* out[kMaxTextCols];       // int64 values, or width bytes a record
  const unsigned long long* nl;  // newline positions
  uint64_t rows;
};

// The field walk of parse_functor (cm.h:599-650) for one record starting at pos: each
// requested field, in increasing field order, is found as the bytes [b, e) up to the
// separator outside double quotes (the quote state runs on across the record's fields)
// and handed to visit(index, b, e). Reads stop at the end of the text.
template <class Visit>
__host__ __device__ inline void cut_fields(const char* text, uint64_t n, uint64_t pos, char sep, uint32_t ncols,
                                           const uint32_t* field, Visit&& visit) {
  uint32_t cur = 0, want = 0;
  bool quoted = false;
  uint64_t j = pos;
  while (want < ncols) {
    const uint64_t b = j;
    while (j < n && (text[j] != sep || quoted)) {
      if (text[j] == '"') quoted = !quoted;
      j++;
    }
    if (field[want] == cur) visit(want++, b, j);
    j++;  // past the separator
    cur++;
  }
}

// A field's bytes into a zero-filled slot of w bytes, NUL bytes dropped (the reference's
// dest slot; bytes beyond w, which it lets run into the next record's slot, are dropped).
__host__ __device__ inline void fill_slot(const char* text, uint64_t b, uint64_t e, char* slot, uint32_t w) {
  uint32_t t = 0;
  for (uint64_t k = b; k < e && t < w; k++)
    if (text[k] != 0) slot[t++] = text[k];
  for (; t < w; t++) slot[t] = 0;
}

// gpu_atoll (cm.h:543-597)
__host__ __device__ inline int64_t parse_int(const char* s) {
  uint32_t i = 0;
  int c;
  do {
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  } while (c == ' ');
  bool neg = false;
  if (c == '-') {
    neg = true;
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  } else if (c == '+') {
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  }
  uint64_t acc = 0;
  for (;; i++) {
    if (c < '0' || c > '9') break;
    acc = neg ? acc * 10 - (uint64_t)(c - '0') : acc * 10 + (uint64_t)(c - '0');
    c = i < kSlot ? (unsigned char)s[i] : 0;
  }
  return (int64_t)acc;
}

// gpu_atold (cm.h:480-541): digits until `scale` digits follow the point (a '.' starts
// the count; the count is tested after every digit, before the point as well), then
// scaled by 10^(scale - digits after the point)
__host__ __device__ inline int64_t parse_decimal(const char* s, uint32_t scale) {
  uint32_t i = 0;
  int c;
  do {
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  } while (c == ' ');
  bool neg = false;
  if (c == '-') {
    neg = true;
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  } else if (c == '+') {
    c = i < kSlot ? (unsigned char)s[i] : 0;
    i++;
  }
  uint64_t acc = 0;
  uint32_t point = 0;
  bool frac = false;
  for (;; i++) {
    if (c >= '0' && c <= '9') {
      acc = neg ? acc * 10 - (uint64_t)(c - '0') : acc * 10 + (uint64_t)(c - '0');
      if (frac) point++;
      if (point == scale) break;
    } else if (c == '.') {
      frac = true;
    } else {
      break;
    }
    c = i < kSlot ? (unsigned char)s[i] : 0;
  }
  uint64_t mul = 1;
  for (uint32_t k = point; k < scale; k++) mul *= 10;  // scale <= 9: an exact power
  return (int64_t)(acc * mul);
}

// gpu_date (cm.h:341-371): the slot's first ten bytes, every byte but '-' taken as a
// digit (c - '0', unchecked)
__host__ __device__ inline int64_t parse_date(const char* s) {
  uint64_t acc = 0;
  for (uint32_t z = 0; z < 10; z++) {
    const int c = (unsigned char)s[z];
    if (c != '-') acc = acc * 10 + (uint64_t)(int64_t)(c - '0');
  }
  return (int64_t)acc;
}

// The first record's slots: a numeric column whose slot has '-' at offset 4 is a date
// column.
struct DateProbe {
  const char* text;
  uint32_t* kind;
  uint32_t* mask;
  __host__ __device__ void operator()(uint32_t c, uint64_t b, uint64_t e) const {
    char slot[kSlot];
    fill_slot(text, b, e, slot, kSlot);
    if (kind[c] != 3 && slot[4] == '-') {
      kind[c] = 2;
      if (mask) *mask |= 1u << c;
    }
  }
};

// MurmurHash64A (MurmurHash2_64.cu:201-242) of each record's w bytes, halved: the
// per-row values of a char column's .hash file (compress_char, cm.cu:1808-1812).
__global__ void __launch_bounds__(kT) k_hash_strings(const uint8_t* chars, uint64_t n, uint32_t w, uint32_t seed,
                                                     uint64_t* out) {
  const uint64_t m = 0xc6a4a7935bd1e995ull;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const uint8_t* p = chars + i * w;
    uint64_t h = seed ^ ((uint64_t)w * m);
    uint32_t k = 0;
    for (; k + 8 <= w; k += 8) {
      uint64_t x = 0;
      for (int b = 7; b >= 0; b--) x = (x << 8) | p[k + b];
      x *= m;
      x ^= x >> 47;
      x *= m;
      h ^= x;
      h *= m;
    }
    if (k < w) {
      for (int b = (int)(w - k) - 1; b >= 0; b--) h ^= (uint64_t)p[k + b] << (8 * b);
      h *= m;
    }
    h ^= h >> 47;
    h *= m;
    h ^= h >> 47;
    out[i] = h / 2;
  }
}

// Newline counts of each thread's kChunk bytes.
__global__ void __launch_bounds__(kT) k_nl_count(const char* text, uint64_t n, unsigned long long* counts) {
  const uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x;
  const uint64_t b = t * kChunk;
  if (b >= n) return;
  const uint64_t e = min(n, b + kChunk);
  unsigned long long c = 0;
  for (uint64_t i = b; i < e; i++) c += text[i] == '\n';
  counts[t] = c;
}

// Newline positions, in order: each thread writes its chunk's at its exclusive offset.
__global__ void __launch_bounds__(kT) k_nl_write(const char* text, uint64_t n, const unsigned long long* offsets,
                                                 unsigned long long* pos) {
  const uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x;
  const uint64_t b = t * kChunk;
  if (b >= n) return;
  const uint64_t e = min(n, b + kChunk);
  unsigned long long o = offsets[t];
  for (uint64_t i = b; i < e; i++)
    if (text[i] == '\n') pos[o++] = i;
}

// One record per thread: its fields cut into slots, each parsed by its column's kind.
__global__ void __launch_bounds__(kT) k_text_parse(const __grid_constant__ TextArgs a) {
  for (uint64_t r = blockIdx.x * (uint64_t)kT + threadIdx.x; r < a.rows; r += (uint64_t)gridDim.x * kT) {
    const uint64_t start = r == 0 ? 0 : a.nl[r - 1] + 1;
    cut_fields(a.text, a.n, start, a.sep, a.ncols, a.field, [&](uint32_t c, uint64_t b, uint64_t e) {
      if (a.kind[c] == 3) {
        fill_slot(a.text, b, e, (char*)a.out[c] + r * a.scale[c], a.scale[c]);
        return;
      }
      char slot[kSlot];
      fill_slot(a.text, b, e, slot, kSlot);
      ((int64_t*)a.out[c])[r] = a.kind[c] == 2   ? parse_date(slot)
                                : a.kind[c] == 1 ? parse_decimal(slot, a.scale[c])
                                                 : parse_int(slot);
    });
  }
}
}  // namespace

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

extern "C" {

int alk_text_load(const char* h_text, uint64_t nbytes, char sep, const alk_text_col* cols, uint32_t ncols,
                  void* const* d_out, uint64_t out_cap, uint64_t* h_rows, uint32_t* h_date_mask, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_rows || !cols || ncols == 0 || ncols > kMaxTextCols || (nbytes && !h_text) || !d_out) return ALK_ERR_ARG;
  *h_rows = 0;
  if (h_date_mask) *h_date_mask = 0;
  for (uint32_t c = 0; c < ncols; c++) {
    if (cols[c].field == 0 || cols[c].kind > ALK_TEXT_CHAR || !d_out[c]) return ALK_ERR_ARG;
    if (cols[c].kind == ALK_TEXT_DECIMAL && cols[c].scale > 9) return ALK_ERR_UNSUPPORTED;
    if (cols[c].kind == ALK_TEXT_CHAR && cols[c].width == 0) return ALK_ERR_ARG;
  }
  if (nbytes == 0) return ALK_OK;
  TextArgs a{};
  a.n = nbytes;
  a.sep = sep;
  a.ncols = ncols;
  // declared column i reads the i-th smallest field number (ind[i] = cl[i], cm.cu:1863-1870, 1945)
  std::vector<uint32_t> f(ncols);
  for (uint32_t c = 0; c < ncols; c++) f[c] = cols[c].field - 1;
  std::sort(f.begin(), f.end());
  for (uint32_t c = 0; c < ncols; c++) {
    a.field[c] = f[c];
    a.kind[c] = cols[c].kind == ALK_TEXT_CHAR ? 3 : cols[c].kind == ALK_TEXT_DECIMAL ? 1 : 0;
    a.scale[c] = cols[c].kind == ALK_TEXT_CHAR ? cols[c].width : cols[c].scale;
    a.out[c] = d_out[c];
  }
  // a column is a date column when its first record's slot has '-' at offset 4 (cm.cu:2024-2026)
  DateProbe probe{h_text, a.kind, h_date_mask};
  cut_fields(h_text, nbytes, 0, sep, ncols, a.field, probe);
  const uint64_t threads = (nbytes + kChunk - 1) / kChunk;
  const size_t off_cnt = (nbytes + 255) & ~size_t(255);
  const size_t off_off = off_cnt + ((threads * 8 + 255) & ~size_t(255));
  const size_t off_pos = off_off + ((threads * 8 + 255) & ~size_t(255));
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, off_pos, s));
  CK(cudaMemcpyAsync(db, h_text, nbytes, cudaMemcpyHostToDevice, s));
  a.text = (const char*)db;
  const unsigned blocks = (unsigned)((threads + kT - 1) / kT);
  k_nl_count<<<blocks, kT, 0, s>>>(a.text, nbytes, (unsigned long long*)(db + off_cnt));
  CK(cudaGetLastError());
  // the exclusive offsets of the per-thread counts (threads = bytes / 1 KB: host scan)
  std::vector<unsigned long long> cnt(threads);
  CK(cudaMemcpyAsync(cnt.data(), db + off_cnt, threads * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  unsigned long long run = 0;
  for (auto& x : cnt) {
    const unsigned long long v = x;
    x = run;
    run += v;
  }
  // records: the newline-terminated lines (text after the last newline is not a record)
  const uint64_t rows = run;
  *h_rows = rows;
  if (rows > out_cap || rows == 0) {
    CK(cudaFreeAsync(db, s));
    CK(cudaStreamSynchronize(s));
    return rows > out_cap ? ALK_ERR_OVERFLOW : ALK_OK;
  }
  unsigned long long* nl = nullptr;
  CK(cudaMallocAsync((void**)&nl, rows * 8, s));
  CK(cudaMemcpyAsync(db + off_off, cnt.data(), threads * 8, cudaMemcpyHostToDevice, s));
  k_nl_write<<<blocks, kT, 0, s>>>(a.text, nbytes, (const unsigned long long*)(db + off_off), nl);
  a.nl = nl;
  a.rows = rows;
  const int grid = (int)std::min<uint64_t>((rows + kT - 1) / kT, 148ull * 16);
  k_text_parse<<<grid, kT, 0, s>>>(a);
  alk::g_kernel_launches += 3;
  CK(cudaGetLastError());
  CK(cudaFreeAsync(nl, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_hash_strings(const uint8_t* d_chars, uint64_t n, uint32_t width, uint32_t seed, uint64_t* d_out,
                     alk_stream stream) {
  if (n == 0) return ALK_OK;
  if (!d_chars || !d_out || width == 0) return ALK_ERR_ARG;
  const int grid = (int)std::min<uint64_t>((n + kT - 1) / kT, 148ull * 16);
  k_hash_strings<<<grid, kT, 0, (cudaStream_t)stream>>>(d_chars, n, width, seed, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

}  // extern "C"
