// Star join with bitmap join indexes: the index writer, the index's code decode, and the
// star join's row fix-up and gathers (include/alenka_b200.h).
//
// An index segment holds, for every row of one fact segment, the dimension attribute
// that the row's foreign key reaches, dictionary-coded: the sorted distinct values, then
// the codes bit-packed MSB first, 64 / bits codes a word (emit_create_bitmap_index
// operators.cu:2188-2268, compress_int cm.cu:4271-4336). The engine keeps the codes of
// each index segment resident at 8, 16 or 32 bits and tests them as sets of codes, so a
// star join's filter is one scan of the fact table like any other FILTER.
#include <algorithm>
#include <cmath>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace {

constexpr int kT = 256;

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

int grid_for(uint64_t n) {
  uint64_t b = (n + kT - 1) / kT;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 16));
}

// First position p in [0, m) whose key is not below v, m when there is none: the binary
// search of std::lower_bound and thrust::lower_bound (halve the range, step past the
// middle when it is below), so that an unsorted key column gives the reference's
// positions too.
__device__ __forceinline__ uint32_t lower_bound_i64(const int64_t* keys, uint32_t m, int64_t v) {
  uint32_t first = 0, len = m;
  while (len > 0) {
    const uint32_t half = len >> 1, mid = first + half;
    if (keys[mid] < v) {
      first = mid + 1;
      len = len - half - 1;
    } else {
      len = half;
    }
  }
  return first;
}

// The same search over a dimension column stored FOR (value = stored + lower).
__device__ __forceinline__ uint32_t lower_bound_for(const alk_colseg& keys, int64_t v) {
  uint32_t first = 0, len = keys.rows;
  while (len > 0) {
    const uint32_t half = len >> 1, mid = first + half;
    if (alkd::load_for(keys.data, keys.bits, keys.lower, mid) < v) {
      first = mid + 1;
      len = len - half - 1;
    } else {
      len = half;
    }
  }
  return first;
}

// First position p in [0, d) with heads[p] > i (heads ascending).
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* heads, uint32_t d, uint32_t i) {
  uint32_t first = 0, len = d;
  while (len > 0) {
    const uint32_t half = len >> 1, mid = first + half;
    if (heads[mid] <= i) {
      first = mid + 1;
      len = len - half - 1;
    } else {
      len = half;
    }
  }
  return first;
}

// out[i] = vals[lower_bound(keys, fk[i])] for i < n (operators.cu:2227-2236), then the
// tail values after them (the char form appends the dimension's hashes beyond n,
// operators.cu:2244-2260). A key past the last dimension key sets err bit 0.
__global__ void __launch_bounds__(kT) k_index_lookup(const int64_t* fk, uint32_t n, const int64_t* keys, uint32_t m,
                                                     const int64_t* vals, const int64_t* tail, uint32_t ntail,
                                                     int64_t* out, int* err) {
  const uint64_t total = (uint64_t)n + ntail;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < total; i += (uint64_t)gridDim.x * kT) {
    if (i < n) {
      const uint32_t p = lower_bound_i64(keys, m, fk[i]);
      if (p >= m) {
        atomicOr(err, 1);
        out[i] = 0;
      } else {
        out[i] = vals[p];
      }
    } else {
      out[i] = tail[i - n];
    }
  }
}

// Head flags of the sorted values: 1 where a new distinct value starts.
__global__ void __launch_bounds__(kT) k_index_heads(const int64_t* vals, const uint32_t* perm, uint32_t n,
                                                    uint64_t* flags) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    flags[i] = (i == 0 || vals[perm[i]] != vals[perm[i - 1]]) ? 1 : 0;
}

// Code of every value = its distinct value's rank (the std::map order of compress_int,
// cm.cu:4284-4296); the dictionary entry is written by the head of its run.
__global__ void __launch_bounds__(kT) k_index_codes(const int64_t* vals, const uint32_t* perm, uint32_t n,
                                                    const uint32_t* heads, uint32_t d, uint32_t* codes,
                                                    int64_t* dict) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const uint32_t code = upper_bound_u32(heads, d, (uint32_t)i) - 1;
    const uint32_t r = perm[i];
    codes[r] = code;
    if (heads[code] == (uint32_t)i) dict[code] = vals[r];
  }
}

// Word w holds codes w*fit .. w*fit+fit-1, the first in the highest bits; a last partial
// word is shifted up the same way (cm.cu:4314-4333).
__global__ void __launch_bounds__(kT) k_index_pack(const uint32_t* codes, uint32_t n, uint32_t bits, uint32_t fit,
                                                   uint32_t words, unsigned long long* out) {
  for (uint64_t w = blockIdx.x * (uint64_t)kT + threadIdx.x; w < words; w += (uint64_t)gridDim.x * kT) {
    unsigned long long v = 0;
    for (uint32_t j = 0; j < fit; j++) {
      const uint64_t i = w * fit + j;
      if (i < n) v |= (unsigned long long)codes[i] << ((fit - 1 - j) * bits);
    }
    out[w] = v;
  }
}

// Code of row i, as cmp_functor_dict reads it (filter.cu:30-50), stored at out_bits.
__global__ void __launch_bounds__(kT) k_index_decode(const unsigned long long* words, uint32_t rows, uint32_t bits,
                                                     uint32_t fit, void* out, uint32_t out_bits) {
  const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * kT) {
    const uint64_t w = i / fit;
    const uint32_t loc = (uint32_t)(i % fit);
    const uint32_t c = (uint32_t)((words[w] >> ((fit - loc - 1) * bits)) & mask);
    if (out_bits == 8) ((uint8_t*)out)[i] = (uint8_t)c;
    else if (out_bits == 16) ((uint16_t*)out)[i] = (uint16_t)c;
    else ((uint32_t*)out)[i] = c;
  }
}

// The star join's row list per fact segment (star_join operators.cu:541-552): the list
// is resized to the survivor count and then filled by copy_if over rows [0, n - 1), so a
// surviving last row is never written and its entry keeps what the list held from the
// previous segment with survivors at that position (0 past its end). One thread walks the
// segments in order, since each segment reads what the previous one left.
__global__ void k_star_fixup(uint32_t* rowid, const uint64_t* offs, const uint64_t* counts, const uint32_t* rows,
                             uint32_t nseg) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint64_t prev_off = 0, prev_size = 0;
  for (uint32_t g = 0; g < nseg; g++) {
    const uint64_t cnt = counts[g];
    if (!cnt) continue;
    const uint64_t off = offs[g];
    if (rows[g] && rowid[off + cnt - 1] == rows[g] - 1)
      rowid[off + cnt - 1] = (cnt - 1 < prev_size) ? rowid[prev_off + cnt - 1] : 0u;
    prev_off = off;
    prev_size = cnt;
  }
}

// Values of the star join's output rows, read from the stored segment payloads as the
// star join reads the segment files (operators.cu:576-650, 678-731): 8-bit values through
// a signed char, 16 and 32-bit ones unsigned, then the header's lower bound added.
// For a fact column, out = that value. For a dimension column the value is a foreign key:
// t = (uint32)value, plus (uint32)(lower - 1) when lower != 1, and out = the dimension
// column's value at lower_bound(dimension keys, t), both read at their stored widths
// (star_join's lower_bound path). A row past its segment sets err bit 1, a key past the
// dimension's keys err bit 0.
__global__ void __launch_bounds__(kT) k_star_gather(const alk_colseg* segs, const uint32_t* rowid,
                                                    const uint32_t* seg, uint64_t n, bool dim, alk_colseg keys,
                                                    alk_colseg vals, int64_t* out, int* err) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const alk_colseg cs = segs[seg[i]];
    const uint32_t r = rowid[i];
    if (r >= cs.rows) {
      atomicOr(err, 2);
      out[i] = 0;
      continue;
    }
    int64_t raw;
    switch (cs.bits) {
      case 8: raw = (int64_t)(int8_t)((const uint8_t*)cs.data)[r]; break;
      case 16: raw = (int64_t)((const uint16_t*)cs.data)[r]; break;
      case 32: raw = (int64_t)((const uint32_t*)cs.data)[r]; break;
      default: raw = ((const int64_t*)cs.data)[r]; break;
    }
    if (!dim) {
      out[i] = (int64_t)((uint64_t)raw + (uint64_t)cs.lower);
      continue;
    }
    uint32_t t = (uint32_t)raw;
    if (cs.lower != 1) t += (uint32_t)(cs.lower - 1);
    const uint32_t p = lower_bound_for(keys, (int64_t)t);
    if (p >= keys.rows) {
      atomicOr(err, 1);
      out[i] = 0;
    } else {
      out[i] = alkd::load_for(vals.data, vals.bits, vals.lower, p);
    }
  }
}

// Stream-ordered scratch owned by one entry-point call.
struct Scratch {
  cudaStream_t s;
  std::vector<void*> p;
  explicit Scratch(cudaStream_t st) : s(st) {}
  ~Scratch() {
    for (void* x : p) cudaFreeAsync(x, s);
  }
  template <class T>
  T* get(size_t n, cudaError_t* e) {
    void* x = nullptr;
    *e = cudaMallocAsync(&x, std::max<size_t>(n * sizeof(T), 16), s);
    if (*e == cudaSuccess) p.push_back(x);
    return (T*)x;
  }
};

}  // namespace

extern "C" {

int alk_bitmap_index_build(const int64_t* d_fk, uint32_t n, const int64_t* d_keys, uint32_t m, const int64_t* d_vals,
                           const int64_t* d_tail, uint32_t ntail, int64_t* h_dict, uint32_t* h_dict_n,
                           uint64_t* h_words, uint32_t* h_words_n, uint32_t* h_bits, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const uint64_t total = (uint64_t)n + ntail;
  if (!h_dict || !h_dict_n || !h_words || !h_words_n || !h_bits || total == 0 || total > 0xFFFFFFFFull)
    return ALK_ERR_ARG;
  if (n && (!d_fk || !d_keys || !d_vals || m == 0)) return ALK_ERR_ARG;
  if (ntail && !d_tail) return ALK_ERR_ARG;
  const uint32_t N = (uint32_t)total;
  Scratch sc(s);
  cudaError_t e;
  int64_t* vals = sc.get<int64_t>(N, &e);
  CK(e);
  uint32_t* perm = sc.get<uint32_t>(N, &e);
  CK(e);
  uint64_t* flags = sc.get<uint64_t>(N, &e);
  CK(e);
  uint32_t* heads = sc.get<uint32_t>(N, &e);
  CK(e);
  uint32_t* codes = sc.get<uint32_t>(N, &e);
  CK(e);
  int64_t* dict = sc.get<int64_t>(N, &e);
  CK(e);
  int* err = sc.get<int>(1, &e);
  CK(e);
  CK(cudaMemsetAsync(err, 0, sizeof(int), s));
  k_index_lookup<<<grid_for(N), kT, 0, s>>>(d_fk, n, d_keys, m, d_vals, d_tail, ntail, vals, err);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  int h_err = 0;
  CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (h_err) return ALK_ERR_UNSUPPORTED;  // the reference would gather past its key column
  // sorted distinct values: a stable sort, head flags, their positions, then each value's rank
  const int64_t* keyp = vals;
  const uint8_t desc = 0;
  int rc = alk_sort_perm(&keyp, &desc, 1, N, perm, stream);
  if (rc) return rc;
  k_index_heads<<<grid_for(N), kT, 0, s>>>(vals, perm, N, flags);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  uint64_t d = 0;
  rc = alk_flags_compact(flags, N, heads, &d, stream);
  if (rc) return rc;
  k_index_codes<<<grid_for(N), kT, 0, s>>>(vals, perm, N, heads, (uint32_t)d, codes, dict);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  // bits and words as compress_int computes them (cm.cu:4298-4312)
  const uint32_t bits = (uint32_t)std::ceil(std::log2(double(d + 1)));
  if (bits == 0 || bits > 32) return ALK_ERR_ARG;
  const uint32_t fit = 64 / bits;
  uint32_t words = N / fit;
  if (!words || N % fit) words++;
  unsigned long long* packed = sc.get<unsigned long long>(words, &e);
  CK(e);
  k_index_pack<<<grid_for(words), kT, 0, s>>>(codes, N, bits, fit, words, packed);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h_dict, dict, d * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h_words, packed, (size_t)words * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *h_dict_n = (uint32_t)d;
  *h_words_n = words;
  *h_bits = bits;
  return ALK_OK;
}

int alk_bitmap_index_decode(const uint64_t* d_words, uint32_t rows, uint32_t bits, uint32_t fit_count, void* d_out,
                            uint32_t out_bits, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (rows == 0) return ALK_OK;
  if (!d_words || !d_out || bits == 0 || bits > 32 || fit_count != 64 / bits) return ALK_ERR_ARG;
  if (out_bits != 8 && out_bits != 16 && out_bits != 32) return ALK_ERR_ARG;
  if (bits > out_bits) return ALK_ERR_ARG;
  k_index_decode<<<grid_for(rows), kT, 0, s>>>((const unsigned long long*)d_words, rows, bits, fit_count, d_out,
                                               out_bits);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_star_rows_fixup(uint32_t* d_rowid, const uint64_t* h_seg_counts, const uint32_t* h_seg_rows, uint32_t nseg,
                        alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nseg == 0) return ALK_OK;
  if (!d_rowid || !h_seg_counts || !h_seg_rows) return ALK_ERR_ARG;
  std::vector<uint64_t> host(3 * (size_t)nseg);
  uint64_t off = 0;
  for (uint32_t g = 0; g < nseg; g++) {
    host[g] = off;
    host[nseg + g] = h_seg_counts[g];
    host[2 * (size_t)nseg + g] = h_seg_rows[g];
    off += h_seg_counts[g];
  }
  Scratch sc(s);
  cudaError_t e;
  uint64_t* dv = sc.get<uint64_t>(2 * (size_t)nseg, &e);
  CK(e);
  uint32_t* dr = sc.get<uint32_t>(nseg, &e);
  CK(e);
  std::vector<uint32_t> rows(h_seg_rows, h_seg_rows + nseg);
  CK(cudaMemcpyAsync(dv, host.data(), 2 * (size_t)nseg * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dr, rows.data(), (size_t)nseg * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  k_star_fixup<<<1, 1, 0, s>>>(d_rowid, dv, dv + nseg, dr, nseg);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_star_gather(const alk_colseg* segs, uint32_t nseg, const uint32_t* d_rowid, const uint32_t* d_seg, uint64_t n,
                    const alk_colseg* dim_key, const alk_colseg* dim_val, int64_t* d_out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return ALK_OK;
  if (!segs || nseg == 0 || !d_rowid || !d_seg || !d_out) return ALK_ERR_ARG;
  if (!dim_key != !dim_val) return ALK_ERR_ARG;
  auto bad = [](const alk_colseg& c) {
    return (c.bits != 8 && c.bits != 16 && c.bits != 32 && c.bits != 64) || (c.rows && !c.data);
  };
  for (uint32_t g = 0; g < nseg; g++)
    if (bad(segs[g])) return ALK_ERR_ARG;
  alk_colseg kd{}, vd{};
  if (dim_key) {
    kd = *dim_key;
    vd = *dim_val;
    if (bad(kd) || bad(vd) || kd.rows == 0 || vd.rows != kd.rows) return ALK_ERR_ARG;
  }
  Scratch sc(s);
  cudaError_t e;
  alk_colseg* ds = sc.get<alk_colseg>(nseg, &e);
  CK(e);
  int* err = sc.get<int>(1, &e);
  CK(e);
  CK(cudaMemcpyAsync(ds, segs, (size_t)nseg * sizeof(alk_colseg), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(err, 0, sizeof(int), s));
  k_star_gather<<<grid_for(n), kT, 0, s>>>(ds, d_rowid, d_seg, n, dim_key != nullptr, kd, vd, d_out, err);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  int h_err = 0;
  CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return h_err ? ALK_ERR_UNSUPPORTED : ALK_OK;
}

}  // extern "C"
