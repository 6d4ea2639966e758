// String predicates and ordering on char columns. LIKE: The reference evaluates LIKE once per dictionary entry with
// gpu_regex (filter.cu:67-129) over the column's dictionary file, keeps the matching
// codes, and then tests each row's code against them (filter.cu:454-500). Here the
// matches become a bitmap over the codes, built by one thread per entry, and the rows'
// test is the register machine's ALK_OP_INSET (a bit lookup that stays in L1/L2).
#include "internal.h"

namespace {
constexpr uint32_t kLikeMaxPattern = 256;  // pattern bytes including the terminator

struct LikeArgs {
  const char* dict;
  uint32_t width;
  uint64_t count;
  uint32_t* bits;
  char pattern[kLikeMaxPattern];
};

// One entry against the NUL-terminated pattern: '%' any run of characters, '?' any
// character except '.', every other pattern character itself. The entry ends at its first
// NUL or at the width, and at most `width` characters are examined in all, each retry one
// character further after a '%' counting as one: the reference's matcher bounds its
// single character counter that way.
__device__ bool like_entry(const char* entry, uint32_t width, const char* pat) {
  bool after_pct = false;
  uint32_t seen = 0;
  const char* from = entry;
  const char* pfrom = pat;
  for (;;) {
    const char* s = from;
    const char* p = pfrom;
    int how = 0;  // 0 entry exhausted, 1 restart after '%', 2 mismatch
    while (seen < width && *s) {
      if (*p == '%') {
        after_pct = true;
        from = s;
        pfrom = p + 1;
        while (*pfrom == '%') ++pfrom;
        if (!*pfrom) return true;
        how = 1;
        break;
      }
      if (*p == '?' ? *s == '.' : *s != *p) {
        how = 2;
        break;
      }
      ++s;
      ++p;
      ++seen;
    }
    if (how == 1) continue;
    if (how == 0) {
      while (*p == '%') ++p;
      return *p == 0;
    }
    if (!after_pct) return false;
    ++from;
    ++seen;
  }
}

// A warp covers 32 consecutive entries: its ballot is one word of the bitmap.
__global__ void k_like_dict(const __grid_constant__ LikeArgs a) {
  __shared__ char pat[kLikeMaxPattern];
  for (uint32_t i = threadIdx.x; i < kLikeMaxPattern; i += blockDim.x) pat[i] = a.pattern[i];
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t words = (a.count + 31) / 32;
  for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; base < words * 32;
       base += stride) {
    const uint64_t k = base + (threadIdx.x & 31);
    const bool m = k < a.count && like_entry(a.dict + k * a.width, a.width, pat);
    const uint32_t word = __ballot_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) a.bits[1 + base / 32] = word;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.bits[0] = (uint32_t)a.count;
}
__global__ void k_code_lookup(const int64_t* __restrict__ codes, uint64_t n, const int64_t* __restrict__ table,
                              uint64_t table_n, int64_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t c = codes[i];
    out[i] = (c >= 0 && (uint64_t)c < table_n) ? __ldg(table + c) : -1;
  }
}
}  // namespace

extern "C" int alk_code_lookup(const int64_t* d_codes, uint64_t n, const int64_t* d_table, uint64_t table_n,
                               int64_t* d_out, alk_stream stream) {
  if (n == 0) return ALK_OK;
  if (!d_codes || !d_table || !d_out) return ALK_ERR_ARG;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148ull * 8));
  k_code_lookup<<<grid, 256, 0, (cudaStream_t)stream>>>(d_codes, n, d_table, table_n, d_out);
  alk::g_kernel_launches++;
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ALK_OK : alk::cuda_fail(e);
}

extern "C" int alk_like_dictionary(const char* d_dict, uint32_t width, uint64_t count, const char* pattern,
                                   uint32_t pattern_len, uint32_t* d_bits, alk_stream stream) {
  if (!pattern || !d_bits || pattern_len >= kLikeMaxPattern || count > 0xffffffffull || (count && (!d_dict || !width)))
    return ALK_ERR_ARG;
  LikeArgs a{};
  a.dict = d_dict;
  a.width = width;
  a.count = count;
  a.bits = d_bits;
  for (uint32_t i = 0; i < pattern_len; i++) a.pattern[i] = pattern[i];  // the rest stays NUL
  const uint64_t threads = ((count + 31) / 32) * 32;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((threads + 255) / 256, 148ull * 8));
  k_like_dict<<<grid, 256, 0, (cudaStream_t)stream>>>(a);
  alk::g_kernel_launches++;
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ALK_OK : alk::cuda_fail(e);
}
