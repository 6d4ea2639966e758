// Segment writer on the GPU: one column segment of int64 values encoded into the
// reference's segment file image, byte for byte what pfor_compress (FOR, byte-aligned
// width, compress.cu:413-527) and pfor_delta_compress (adjacent differences, the first
// replaced by the second, minus their minimum, packed MSB-first, compress.cu:271-408)
// write, so that STORE ... BINARY runs at device speed.
//
// Two passes over the values, both streaming: statistics (minimum and maximum of the
// values and of the adjacent differences, and whether the values are sorted), then the
// packing of the payload. Between them the host reads the statistics and picks the width
// with the same function as the host writer (a double-precision log2, as the reference
// computes it), so the two writers cannot disagree on it. The statistics are kept in the
// first bytes of the caller's output image until the header overwrites them: the entry
// point allocates nothing.
#include <climits>
#include <cstring>
#include <vector>

#include "../host/format.h"
#include "internal.h"

namespace {
constexpr int kEncThreads = 256;

// Scratch statistics at the start of the output image (56 bytes; an image is at least
// 57 bytes when there is a value).
struct EncStats {
  long long vmin, vmax;  // values
  long long dmin, dmax;  // differences v[i] - v[i-1], i >= 1
  long long first, last;
  unsigned int unsorted, pad;
};
static_assert(sizeof(EncStats) == 56, "statistics layout");

__global__ void k_enc_init(const int64_t* v, uint32_t n, EncStats* s) {
  s->vmin = LLONG_MAX;
  s->vmax = LLONG_MIN;
  s->dmin = LLONG_MAX;
  s->dmax = LLONG_MIN;
  s->first = v[0];
  s->last = v[n - 1];
  s->unsorted = 0;
  s->pad = 0;
}

__device__ __forceinline__ void warp_minmax(long long& lo, long long& hi) {
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, (long long)__shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, (long long)__shfl_xor_sync(0xffffffffu, hi, o));
  }
}

__global__ void __launch_bounds__(kEncThreads) k_enc_stats(const int64_t* __restrict__ v, uint32_t n,
                                                           EncStats* s) {
  long long vmin = LLONG_MAX, vmax = LLONG_MIN, dmin = LLONG_MAX, dmax = LLONG_MIN;
  unsigned int uns = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const long long x = v[i];
    vmin = min(vmin, x);
    vmax = max(vmax, x);
    if (i > 0) {
      const long long p = v[i - 1];
      const long long d = (long long)((unsigned long long)x - (unsigned long long)p);
      dmin = min(dmin, d);
      dmax = max(dmax, d);
      uns |= x < p ? 1u : 0u;
    }
  }
  warp_minmax(vmin, vmax);
  warp_minmax(dmin, dmax);
  uns = __any_sync(0xffffffffu, uns) ? 1u : 0u;
  __shared__ long long sh[4][kEncThreads / 32];
  __shared__ unsigned int su[kEncThreads / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][w] = vmin;
    sh[1][w] = vmax;
    sh[2][w] = dmin;
    sh[3][w] = dmax;
    su[w] = uns;
  }
  __syncthreads();
  if (w == 0) {
    const bool in = lane < kEncThreads / 32;
    vmin = in ? sh[0][lane] : LLONG_MAX;
    vmax = in ? sh[1][lane] : LLONG_MIN;
    dmin = in ? sh[2][lane] : LLONG_MAX;
    dmax = in ? sh[3][lane] : LLONG_MIN;
    uns = __any_sync(0xffffffffu, in && su[lane]) ? 1u : 0u;
    warp_minmax(vmin, vmax);
    warp_minmax(dmin, dmax);
    if (lane == 0) {
      atomicMin(&s->vmin, vmin);
      atomicMax(&s->vmax, vmax);
      atomicMin(&s->dmin, dmin);
      atomicMax(&s->dmax, dmax);
      if (uns) atomicOr(&s->unsorted, 1u);
    }
  }
}

// FOR payload: (value - lower) at `bytes` bytes per value, little endian. Each thread
// writes whole 8-byte words; the last, partial word goes byte by byte so that nothing is
// written past the payload.
__global__ void __launch_bounds__(kEncThreads) k_enc_for(const int64_t* __restrict__ v, uint32_t n, int64_t lo,
                                                         uint32_t bytes, uint8_t* __restrict__ out) {
  const uint64_t total = (uint64_t)n * bytes, words = (total + 7) / 8;
  const uint32_t per = 8 / bytes, shift = bytes * 8;
  const uint64_t mask = bytes == 8 ? ~0ull : (1ull << shift) - 1;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
    const uint64_t i0 = (uint64_t)w * per;
    uint64_t word = 0;
    for (uint32_t j = 0; j < per; j++) {
      const uint64_t i = i0 + j;
      if (i < n) word |= (((uint64_t)v[i] - (uint64_t)lo) & mask) << (j * shift);
    }
    if ((w + 1) * 8 <= total) {
      reinterpret_cast<uint64_t*>(out)[w] = word;
    } else {
      for (uint64_t b = 0; w * 8 + b < total; b++) out[w * 8 + b] = (uint8_t)(word >> (8 * b));
    }
  }
}

// FOR-delta payload: word w holds values w * fit ... w * fit + fit - 1, value j of the word
// (difference minus lo) shifted left by 64 - bits - j * bits and summed in, as the
// reference sums the shifted values of a word.
__global__ void __launch_bounds__(kEncThreads) k_enc_delta(const int64_t* __restrict__ v, uint32_t n, int64_t lo,
                                                           uint32_t bits, uint32_t fit, uint64_t* __restrict__ out) {
  const uint64_t words = ((uint64_t)n + fit - 1) / fit;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
    uint64_t word = 0;
    const uint64_t i0 = (uint64_t)w * fit;
    for (uint32_t j = 0; j < fit; j++) {
      const uint64_t i = i0 + j;
      if (i >= n) break;
      const uint64_t d = i == 0 ? (n > 1 ? (uint64_t)v[1] - (uint64_t)v[0] : (uint64_t)v[0])
                                : (uint64_t)v[i] - (uint64_t)v[i - 1];
      word += (d - (uint64_t)lo) << (64 - bits - j * bits);
    }
    out[w] = word;
  }
}

int grid_for_values(uint64_t n) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const uint64_t blocks = (n + kEncThreads - 1) / kEncThreads;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sms * 8));
}
}  // namespace

extern "C" int alk_encode_segment_device(const int64_t* d_values, uint32_t n, int mode, void* d_image, size_t cap,
                                         size_t* h_len, alk_stream stream) {
  if (!h_len || !d_image || mode < 0 || mode > 2 || ((uintptr_t)d_image & 7)) return ALK_ERR_ARG;
  if (n && (!d_values || ((uintptr_t)d_values & 7))) return ALK_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  alk::SegMeta m;
  if (n == 0) {  // no values: the host writer's image for an empty segment
    std::vector<uint8_t> payload;
    alk::encode_for(nullptr, 0, m, payload);
    const std::vector<uint8_t> img = alk::segment_image(m, payload);
    *h_len = img.size();
    if (img.size() > cap) return ALK_ERR_OVERFLOW;
    cudaError_t e = cudaMemcpyAsync(d_image, img.data(), img.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? ALK_OK : alk::cuda_fail(e);
  }
  if (cap < sizeof(EncStats)) {  // room for the statistics: a size that always suffices
    *h_len = alk::kSegHeadBytes + (size_t)n * 8 + alk::kSegTailBytes;
    return ALK_ERR_OVERFLOW;
  }
  EncStats* st = (EncStats*)d_image;
  k_enc_init<<<1, 1, 0, s>>>(d_values, n, st);
  k_enc_stats<<<grid_for_values(n), kEncThreads, 0, s>>>(d_values, n, st);
  alk::g_kernel_launches += 2;
  EncStats h{};
  cudaError_t e = cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return alk::cuda_fail(e);
  // the reference's choice (pfor_compress with its delta switch): mode 2 writes FOR-delta
  // when the values are sorted
  const bool delta = mode == 1 || (mode == 2 && !h.unsorted);
  uint64_t payload_bytes;
  if (delta) {
    // the differences: the first replaced by the second, so their range is that of
    // v[i] - v[i-1] for i >= 1; one value: the value itself
    const int64_t lo = n > 1 ? h.dmin : h.first, hi = n > 1 ? h.dmax : h.first;
    uint32_t bits = alk::range_bits(lo, hi);
    if (bits == 0) bits = 1;
    const uint32_t fit = 64 / bits;
    const uint64_t words = ((uint64_t)n + fit - 1) / fit;
    payload_bytes = words * 8;
    m.lower = h.first;
    m.upper = h.last;
    m.comp_type = 1;
    m.bits = bits;
    m.orig_lower = lo;
    m.fit_count = fit;
    m.start_val = h.first;
  } else {
    uint32_t bits = alk::range_bits(h.vmin, h.vmax);
    if (bits != 8 && bits != 16 && bits != 32 && bits != 64) bits = bits < 8 ? 8 : bits < 16 ? 16 : bits < 32 ? 32 : 64;
    payload_bytes = (uint64_t)n * (bits / 8);
    m.lower = h.vmin;
    m.upper = h.vmax;
    m.comp_type = 0;
    m.bits = bits;
    m.orig_lower = h.vmin;
    m.fit_count = 64 / bits;
    m.start_val = 0;
  }
  const uint64_t len = alk::kSegHeadBytes + payload_bytes + alk::kSegTailBytes;
  *h_len = (size_t)len;
  if (payload_bytes > UINT32_MAX) return ALK_ERR_ARG;  // the format's u32 payload size
  if (len > cap) return ALK_ERR_OVERFLOW;
  m.cnt = (uint32_t)payload_bytes;
  m.rec_count = n;
  uint8_t* out = (uint8_t*)d_image + alk::kSegHeadBytes;
  if (delta) {
    const uint64_t words = payload_bytes / 8;
    k_enc_delta<<<grid_for_values(words), kEncThreads, 0, s>>>(d_values, n, m.orig_lower, m.bits, m.fit_count,
                                                                (uint64_t*)out);
  } else {
    k_enc_for<<<grid_for_values((payload_bytes + 7) / 8), kEncThreads, 0, s>>>(d_values, n, m.lower, m.bits / 8,
                                                                             out);
  }
  alk::g_kernel_launches++;
  const std::vector<uint8_t> frame = alk::segment_image(m, {});  // header then trailer, no payload
  e = cudaMemcpyAsync(d_image, frame.data(), alk::kSegHeadBytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out + payload_bytes, frame.data() + alk::kSegHeadBytes, alk::kSegTailBytes,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host frame is released on return
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? ALK_OK : alk::cuda_fail(e);
}
