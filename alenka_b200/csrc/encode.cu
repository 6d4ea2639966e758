// Segment writer on the GPU: one column segment of int64 values encoded into the
// reference's segment file image, byte for byte what pfor_compress (FOR, byte-aligned
// width, compress.cu:413-527) and pfor_delta_compress (adjacent differences, the first
// replaced by the second, minus their minimum, packed MSB-first, compress.cu:271-408)
// write, so that STORE ... BINARY runs at device speed.
//
// Two passes over the values, both streaming: statistics (minimum and maximum of the
// values and of the adjacent differences, and whether the values are sorted), then the
// packing of the payload.
//
// Batched form (alk_encode_segments_device): the segments of a call go, in groups small
// enough to stay in L2 between the two passes, through four launches per group
// (statistics identities, statistics, plan, pack), with one synchronisation at the end. The plan picks the width on the device: the reference
// computes ceil(log2((double)span)), which equals the exact bit length of span - 1 for
// every span up to 2^46 (log2 of the nearest integers to a power of two is then at least
// 2.8 units in the last place away from the integer), and FOR widths above 32 bits are
// all written as 64. The remaining cases (a delta range above 2^46, a value range of
// 2^63 or more) go through the single-segment path.
//
// Single-segment path: between the two passes the host reads the statistics and picks
// the width with the same function as the host writer, so the two writers cannot
// disagree on it. The statistics are kept in the first bytes of the caller's output image
// until the header overwrites them: that path allocates nothing.
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

// ---- batched form
constexpr int kEncItems = 8;  // independent loads in flight per thread
constexpr uint32_t kEncTile = kEncThreads * kEncItems;  // values per tile of the batched passes

struct EncSeg {
  const int64_t* v;
  uint8_t* img;
  uint32_t n, tile0;  // values; first tile of the segment in the call's tile space
};
struct EncPlan {  // statistics, then the plan the pack pass follows
  long long vmin, vmax, dmin, dmax, first, last;
  unsigned int unsorted;
  uint32_t status;  // 0 planned; 1 the single-segment path must write it
  long long lo;     // subtracted value (FOR: minimum; delta: minimum difference)
  uint32_t comp, bits, fit, cnt;
  unsigned long long len;
};

__device__ __forceinline__ uint32_t seg_of_tile(const EncSeg* segs, uint32_t count, uint32_t tile) {
  uint32_t lo = 0, hi = count;  // segs[lo].tile0 <= tile < segs[hi].tile0
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (segs[mid].tile0 <= tile) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_enc_plan_init(const EncSeg* segs, uint32_t count, EncPlan* plans) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  EncPlan& p = plans[i];
  p.vmin = LLONG_MAX;
  p.vmax = LLONG_MIN;
  p.dmin = LLONG_MAX;
  p.dmax = LLONG_MIN;
  p.first = segs[i].v[0];
  p.last = segs[i].v[segs[i].n - 1];
  p.unsorted = 0;
  p.status = 0;
}

// Statistics of every tile: a thread per value, coalesced, with the previous value read
// by a second coalesced load (it hits L1). kDiffs false (FOR forced): values only.
template <bool kDiffs>
__global__ void __launch_bounds__(kEncThreads) k_enc_stats_batch(const EncSeg* __restrict__ segs, uint32_t count,
                                                                 uint32_t ntiles, EncPlan* plans) {
  __shared__ long long sh[4][kEncThreads / 32];
  __shared__ unsigned int su[kEncThreads / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long vmin = LLONG_MAX, vmax = LLONG_MIN, dmin = LLONG_MAX, dmax = LLONG_MIN;
  unsigned int uns = 0;
  uint32_t cur = 0xffffffffu;  // segment whose partials the threads hold
  // the block's partials go to the segment's plan when the block moves on to another
  // segment and at the end: one set of atomics per block and segment
  auto flush = [&]() {
    warp_minmax(vmin, vmax);
    warp_minmax(dmin, dmax);
    uns = __any_sync(0xffffffffu, uns) ? 1u : 0u;
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
        EncPlan& pl = plans[cur];
        atomicMin(&pl.vmin, vmin);
        atomicMax(&pl.vmax, vmax);
        if (dmin <= dmax) {
          atomicMin(&pl.dmin, dmin);
          atomicMax(&pl.dmax, dmax);
        }
        if (uns) atomicOr(&pl.unsorted, 1u);
      }
    }
    __syncthreads();  // the shared partials are rewritten by the next flush
    vmin = LLONG_MAX;
    vmax = LLONG_MIN;
    dmin = LLONG_MAX;
    dmax = LLONG_MIN;
    uns = 0;
  };
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t si = seg_of_tile(segs, count, tile);
    if (si != cur) {
      if (cur != 0xffffffffu) flush();
      cur = si;
    }
    const EncSeg sg = segs[si];
    const uint64_t t0 = (uint64_t)(tile - sg.tile0) * kEncTile;
    const uint64_t t1 = min((uint64_t)sg.n, t0 + kEncTile);
    // a warp takes 32 x kEncItems consecutive values: kEncItems independent coalesced
    // loads per lane, and as many for the previous values (they hit L1)
    const uint64_t b = t0 + (uint64_t)w * 32 * kEncItems;
    if (b >= t1) continue;
    long long x[kEncItems], p[kEncItems];
    if (b + 32 * kEncItems <= t1 && b > 0) {  // no bound and no first value inside
#pragma unroll
      for (int k = 0; k < kEncItems; k++) {
        x[k] = sg.v[b + k * 32 + lane];
        if (kDiffs) p[k] = sg.v[b + k * 32 + lane - 1];
      }
#pragma unroll
      for (int k = 0; k < kEncItems; k++) {
        vmin = min(vmin, x[k]);
        vmax = max(vmax, x[k]);
        if (kDiffs) {
          const long long d = (long long)((unsigned long long)x[k] - (unsigned long long)p[k]);
          dmin = min(dmin, d);
          dmax = max(dmax, d);
          uns |= x[k] < p[k] ? 1u : 0u;
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < kEncItems; k++) {
        const uint64_t i = b + k * 32 + lane;
        x[k] = i < t1 ? sg.v[i] : 0;
        p[k] = (kDiffs && i < t1 && i > 0) ? sg.v[i - 1] : 0;
      }
#pragma unroll
      for (int k = 0; k < kEncItems; k++) {
        const uint64_t i = b + k * 32 + lane;
        if (i < t1) {
          vmin = min(vmin, x[k]);
          vmax = max(vmax, x[k]);
          if (kDiffs && i > 0) {
            const long long d = (long long)((unsigned long long)x[k] - (unsigned long long)p[k]);
            dmin = min(dmin, d);
            dmax = max(dmax, d);
            uns |= x[k] < p[k] ? 1u : 0u;
          }
        }
      }
    }
  }
  if (cur != 0xffffffffu) flush();
}

__device__ void put_bytes(uint8_t* dst, const void* src, int n) {
  for (int k = 0; k < n; k++) dst[k] = ((const uint8_t*)src)[k];
}

// One thread per segment: the width and layout, then the header and trailer (the same
// fields in the same order as the host writer's segment_image).
__global__ void k_enc_plan(const EncSeg* segs, uint32_t count, int mode, EncPlan* plans) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  EncPlan& p = plans[i];
  const uint32_t n = segs[i].n;
  const bool delta = mode == 1 || (mode == 2 && !p.unsorted);
  const long long lo = delta ? (n > 1 ? p.dmin : p.first) : p.vmin;
  const long long hi = delta ? (n > 1 ? p.dmax : p.first) : p.vmax;
  const unsigned long long span = (unsigned long long)hi - (unsigned long long)lo + 1ull;
  uint32_t bits;
  if (span - 1 >= (1ull << 46)) {  // above 2^46, or a range of 2^64 values (span 0)
    if (delta || span == 0 || span > (unsigned long long)LLONG_MAX) {
      p.status = 1;
      return;
    }
    bits = 64;  // FOR: every width above 32 bits is written as 64
  } else {
    bits = span == 1 ? 0 : 64 - __clzll((long long)(span - 1));
  }
  uint64_t cnt;
  long long lower, upper, start = 0;
  if (delta) {
    if (bits == 0) bits = 1;
    p.fit = 64 / bits;
    cnt = ((uint64_t)n + p.fit - 1) / p.fit * 8;
    lower = p.first;
    upper = p.last;
    start = p.first;
  } else {
    bits = bits <= 8 ? 8 : bits <= 16 ? 16 : bits <= 32 ? 32 : 64;
    p.fit = 64 / bits;
    cnt = (uint64_t)n * (bits / 8);
    lower = p.vmin;
    upper = p.vmax;
  }
  if (cnt > 0xffffffffull) {  // the format's u32 payload size
    p.status = 1;
    return;
  }
  p.lo = lo;
  p.comp = delta ? 1 : 0;
  p.bits = bits;
  p.cnt = (uint32_t)cnt;
  p.len = alk::kSegHeadBytes + cnt + alk::kSegTailBytes;
  uint8_t* img = segs[i].img;
  const uint32_t c32 = p.cnt, comp = p.comp, rec = n, fit = p.fit;
  const long long orig = lo;
  put_bytes(img, &c32, 4);
  put_bytes(img + 4, &lower, 8);
  put_bytes(img + 12, &upper, 8);
  put_bytes(img + 20, &comp, 4);
  uint8_t* t = img + alk::kSegHeadBytes + cnt;
  put_bytes(t, &c32, 4);
  put_bytes(t + 4, &rec, 4);
  put_bytes(t + 8, &bits, 4);
  put_bytes(t + 12, &orig, 8);
  put_bytes(t + 20, &fit, 4);
  put_bytes(t + 24, &start, 8);
}

// Payload of every planned segment. FOR: a thread per value, each store at the value's
// own width (coalesced; the payload starts 24 bytes into an 8-byte aligned image). Delta:
// a thread per 64-bit word whose first value lies in the tile.
__global__ void __launch_bounds__(kEncThreads) k_enc_pack_batch(const EncSeg* __restrict__ segs, uint32_t count,
                                                                uint32_t ntiles, const EncPlan* __restrict__ plans) {
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t si = seg_of_tile(segs, count, tile);
    const EncPlan& p = plans[si];
    if (p.status) continue;
    const EncSeg sg = segs[si];
    const uint64_t t0 = (uint64_t)(tile - sg.tile0) * kEncTile;
    const uint64_t t1 = min((uint64_t)sg.n, t0 + kEncTile);
    uint8_t* out = sg.img + alk::kSegHeadBytes;
    const uint64_t lo = (uint64_t)p.lo;
    if (p.comp == 0) {
      const uint32_t bits = p.bits;
      for (uint64_t b = t0 + threadIdx.x; b < t1; b += kEncThreads * kEncItems) {
        uint64_t d[kEncItems];
#pragma unroll
        for (int k = 0; k < kEncItems; k++) {
          const uint64_t i = b + (uint64_t)k * kEncThreads;
          d[k] = i < t1 ? (uint64_t)sg.v[i] - lo : 0;
        }
#pragma unroll
        for (int k = 0; k < kEncItems; k++) {
          const uint64_t i = b + (uint64_t)k * kEncThreads;
          if (i >= t1) break;
          if (bits == 8) out[i] = (uint8_t)d[k];
          else if (bits == 16) reinterpret_cast<uint16_t*>(out)[i] = (uint16_t)d[k];
          else if (bits == 32) reinterpret_cast<uint32_t*>(out)[i] = (uint32_t)d[k];
          else reinterpret_cast<uint64_t*>(out)[i] = d[k];
        }
      }
    } else {
      const uint32_t fit = p.fit, bits = p.bits, n = sg.n;
      const uint64_t w0 = (t0 + fit - 1) / fit, w1 = (t1 + fit - 1) / fit;
      for (uint64_t w = w0 + threadIdx.x; w < w1; w += kEncThreads) {
        uint64_t word = 0;
        const uint64_t i0 = w * fit;
        // the word's values and the one before them, loaded before any is used
        uint64_t prev = i0 == 0 ? (n > 1 ? (uint64_t)sg.v[0] - ((uint64_t)sg.v[1] - (uint64_t)sg.v[0]) : 0)
                                : (uint64_t)sg.v[i0 - 1];
#pragma unroll 8
        for (uint32_t j = 0; j < fit; j++) {
          const uint64_t i = i0 + j;
          const uint64_t x = i < n ? (uint64_t)sg.v[i] : prev;
          const uint64_t d = (i == 0 && n == 1) ? x : x - prev;
          if (i < n) word += (d - lo) << (64 - bits - j * bits);
          prev = x;
        }
        reinterpret_cast<uint64_t*>(out)[w] = word;
      }
    }
  }
}

// Blocks of a batched pass: one per tile up to what the GPU holds at once (tiles are
// small, so the blocks that take one tile more than others finish soon after).
template <class K>
int resident_grid(K kernel, uint64_t tiles) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kEncThreads, 0);
  const uint64_t most = (uint64_t)std::max(1, sms) * (uint64_t)std::max(1, per);
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(tiles, most));
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

// Many segments, one synchronisation: see the batched form above. Segments that the
// device plan leaves to the single-segment path (or that hold no values) are written
// by alk_encode_segment_device after the batch.
extern "C" int alk_encode_segments_device(const int64_t* const* d_values, const uint32_t* n, uint32_t count, int mode,
                                          void* const* d_images, const size_t* caps, size_t* h_lens,
                                          alk_stream stream) {
  if (count == 0) return ALK_OK;
  if (!d_values || !n || !d_images || !caps || !h_lens || mode < 0 || mode > 2) return ALK_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<EncSeg> segs;
  std::vector<uint32_t> which;  // call index of each batched segment
  std::vector<uint32_t> alone;  // segments written one at a time
  uint64_t tiles = 0;
  int rc = ALK_OK;
  for (uint32_t i = 0; i < count; i++) {
    if (!d_images[i] || ((uintptr_t)d_images[i] & 7) || (n[i] && (!d_values[i] || ((uintptr_t)d_values[i] & 7))))
      return ALK_ERR_ARG;
    const size_t worst = alk::kSegHeadBytes + (size_t)n[i] * 8 + alk::kSegTailBytes;
    if (caps[i] < worst) {  // the batch writes before it knows the size: room for the largest
      h_lens[i] = worst;
      rc = ALK_ERR_OVERFLOW;
      continue;
    }
    if (n[i] == 0) {
      alone.push_back(i);
      continue;
    }
    segs.push_back(EncSeg{d_values[i], (uint8_t*)d_images[i], n[i], 0});
    which.push_back(i);
    tiles += (n[i] + kEncTile - 1) / kEncTile;
  }
  if (rc != ALK_OK) return rc;
  if (tiles > 0xffffffffull) return ALK_ERR_ARG;
  // groups of consecutive segments whose values fit in L2 together: a group's pack pass
  // re-reads what its statistics pass just brought into L2. Tiles count from each
  // group's first segment.
  constexpr uint64_t kGroupBytes = 48ull << 20;
  struct Group {
    uint32_t first, count, tiles;
  };
  std::vector<Group> groups;
  {
    uint64_t bytes = 0;
    for (uint32_t k = 0; k < segs.size(); k++) {
      const uint64_t b = (uint64_t)segs[k].n * 8;
      if (groups.empty() || bytes + b > kGroupBytes) {
        groups.push_back(Group{k, 0, 0});
        bytes = 0;
      }
      Group& g = groups.back();
      segs[k].tile0 = g.tiles;
      g.tiles += (segs[k].n + kEncTile - 1) / kEncTile;
      g.count++;
      bytes += b;
    }
  }
  if (!segs.empty()) {
    const uint32_t m = (uint32_t)segs.size();
    void* work = nullptr;
    const size_t seg_bytes = (sizeof(EncSeg) * m + 255) & ~size_t(255);
    cudaError_t e = cudaMallocAsync(&work, seg_bytes + sizeof(EncPlan) * m, s);
    if (e != cudaSuccess) return alk::cuda_fail(e);
    EncSeg* d_segs = (EncSeg*)work;
    EncPlan* d_plans = (EncPlan*)((uint8_t*)work + seg_bytes);
    std::vector<EncPlan> plans(m);
    e = cudaMemcpyAsync(d_segs, segs.data(), sizeof(EncSeg) * m, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      static const int g_stats0 = resident_grid(k_enc_stats_batch<false>, ~0ull);
      static const int g_stats1 = resident_grid(k_enc_stats_batch<true>, ~0ull);
      static const int g_pack = resident_grid(k_enc_pack_batch, ~0ull);
      for (const Group& gr : groups) {  // four launches per group, no host round trip
        const EncSeg* gs = d_segs + gr.first;
        EncPlan* gp = d_plans + gr.first;
        const int pb = (int)((gr.count + 127) / 128);
        k_enc_plan_init<<<pb, 128, 0, s>>>(gs, gr.count, gp);
        if (mode == 0)
          k_enc_stats_batch<false><<<std::min<int>(g_stats0, (int)gr.tiles), kEncThreads, 0, s>>>(gs, gr.count,
                                                                                                gr.tiles, gp);
        else
          k_enc_stats_batch<true><<<std::min<int>(g_stats1, (int)gr.tiles), kEncThreads, 0, s>>>(gs, gr.count,
                                                                                               gr.tiles, gp);
        k_enc_plan<<<pb, 128, 0, s>>>(gs, gr.count, mode, gp);
        k_enc_pack_batch<<<std::min<int>(g_pack, (int)gr.tiles), kEncThreads, 0, s>>>(gs, gr.count, gr.tiles, gp);
        alk::g_kernel_launches += 4;
      }
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(plans.data(), d_plans, sizeof(EncPlan) * m, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the segment table is read until here
    cudaFreeAsync(work, s);
    if (e != cudaSuccess) return alk::cuda_fail(e);
    for (uint32_t k = 0; k < m; k++) {
      if (plans[k].status) alone.push_back(which[k]);
      else h_lens[which[k]] = (size_t)plans[k].len;
    }
  }
  for (uint32_t i : alone) {
    size_t len = 0;
    const int r = alk_encode_segment_device(d_values[i], n[i], mode, d_images[i], caps[i], &len, stream);
    h_lens[i] = len;
    if (r != ALK_OK) return r;
  }
  return ALK_OK;
}
