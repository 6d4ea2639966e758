// Shared pieces of the scan kernels: tile geometry, conjunct tests rewritten on the stored
// (frame-of-reference) values of a segment, loads of stored values, and the mbarrier and
// bulk-copy helpers of the producer/consumer tile pipelines. Included by the kernel
// translation units; everything is internal to each.
#pragma once
#include <stdint.h>

#include "../../include/alenka_b200.h"
#include "device.cuh"

namespace {
using namespace alkd;

constexpr int kT = 256;
constexpr int kItems = 8;
constexpr int kTile = kT * kItems;
constexpr int kMaxConj = 4;
constexpr uint32_t kWaitLimit = 1u << 22;

struct Conj {
  int64_t mul, k;
  uint32_t slot, op;
};
enum : uint32_t { kCjGeneric = 0, kCjIn = 1, kCjOut = 2, kCjNever = 3, kCjAlways = 4 };
struct ConjSeg {
  uint64_t lo, span;  // kCjIn: x - lo <= span (unsigned); kCjOut: its negation
  uint32_t mode, pad;
};

// Raw-domain form of `(x + lower) * mul OP k` over the stored values x of one segment
// (0 <= x < 2^bits). Exact whenever mul == 1 and no decoded value can wrap; otherwise
// the kernels evaluate the conjunct on the decoded value (kCjGeneric).
ConjSeg conj_seg(const Conj& cj, const alk_colseg& d) {
  ConjSeg r{0, 0, kCjGeneric, 0};
  if (cj.mul != 1 || d.bits >= 64) return r;
  const __int128 xmax = ((__int128)1 << d.bits) - 1;
  if ((__int128)d.lower + xmax > (__int128)INT64_MAX) return r;
  const __int128 t = (__int128)cj.k - d.lower;  // value OP k  <=>  x OP t
  __int128 lo = 0, hi = xmax;
  bool out = false;
  switch (cj.op) {
    case ALK_OP_LT: hi = t - 1; break;
    case ALK_OP_LE: hi = t; break;
    case ALK_OP_GT: lo = t + 1; break;
    case ALK_OP_GE: lo = t; break;
    case ALK_OP_EQ: lo = hi = t; break;
    case ALK_OP_NE: lo = hi = t; out = true; break;
    default: return r;
  }
  if (lo < 0) lo = 0;
  if (hi > xmax) hi = xmax;
  if (lo > hi) {
    r.mode = out ? kCjAlways : kCjNever;
    return r;
  }
  r.mode = out ? kCjOut : kCjIn;
  r.lo = (uint64_t)lo;
  r.span = (uint64_t)(hi - lo);
  return r;
}

template <uint32_t kOp>
__device__ __forceinline__ uint32_t cmp_items(const uint64_t (&x)[kItems], uint64_t lower, int64_t mul, int64_t c,
                                              uint32_t live) {
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    const int64_t v = wrap_mul((int64_t)(x[k] + lower), mul);
    bool ok;
    if (kOp == ALK_OP_LT) ok = v < c;
    else if (kOp == ALK_OP_GT) ok = v > c;
    else if (kOp == ALK_OP_LE) ok = v <= c;
    else if (kOp == ALK_OP_GE) ok = v >= c;
    else if (kOp == ALK_OP_EQ) ok = v == c;
    else ok = v != c;
    if (!ok) live &= ~(1u << k);
  }
  return live;
}

// Applies one conjunct to the thread's items (stored values x of one segment).
__device__ __forceinline__ uint32_t conj_filter(const Conj& cj, const ConjSeg& cs, int64_t lower,
                                                const uint64_t (&x)[kItems], uint32_t live) {
  switch (cs.mode) {
    case kCjAlways: return live;
    case kCjNever: return 0;
    case kCjIn:
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if (x[k] - cs.lo > cs.span) live &= ~(1u << k);
      return live;
    case kCjOut:
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if (x[k] - cs.lo <= cs.span) live &= ~(1u << k);
      return live;
    default:
      switch (cj.op) {
        case ALK_OP_LT: return cmp_items<ALK_OP_LT>(x, (uint64_t)lower, cj.mul, cj.k, live);
        case ALK_OP_GT: return cmp_items<ALK_OP_GT>(x, (uint64_t)lower, cj.mul, cj.k, live);
        case ALK_OP_LE: return cmp_items<ALK_OP_LE>(x, (uint64_t)lower, cj.mul, cj.k, live);
        case ALK_OP_GE: return cmp_items<ALK_OP_GE>(x, (uint64_t)lower, cj.mul, cj.k, live);
        case ALK_OP_EQ: return cmp_items<ALK_OP_EQ>(x, (uint64_t)lower, cj.mul, cj.k, live);
        default: return cmp_items<ALK_OP_NE>(x, (uint64_t)lower, cj.mul, cj.k, live);
      }
  }
}

// 32-bit forms for segments whose staged columns store at most 32 bits: range tests and
// bitmap indexes on the stored values need no 64-bit arithmetic.
__device__ __forceinline__ uint32_t conj_filter32(const Conj& cj, const ConjSeg& cs, int64_t lower,
                                                  const uint32_t (&x)[kItems], uint32_t live) {
  const uint32_t lo = (uint32_t)cs.lo, span = (uint32_t)cs.span;
  switch (cs.mode) {
    case kCjAlways: return live;
    case kCjNever: return 0;
    case kCjIn:
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if (x[k] - lo > span) live &= ~(1u << k);
      return live;
    case kCjOut:
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if (x[k] - lo <= span) live &= ~(1u << k);
      return live;
    default: {
      uint64_t w[kItems];
#pragma unroll
      for (int k = 0; k < kItems; k++) w[k] = x[k];
      return conj_filter(cj, cs, lower, w, live);
    }
  }
}
template <int kStride>
__device__ __forceinline__ void load_raw32(const void* p, uint32_t bits, uint32_t i0, uint32_t (&x)[kItems]) {
  switch (bits) {
    case 8: {
      const uint8_t* q = (const uint8_t*)p + i0;
#pragma unroll
      for (int k = 0; k < kItems; k++) x[k] = q[k * kStride];
    } break;
    case 16: {
      const uint16_t* q = (const uint16_t*)p + i0;
#pragma unroll
      for (int k = 0; k < kItems; k++) x[k] = q[k * kStride];
    } break;
    default: {
      const uint32_t* q = (const uint32_t*)p + i0;
#pragma unroll
      for (int k = 0; k < kItems; k++) x[k] = q[k * kStride];
    } break;
  }
}

// Stored values of one column for the thread's items (elements i0 + k * kStride); from
// global memory only the live items are read.
template <bool kGlobal, int kStride, class T>
__device__ __forceinline__ void load_raw_t(const T* p, uint32_t live, uint64_t (&x)[kItems]) {
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    if (kGlobal) x[k] = ((live >> k) & 1) ? (uint64_t)__ldg(p + k * kStride) : 0;
    else x[k] = (uint64_t)p[k * kStride];
  }
}
template <bool kGlobal, int kStride = kT>
__device__ __forceinline__ void load_raw(const void* p, uint32_t bits, uint64_t i0, uint32_t live,
                                         uint64_t (&x)[kItems]) {
  switch (bits) {
    case 8: load_raw_t<kGlobal, kStride>((const uint8_t*)p + i0, live, x); break;
    case 16: load_raw_t<kGlobal, kStride>((const uint16_t*)p + i0, live, x); break;
    case 32: load_raw_t<kGlobal, kStride>((const uint32_t*)p + i0, live, x); break;
    default: load_raw_t<kGlobal, kStride>((const unsigned long long*)p + i0, live, x); break;
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait of one thread for a phase; false when the limit expired.
// (Used by the producers, which mostly wait for a consumer to free a stage: they back
// off quickly so that their polling takes few issue slots from the consumers.)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t spins = 0; spins < kWaitLimit; spins++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (spins > 2) __nanosleep(128);
  }
  return false;
}
// Bounded wait of a whole warp; the outcome is the same in every lane.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity) {
  bool done = false;
  for (uint32_t spins = 0; spins < kWaitLimit; spins++) {
    if (!done) done = mbar_try_wait(bar, parity);
    if (__all_sync(0xffffffffu, done)) return true;
    if (spins > 16) __nanosleep(32);
  }
  return false;
}

}  // namespace
