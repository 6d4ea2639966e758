// Device-side building blocks shared by the sm_100a kernels: MurmurHash64A,
// FOR decode, the predicate/expression register machine, bounded decoupled
// look-back for ordered single-pass scans, and block/warp scans.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/alenka_b200.h"

namespace alkd {

constexpr uint64_t kMurmurM = 0xc6a4a7935bd1e995ULL;
constexpr uint32_t kSeed = 100;  // hash_seed (bison.y:304)
// Upper bound on polls of a predecessor's status word before a wait gives up and the
// kernel reports ALK_ERR_TIMEOUT (every predecessor is resident, so this only fires
// on a logic error).
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint64_t mm_block(uint64_t h, uint64_t k) {
  k *= kMurmurM;
  k ^= k >> 47;
  k *= kMurmurM;
  h ^= k;
  h *= kMurmurM;
  return h;
}
__device__ __forceinline__ uint64_t mm_final(uint64_t h) {
  h ^= h >> 47;
  h *= kMurmurM;
  h ^= h >> 47;
  return h;
}
// MurmurHash64A (MurmurHash2_64.cu:201-242) of one 8-byte little-endian key.
__device__ __forceinline__ uint64_t murmur_u64(uint64_t key, uint32_t seed = kSeed) {
  return mm_final(mm_block(seed ^ (8ull * kMurmurM), key));
}

__device__ __forceinline__ int64_t wrap_add(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
__device__ __forceinline__ int64_t wrap_sub(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }
__device__ __forceinline__ int64_t wrap_mul(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
// Truncating division; x/0 is defined as 0 and INT64_MIN/-1 wraps (the reference leaves
// both undefined; the oracle uses the same definition).
__device__ __forceinline__ int64_t safe_div(int64_t a, int64_t b) {
  if (b == 0) return 0;
  if (b == -1) return (int64_t)(0 - (uint64_t)a);
  return a / b;
}

// FOR-decoded value i of a column segment: stored width + lower (type_to_int64,
// compress.cu:33-46).
__device__ __forceinline__ int64_t load_for(const void* p, uint32_t bits, int64_t lower, uint64_t i) {
  uint64_t x;
  switch (bits) {
    case 8: x = __ldg((const uint8_t*)p + i); break;
    case 16: x = __ldg((const uint16_t*)p + i); break;
    case 32: x = __ldg((const uint32_t*)p + i); break;
    default: x = __ldg((const unsigned long long*)p + i); break;
  }
  return (int64_t)(x + (uint64_t)lower);
}

__device__ __forceinline__ int64_t vm_apply(uint8_t op, int64_t a, int64_t b) {
  switch (op) {
    case ALK_OP_ADD: return wrap_add(a, b);
    case ALK_OP_SUB: return wrap_sub(a, b);
    case ALK_OP_MUL: return wrap_mul(a, b);
    case ALK_OP_DIV: return safe_div(a, b);
    case ALK_OP_LT: return a < b;
    case ALK_OP_GT: return a > b;
    case ALK_OP_LE: return a <= b;
    case ALK_OP_GE: return a >= b;
    case ALK_OP_EQ: return a == b;
    case ALK_OP_NE: return a != b;
    case ALK_OP_AND: return (a != 0) && (b != 0);
    case ALK_OP_OR: return (a != 0) || (b != 0);
    case ALK_OP_INSET: {  // b: device address of [n, bits...]
      const uint32_t* set = (const uint32_t*)(uintptr_t)b;
      const uint64_t n = __ldg(set);
      return (uint64_t)a < n ? (__ldg(set + 1 + ((uint64_t)a >> 5)) >> (a & 31)) & 1 : 0;
    }
    default: return a;  // MOV
  }
}

// Register machine. Instructions and constants live in shared memory (uniform
// broadcast reads); registers live in shared memory at regs[r * STRIDE] so that the
// dynamic register index never forces local memory. col(slot) returns the current
// row's value of a column slot.
template <int STRIDE, class Col>
__device__ __forceinline__ int64_t vm_eval(const alk_instr* ins, uint32_t n, uint32_t result,
                                           const int64_t* consts, int64_t* regs, Col&& col) {
  for (uint32_t pc = 0; pc < n; pc++) {
    const alk_instr in = ins[pc];
    int64_t a = in.ka == ALK_K_REG ? regs[in.a * STRIDE] : (in.ka == ALK_K_COL ? col(in.a) : consts[in.a]);
    int64_t b = in.kb == ALK_K_REG ? regs[in.b * STRIDE] : (in.kb == ALK_K_COL ? col(in.b) : consts[in.b]);
    regs[in.dst * STRIDE] = vm_apply(in.op, a, b);
  }
  return regs[result * STRIDE];
}

// Decoupled look-back over tiles claimed in increasing order. Called by one thread per
// tile with the tile's aggregate; returns the exclusive prefix. flags must be zeroed
// before the launch. On an expired wait *err is set and 0 is returned (callers then
// skip their writes).
__device__ __forceinline__ uint64_t lookback_u64(volatile uint32_t* flags, volatile uint64_t* aggs,
                                                 volatile uint64_t* incls, uint32_t tile, uint64_t agg,
                                                 int* err, bool* ok) {
  *ok = true;
  if (tile == 0) {
    incls[0] = agg;
    __threadfence();
    flags[0] = 2;
    return 0;
  }
  aggs[tile] = agg;
  __threadfence();
  flags[tile] = 1;
  uint64_t excl = 0;
  int64_t j = (int64_t)tile - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    uint32_t f = flags[j];
    if (f == 0) {
      if (++spins > kSpinLimit) {
        atomicExch(err, ALK_ERR_TIMEOUT);
        *ok = false;
        break;
      }
      __nanosleep(64);
      continue;
    }
    __threadfence();
    if (f == 2) {
      excl += incls[j];
      break;
    }
    excl += aggs[j];
    j--;
  }
  incls[tile] = excl + agg;
  __threadfence();
  flags[tile] = 2;
  return excl;
}

// The same look-back run by a whole warp (all 32 lanes call it with the same tile and
// aggregate): each step reads 32 predecessors' flags at once, waits only while one of them
// up to the nearest inclusive prefix is still unpublished, and sums their aggregates (and
// that inclusive prefix) with a warp reduction, so a tile walks back over a run of
// unresolved tiles 32 at a time. Waits are bounded like lookback_u64's.
__device__ __forceinline__ uint64_t lookback_warp_u64(volatile uint32_t* flags, volatile uint64_t* aggs,
                                                      volatile uint64_t* incls, uint32_t tile, uint64_t agg,
                                                      int* err, bool* ok) {
  const int lane = threadIdx.x & 31;
  *ok = true;
  if (tile == 0) {
    if (lane == 0) {
      incls[0] = agg;
      __threadfence();
      flags[0] = 2;
    }
    __syncwarp();
    return 0;
  }
  if (lane == 0) {
    aggs[tile] = agg;
    __threadfence();
    flags[tile] = 1;
  }
  __syncwarp();
  uint64_t excl = 0;
  int64_t top = (int64_t)tile - 1;  // nearest predecessor not yet summed
  uint32_t spins = 0;
  bool timed_out = false;
  while (true) {
    const int64_t j = top - lane;  // lane 0 is the nearest predecessor
    const uint32_t f = j >= 0 ? flags[j] : 2u;  // before tile 0 counts as an inclusive prefix of 0
    const uint32_t inc = __ballot_sync(0xffffffffu, f == 2);
    const uint32_t upto = inc ? ((inc & (0u - inc)) << 1) - 1 : 0xffffffffu;  // lanes up to the first inclusive
    if (__ballot_sync(0xffffffffu, f == 0) & upto) {
      if (++spins > kSpinLimit) {
        timed_out = true;
        break;
      }
      __nanosleep(64);
      continue;
    }
    __threadfence();
    uint64_t v = 0;
    if ((upto >> lane) & 1) {
      if (f == 2) v = j >= 0 ? incls[j] : 0;
      else v = aggs[j];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (inc) break;
    top -= 32;
  }
  if (timed_out) {
    if (lane == 0) atomicExch(err, ALK_ERR_TIMEOUT);
    *ok = false;
  }
  if (lane == 0) {
    incls[tile] = excl + agg;
    __threadfence();
    flags[tile] = 2;
  }
  __syncwarp();
  return excl;
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

// Exclusive block scan of one value per thread; returns the exclusive prefix and the
// block total. s_warp must hold T/32 entries.
template <int T, class V>
__device__ __forceinline__ V block_excl_scan(V v, V* s_warp, V* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  V inc = warp_incl_scan(v);
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  if (w == 0) {
    V x = lane < T / 32 ? s_warp[lane] : V(0);
    V xi = warp_incl_scan(x);
    if (lane < T / 32) s_warp[lane] = xi - x;
    if (lane == T / 32 - 1) s_warp[T / 32] = xi;
  }
  __syncthreads();
  V res = s_warp[w] + inc - v;
  *total = s_warp[T / 32];
  __syncthreads();
  return res;
}

}  // namespace alkd
