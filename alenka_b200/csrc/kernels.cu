// Operator-level sm_100a kernels and their C entry points (include/alenka_b200.h):
// segment decode, fused scan/filter/compaction, expression evaluation, hash
// group-by, stable LSD radix sort, gather, tuple hashing and the hash join.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "device.cuh"
#include "internal.h"

using namespace alkd;

namespace {

constexpr int kT = 256;                  // threads per block
constexpr int kItems = 8;                // rows per thread per tile
constexpr int kTile = kT * kItems;       // rows per tile
constexpr int kMaxCols = 16;             // column slots per scan

int g_sm_count = 0;
int sm_count() {
  if (!g_sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

// ------------------------------------------------------------ decode
__global__ void __launch_bounds__(kT) k_decode_for(const void* p, uint32_t bits, int64_t lower,
                                                   uint32_t rows, int64_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * kT)
    out[i] = load_for(p, bits, lower, i);
}

// FOR-delta: value i (i >= 1) = unpacked(i) + lower, value 0 = start_val, then an
// inclusive prefix sum (compress.cu:123-144, 204-219). One tile per block claim, ordered
// by a look-back over tile sums.
struct DeltaArgs {
  const unsigned long long* words;
  uint32_t bits, fit;
  int64_t lower, start;
  uint32_t rows, ntiles;
  uint32_t* flags;
  uint64_t* aggs;
  uint64_t* incls;
  uint32_t* ctr;
  int* err;
  int64_t* out;
};
__global__ void __launch_bounds__(kT) k_decode_delta(DeltaArgs a) {
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_warp[kT / 32 + 1];
  __shared__ uint64_t s_base;
  __shared__ int s_ok;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.ctr, 1u);
    __syncthreads();
    uint32_t tile = s_tile;
    __syncthreads();
    if (tile >= a.ntiles) break;
    uint64_t r0 = (uint64_t)tile * kTile + (uint64_t)threadIdx.x * kItems;  // blocked
    uint64_t v[kItems];
    uint64_t sum = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      uint64_t i = r0 + k;
      uint64_t x = 0;
      if (i < a.rows) {
        if (i == 0) {
          x = (uint64_t)a.start;
        } else {
          uint64_t w = __ldg(a.words + i / a.fit);
          uint32_t sh = 64 - a.bits - (uint32_t)(i % a.fit) * a.bits;
          uint64_t t = w >> sh;
          t = a.bits == 64 ? t : (t & ((1ull << a.bits) - 1));
          x = t + (uint64_t)a.lower;
        }
      }
      sum += x;
      v[k] = sum;  // thread-local inclusive prefix (wrapping arithmetic)
    }
    uint64_t tot;
    uint64_t excl = block_excl_scan<kT>(sum, s_warp, &tot);
    if (threadIdx.x < 32) {
      bool ok;
      const uint64_t b = lookback_warp_u64(a.flags, a.aggs, a.incls, tile, tot, a.err, &ok);
      if (threadIdx.x == 0) {
        s_base = b;
        s_ok = ok;
      }
    }
    __syncthreads();
    if (s_ok) {
      uint64_t base = s_base + excl;
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if (r0 + k < a.rows) a.out[r0 + k] = (int64_t)(base + v[k]);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ ordered flag compaction
// out = the indices i (ascending) with flags[i] != 0: tiles claimed in increasing order,
// each thread counting 8 consecutive flags, a block scan and a decoupled look-back for the
// tile's base (the semi / anti joins keep their side's row order, operators.cu:1357-1399).
struct CompactArgs {
  const unsigned long long* flags;
  uint64_t n;
  uint32_t ntiles;
  uint32_t* tflags;
  uint64_t* aggs;
  uint64_t* incls;
  uint32_t* ctr;
  int* err;
  uint32_t* out;
  unsigned long long* count;
};
__global__ void __launch_bounds__(kT) k_flags_compact(CompactArgs a) {
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_warp[kT / 32 + 1];
  __shared__ uint64_t s_base;
  __shared__ int s_ok;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    __syncthreads();
    if (tile >= a.ntiles) break;
    const uint64_t r0 = (uint64_t)tile * kTile + (uint64_t)threadIdx.x * kItems;  // blocked
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (r0 + k < a.n && a.flags[r0 + k]) m |= 1u << k;
    uint64_t tot;
    const uint64_t excl = block_excl_scan<kT>((uint64_t)__popc(m), s_warp, &tot);
    if (threadIdx.x < 32) {
      bool ok;
      const uint64_t b = lookback_warp_u64(a.tflags, a.aggs, a.incls, tile, tot, a.err, &ok);
      if (threadIdx.x == 0) {
        s_base = b;
        s_ok = ok;
        if (ok && tile == a.ntiles - 1) *a.count = b + tot;
      }
    }
    __syncthreads();
    if (s_ok) {
      uint64_t o = s_base + excl;
      for (uint32_t q = m; q; q &= q - 1) a.out[o++] = (uint32_t)(r0 + (uint32_t)(__ffs(q) - 1));
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ fused scan
struct ScanArgs {
  const alk_colseg* cols;  // [ncols][nseg]
  uint32_t ncols, nseg;
  const uint8_t* seg_mode;
  const uint32_t* tile_seg;
  const uint32_t* tile_row0;
  uint32_t ntiles;
  const alk_program* prog;  // may be null
  const uint32_t* out_cols;
  uint32_t nout;
  int64_t* const* out;
  uint32_t* out_rowid;
  uint32_t* out_seg;
  unsigned long long* seg_counts;
  uint64_t cap;
  uint32_t* flags;
  uint64_t* aggs;
  uint64_t* incls;
  uint32_t* ctr;
  unsigned long long* total;
  int* err;
};

__global__ void __launch_bounds__(kT) k_scan(ScanArgs a) {
  __shared__ alk_instr s_ins[ALK_MAX_INSTR];
  __shared__ int64_t s_consts[ALK_MAX_CONST];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  __shared__ alk_colseg s_desc[kMaxCols];
  __shared__ uint32_t s_cnt[kItems * (kT / 32)];
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_base;
  __shared__ int s_ok;
  uint32_t nins = 0, result = 0;
  if (a.prog) {
    nins = a.prog->n_instr;
    result = a.prog->result;
    for (uint32_t i = threadIdx.x; i < nins; i += kT) s_ins[i] = a.prog->ins[i];
    for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[i] = a.prog->consts[i];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= a.ntiles) break;
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t seg_rows = s_desc[0].rows;
    const uint32_t rows = min((uint32_t)kTile, seg_rows - row0);
    const bool all = a.seg_mode[seg] == 1 || nins == 0;
    uint32_t ballots[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      const uint32_t r = k * kT + threadIdx.x;
      bool pass = false;
      if (r < rows) {
        if (all) {
          pass = true;
        } else {
          const uint64_t row = (uint64_t)row0 + r;
          auto col = [&](uint32_t slot) {
            const alk_colseg& d = s_desc[slot];
            return load_for(d.data, d.bits, d.lower, row);
          };
          pass = vm_eval<kT>(s_ins, nins, result, s_consts, s_regs + threadIdx.x, col) != 0;
        }
      }
      ballots[k] = __ballot_sync(0xffffffffu, pass);
      if (lane == 0) s_cnt[k * (kT / 32) + w] = __popc(ballots[k]);
    }
    __syncthreads();
    // exclusive scan of the (item round, warp) counts = row order within the tile
    if (w == 0) {
      uint32_t carry = 0;
      for (int base = 0; base < kItems * (kT / 32); base += 32) {
        uint32_t x = s_cnt[base + lane];
        uint32_t inc = warp_incl_scan(x);
        s_cnt[base + lane] = carry + inc - x;
        carry += __shfl_sync(0xffffffffu, inc, 31);
      }
      bool ok;
      const uint64_t b = lookback_warp_u64(a.flags, a.aggs, a.incls, tile, carry, a.err, &ok);
      if (lane == 0) {
        s_base = b;
        s_ok = ok;
        if (carry) {
          atomicAdd(a.total, (unsigned long long)carry);
          if (a.seg_counts) atomicAdd(a.seg_counts + seg, (unsigned long long)carry);
        }
      }
    }
    __syncthreads();
    if (s_ok) {
      const uint32_t lt = (1u << lane) - 1;
#pragma unroll
      for (int k = 0; k < kItems; k++) {
        if (!((ballots[k] >> lane) & 1)) continue;
        const uint64_t pos = s_base + s_cnt[k * (kT / 32) + w] + __popc(ballots[k] & lt);
        if (pos >= a.cap) continue;
        const uint32_t r = row0 + k * kT + threadIdx.x;
        for (uint32_t o = 0; o < a.nout; o++) {
          const alk_colseg& d = s_desc[a.out_cols[o]];
          a.out[o][pos] = load_for(d.data, d.bits, d.lower, r);
        }
        if (a.out_rowid) a.out_rowid[pos] = r;
        if (a.out_seg) a.out_seg[pos] = seg;
      }
    }
    __syncthreads();
  }
}

// Ordered scan for a filter that is one set test of one column (ALK_OP_INSET: the star
// join's filter on a bitmap index column, whose comparisons fold into one code set) with
// no output columns, in two passes without a look-back chain. Every block owns a
// contiguous run of tiles: k_set_pass<false> counts the run's survivors, k_block_offsets
// turns the blocks' counts into exclusive offsets, and k_set_pass<true> tests the rows
// again and writes the survivors' row positions and segments in row order from its
// block's offset. A block step covers kSetTiles tiles: each thread issues one vector load
// per tile for its 8 consecutive rows (8, 16 or 32-bit stored values, 16-byte aligned
// payloads) before testing any, tests them against the set (copied to shared memory when
// it fits), and one block scan over the threads' per-tile counts packed in 16-bit fields
// orders all kSetTiles tiles at once.
constexpr int kSetTiles = 4;
constexpr uint32_t kSetSmemWords = 4096;

struct SetTile {
  uint4 w0, w1;
  int64_t lower;
  uint32_t seg, row, rows, bits;  // row: this thread's first row; rows: its rows in the tile (0..8)
  bool all;
};

// The tile at (row0 of segment seg, descriptor d): this thread's 8 rows, loaded.
__device__ __forceinline__ SetTile set_tile_load(const alk_colseg& d, uint32_t seg, uint32_t row0, bool all) {
  SetTile t;
  t.seg = seg;
  const uint32_t tile_rows = min((uint32_t)kTile, d.rows - row0);
  const uint32_t r = (uint32_t)threadIdx.x * kItems;
  t.row = row0 + r;
  t.rows = r < tile_rows ? min((uint32_t)kItems, tile_rows - r) : 0;
  t.bits = d.bits;
  t.lower = d.lower;
  t.all = all;
  t.w0 = t.w1 = make_uint4(0, 0, 0, 0);
  if (t.rows) {
    if (d.bits == 8) {
      const uint2 w = *(const uint2*)((const uint8_t*)d.data + t.row);
      t.w0.x = w.x;
      t.w0.y = w.y;
    } else if (d.bits == 16) {
      t.w0 = *(const uint4*)((const uint16_t*)d.data + t.row);
    } else {
      t.w0 = *(const uint4*)((const uint32_t*)d.data + t.row);
      if (t.rows > 4) t.w1 = *(const uint4*)((const uint32_t*)d.data + t.row + 4);
    }
  }
  return t;
}

__device__ __forceinline__ uint32_t set_tile_mask(const SetTile& t, const uint32_t* set, uint64_t nset) {
  uint32_t v[kItems];
  if (t.bits == 8) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[k] = (t.w0.x >> (8 * k)) & 0xffu;
      v[k + 4] = (t.w0.y >> (8 * k)) & 0xffu;
    }
  } else if (t.bits == 16) {
    const uint32_t x[4] = {t.w0.x, t.w0.y, t.w0.z, t.w0.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[2 * k] = x[k] & 0xffffu;
      v[2 * k + 1] = x[k] >> 16;
    }
  } else {
    v[0] = t.w0.x, v[1] = t.w0.y, v[2] = t.w0.z, v[3] = t.w0.w;
    v[4] = t.w1.x, v[5] = t.w1.y, v[6] = t.w1.z, v[7] = t.w1.w;
  }
  const uint32_t valid = (1u << t.rows) - 1;  // rows <= 8
  if (t.all) return valid;
  uint32_t m = 0;
  if (t.lower >= 0 && (uint64_t)t.lower + (1ull << t.bits) <= 0xFFFFFFFFull && nset <= 0xFFFFFFFFull) {
    // every value and the set's size fit 32 bits (index codes offset by their segment)
    const uint32_t lo = (uint32_t)t.lower, n32 = (uint32_t)nset;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      const uint32_t x = v[k] + lo;
      m |= (uint32_t)(x < n32 && ((set[1 + (x >> 5)] >> (x & 31)) & 1)) << k;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      const uint64_t x = (uint64_t)v[k] + (uint64_t)t.lower;
      m |= (uint32_t)(x < nset && ((set[1 + (x >> 5)] >> (x & 31)) & 1)) << k;
    }
  }
  return m & valid;
}

template <bool WRITE>
__global__ void __launch_bounds__(kT, 3) k_set_pass(ScanArgs a, uint32_t slot, const uint32_t* set,
                                                 uint64_t* blk /* counts (count pass) or offsets (write pass) */) {
  __shared__ uint64_t s_warp[kT / 32 + 1];
  __shared__ uint32_t s_set[kSetSmemWords];
  const uint64_t nset = __ldg(set);
  const uint64_t words = 1 + (nset + 31) / 32;
  const bool in_smem = words <= kSetSmemWords;
  if (in_smem)
    for (uint32_t i = threadIdx.x; i < words; i += kT) s_set[i] = __ldg(set + i);
  __syncthreads();
  const uint32_t* bits = in_smem ? (const uint32_t*)s_set : set;
  const uint32_t per = (a.ntiles + gridDim.x - 1) / gridDim.x;
  const uint32_t t0 = min(a.ntiles, blockIdx.x * per), t1 = min(a.ntiles, t0 + per);
  uint64_t carry = WRITE ? blk[blockIdx.x] : 0;
  uint32_t cur_seg = 0;
  uint64_t seg_sum = 0;  // count pass, thread 0: survivors of the current segment not yet added
  // The tile list holds each scanned segment's tiles in order, kTile rows apart, so the
  // next tile is found by arithmetic; the list and the descriptors are read only where a
  // segment starts.
  uint32_t seg = 0, row0 = 0;
  alk_colseg d{};
  bool all = false;
  if (t0 < t1) {
    seg = a.tile_seg[t0];
    row0 = a.tile_row0[t0];
    d = a.cols[slot * a.nseg + seg];
    all = a.seg_mode[seg] == 1;
  }
  for (uint32_t tile = t0; tile < t1; tile += kSetTiles) {
    SetTile t[kSetTiles];
#pragma unroll
    for (int j = 0; j < kSetTiles; j++) {
      if (tile + j < t1) {
        if (j > 0 || tile > t0) {  // step from the previous tile
          const uint64_t next = (uint64_t)row0 + kTile;
          row0 = (uint32_t)next;
          if (next >= d.rows) {
            seg = a.tile_seg[tile + j];
            row0 = a.tile_row0[tile + j];
            d = a.cols[slot * a.nseg + seg];
            all = a.seg_mode[seg] == 1;
          }
        }
        t[j] = set_tile_load(d, seg, row0, all);
      } else {
        t[j].rows = 0;
        t[j].seg = 0;
      }
    }
    uint32_t m[kSetTiles];
    uint64_t packed = 0;
#pragma unroll
    for (int j = 0; j < kSetTiles; j++) {
      m[j] = t[j].rows ? set_tile_mask(t[j], bits, nset) : 0;
      packed |= (uint64_t)__popc(m[j]) << (16 * j);
    }
    uint64_t totp;
    const uint64_t exclp = block_excl_scan<kT>(packed, s_warp, &totp);
#pragma unroll
    for (int j = 0; j < kSetTiles; j++) {
      const uint64_t tj = (totp >> (16 * j)) & 0xffffu;
      if (WRITE) {
        uint64_t o = carry + ((exclp >> (16 * j)) & 0xffffu);
        for (uint32_t q = m[j]; q && o < a.cap; q &= q - 1, o++) {
          const uint32_t rr = t[j].row + (uint32_t)(__ffs(q) - 1);
          if (a.out_rowid) a.out_rowid[o] = rr;
          if (a.out_seg) a.out_seg[o] = t[j].seg;
        }
      } else if (threadIdx.x == 0 && a.seg_counts && tile + j < t1) {
        if (t[j].seg != cur_seg && seg_sum) {
          atomicAdd(a.seg_counts + cur_seg, (unsigned long long)seg_sum);
          seg_sum = 0;
        }
        cur_seg = t[j].seg;
        seg_sum += tj;
      }
      carry += tj;
    }
  }
  if (!WRITE && threadIdx.x == 0) {
    if (a.seg_counts && seg_sum) atomicAdd(a.seg_counts + cur_seg, (unsigned long long)seg_sum);
    blk[blockIdx.x] = carry;
  }
}

// Exclusive offsets of n block counts (in place), by one block; the total goes to *total.
constexpr int kOffT = 1024;
__global__ void __launch_bounds__(kOffT) k_block_offsets(uint64_t* blk, uint32_t n, unsigned long long* total) {
  __shared__ uint64_t s_warp[kOffT / 32 + 1];
  uint64_t carry = 0;
  for (uint32_t base = 0; base < n; base += kOffT) {
    const uint32_t i = base + threadIdx.x;
    const uint64_t v = i < n ? blk[i] : 0;
    uint64_t tot;
    const uint64_t excl = block_excl_scan<kOffT>(v, s_warp, &tot);
    if (i < n) blk[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

// ------------------------------------------------------------ expression evaluation
__global__ void __launch_bounds__(kT) k_eval(const int64_t* const* cols, uint32_t ncols, uint64_t n,
                                             const alk_program* prog, int64_t* out) {
  __shared__ alk_instr s_ins[ALK_MAX_INSTR];
  __shared__ int64_t s_consts[ALK_MAX_CONST];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  __shared__ const int64_t* s_cols[kMaxCols];
  const uint32_t nins = prog->n_instr, result = prog->result;
  for (uint32_t i = threadIdx.x; i < nins; i += kT) s_ins[i] = prog->ins[i];
  for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[i] = prog->consts[i];
  if (threadIdx.x < ncols) s_cols[threadIdx.x] = cols[threadIdx.x];
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    auto col = [&](uint32_t slot) { return __ldg(s_cols[slot] + i); };
    out[i] = vm_eval<kT>(s_ins, nins, result, s_consts, s_regs + threadIdx.x, col);
  }
}

// ------------------------------------------------------------ tuple hashing
__global__ void __launch_bounds__(kT) k_hash_tuples(const int64_t* const* cols, uint32_t k, uint64_t n,
                                                    uint32_t seed, uint64_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    uint64_t h = seed ^ ((uint64_t)(8 * k) * kMurmurM);
    for (uint32_t j = 0; j < k; j++) h = mm_block(h, (uint64_t)cols[j][i]);
    out[i] = mm_final(h);
  }
}

// ------------------------------------------------------------ gather
__global__ void __launch_bounds__(kT) k_gather(const int64_t* src, const uint32_t* idx, uint64_t n, int64_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    out[i] = __ldg(src + __ldg(idx + i));
}

__global__ void __launch_bounds__(kT) k_gather_u32(const uint32_t* src, const uint32_t* idx, uint64_t n,
                                                   uint32_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    out[i] = __ldg(src + __ldg(idx + i));
}

// Join forms of emit_multijoin (operators.cu:1288-1399) on the pairs a hash join found.
// flags[i] = (lcol[pl[i]] == rcol[pr[i]]) (!= when neq): the AND-ed key pairs.
__global__ void __launch_bounds__(kT) k_pair_match(const uint32_t* pl, const uint32_t* pr, uint64_t n,
                                                   const int64_t* lcol, const int64_t* rcol, int neq,
                                                   unsigned long long* flags) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const bool eq = lcol[pl[i]] == rcol[pr[i]];
    flags[i] = (eq != (neq != 0)) ? 1ull : 0ull;
  }
}
// flags[rows[i]] = v: the rows a semi or anti join keeps or drops.
__global__ void __launch_bounds__(kT) k_rows_mark(const uint32_t* rows, uint64_t n, unsigned long long* flags,
                                                  unsigned long long v) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    flags[rows[i]] = v;
}
// Per segment g (rows [start[g], start[g + 1])), the least and greatest key: out[2g],
// out[2g + 1] (preset to INT64_MAX / INT64_MIN).
__global__ void __launch_bounds__(kT) k_seg_minmax(const int64_t* keys, const uint64_t* start, uint32_t nseg,
                                                   long long* out) {
  for (uint32_t g = 0; g < nseg; g++) {
    const uint64_t b = start[g], e = start[g + 1];
    long long mn = INT64_MAX, mx = INT64_MIN;
    for (uint64_t i = b + blockIdx.x * (uint64_t)kT + threadIdx.x; i < e; i += (uint64_t)gridDim.x * kT) {
      const long long k = keys[i];
      mn = k < mn ? k : mn;
      mx = k > mx ? k : mx;
    }
    for (int o = 16; o; o >>= 1) {
      mn = min(mn, (long long)__shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, (long long)__shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0 && b < e) {
      atomicMin(out + 2 * g, mn);
      atomicMax(out + 2 * g + 1, mx);
    }
  }
}

// ------------------------------------------------------------ hash group-by
constexpr int kMaxKeys = 8;
constexpr int kMaxVals = 16;
struct GbArgs {
  const int64_t* const* keys;
  uint32_t nkeys;
  const int64_t* const* vals;
  const uint8_t* aggs;
  uint32_t nvals;
  uint64_t n;
  uint64_t cap;  // power of two
  uint32_t* state;
  int64_t* tkeys;
  int64_t* tvals;
  uint32_t* first;
  unsigned long long* ngroups;
  int* err;
};

__global__ void __launch_bounds__(kT) k_gb_init(GbArgs a) {
  for (uint64_t h = blockIdx.x * (uint64_t)kT + threadIdx.x; h < a.cap; h += (uint64_t)gridDim.x * kT) {
    a.state[h] = 0;
    a.first[h] = 0xffffffffu;
    for (uint32_t v = 0; v < a.nvals; v++) {
      int64_t init = 0;
      if (a.aggs[v] == ALK_AGG_MIN) init = INT64_MAX;
      if (a.aggs[v] == ALK_AGG_MAX) init = INT64_MIN;
      a.tvals[v * a.cap + h] = init;
    }
  }
}

__global__ void __launch_bounds__(kT) k_gb_insert(GbArgs a) {
  const uint64_t mask = a.cap - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < a.n; i += (uint64_t)gridDim.x * kT) {
    int64_t key[kMaxKeys];
    uint64_t h = kSeed ^ ((uint64_t)(8 * a.nkeys) * kMurmurM);
#pragma unroll
    for (int j = 0; j < kMaxKeys; j++) {
      if (j < (int)a.nkeys) {
        key[j] = __ldg(a.keys[j] + i);
        h = mm_block(h, (uint64_t)key[j]);
      }
    }
    h = mm_final(h) & mask;
    uint64_t probes = 0;
    uint32_t spins = 0;
    bool found = false;
    while (probes <= mask) {
      uint32_t s = *((volatile uint32_t*)a.state + h);
      if (s == 0) {
        if (atomicCAS(a.state + h, 0u, 1u) == 0u) {
#pragma unroll
          for (int j = 0; j < kMaxKeys; j++)
            if (j < (int)a.nkeys) a.tkeys[j * a.cap + h] = key[j];
          __threadfence();
          atomicExch(a.state + h, 2u);
          found = true;
          break;
        }
        continue;
      }
      if (s == 1) {
        if (++spins > kSpinLimit) {
          atomicExch(a.err, ALK_ERR_TIMEOUT);
          break;
        }
        continue;
      }
      __threadfence();
      bool eq = true;
#pragma unroll
      for (int j = 0; j < kMaxKeys; j++)
        if (j < (int)a.nkeys && __ldcg(a.tkeys + j * a.cap + h) != key[j]) eq = false;
      if (eq) {
        found = true;
        break;
      }
      h = (h + 1) & mask;
      probes++;
    }
    if (!found) {
      atomicCAS(a.err, 0, ALK_ERR_OVERFLOW);
      continue;
    }
    for (uint32_t v = 0; v < a.nvals; v++) {
      unsigned long long* dst = (unsigned long long*)(a.tvals + v * a.cap + h);
      switch (a.aggs[v]) {
        case ALK_AGG_SUM: atomicAdd(dst, (unsigned long long)__ldg(a.vals[v] + i)); break;
        case ALK_AGG_COUNT: atomicAdd(dst, 1ull); break;
        case ALK_AGG_MIN: atomicMin((long long*)dst, (long long)__ldg(a.vals[v] + i)); break;
        default: atomicMax((long long*)dst, (long long)__ldg(a.vals[v] + i)); break;
      }
    }
    atomicMin(a.first + h, (uint32_t)i);
  }
}

__global__ void __launch_bounds__(kT) k_gb_compact(GbArgs a, int64_t* const* out_keys, int64_t* const* out_vals,
                                                   uint32_t* out_first) {
  for (uint64_t h = blockIdx.x * (uint64_t)kT + threadIdx.x; h < a.cap; h += (uint64_t)gridDim.x * kT) {
    if (a.state[h] != 2) continue;
    unsigned long long pos = atomicAdd(a.ngroups, 1ull);
    for (uint32_t j = 0; j < a.nkeys; j++) out_keys[j][pos] = a.tkeys[j * a.cap + h];
    for (uint32_t v = 0; v < a.nvals; v++) out_vals[v][pos] = a.tvals[v * a.cap + h];
    if (out_first) out_first[pos] = a.first[h];
  }
}

// ------------------------------------------------------------ radix sort (stable LSD, 4-bit digits)
constexpr int kRadixBits = 4;
constexpr int kRadix = 1 << kRadixBits;

__global__ void __launch_bounds__(kT) k_minmax_u64(const uint64_t* k, uint64_t n, unsigned long long* mm) {
  uint64_t lo = ~0ull, hi = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    uint64_t x = k[i];
    lo = min(lo, x);
    hi = max(hi, x);
  }
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, (unsigned long long)lo);
    atomicMax(mm + 1, (unsigned long long)hi);
  }
}

// Per-block digit histogram; hist is digit-major: hist[d * nblocks + b].
__global__ void __launch_bounds__(kT) k_radix_hist(const uint64_t* keys, uint64_t n, uint32_t shift,
                                                   uint32_t* hist, uint32_t nblocks) {
  __shared__ uint32_t s_h[kRadix];
  if (threadIdx.x < kRadix) s_h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t b0 = (uint64_t)blockIdx.x * kTile;
  for (int k = 0; k < kItems; k++) {
    uint64_t i = b0 + (uint64_t)k * kT + threadIdx.x;
    if (i < n) atomicAdd(&s_h[(keys[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  if (threadIdx.x < kRadix) hist[threadIdx.x * nblocks + blockIdx.x] = s_h[threadIdx.x];
}

// Exclusive scan of a u32 array in one block (the histogram is small: 16 x blocks).
__global__ void __launch_bounds__(1024) k_scan_small(uint32_t* x, uint32_t n) {
  __shared__ uint32_t s_w[33];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < n ? x[i] : 0;
    uint32_t inc = warp_incl_scan(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
      uint32_t t = s_w[lane];
      uint32_t ti = warp_incl_scan(t);
      s_w[lane] = ti - t;
      if (lane == 31) s_w[32] = ti;
    }
    __syncthreads();
    uint32_t carry = s_carry;
    if (i < n) x[i] = carry + s_w[w] + inc - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + s_w[32];
    __syncthreads();
  }
}

// Stable scatter: blocked arrangement so that thread order is input order.
__global__ void __launch_bounds__(kT) k_radix_scatter(const uint64_t* keys, const uint32_t* vals, uint64_t n,
                                                      uint32_t shift, const uint32_t* offs, uint32_t nblocks,
                                                      uint64_t* okeys, uint32_t* ovals) {
  __shared__ uint32_t s_w[kRadix][kT / 32 + 1];
  const uint64_t b0 = (uint64_t)blockIdx.x * kTile + (uint64_t)threadIdx.x * kItems;
  uint32_t cnt[kRadix];
#pragma unroll
  for (int d = 0; d < kRadix; d++) cnt[d] = 0;
  uint64_t kk[kItems];
  uint32_t vv[kItems];
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    uint64_t i = b0 + k;
    if (i < n) {
      kk[k] = keys[i];
      vv[k] = vals[i];
      uint32_t d = (kk[k] >> shift) & (kRadix - 1);
#pragma unroll
      for (int e = 0; e < kRadix; e++) cnt[e] += (d == (uint32_t)e);
    }
  }
  // per-digit exclusive prefix over threads (thread order == input order)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t pre[kRadix];
#pragma unroll
  for (int d = 0; d < kRadix; d++) {
    uint32_t inc = warp_incl_scan(cnt[d]);
    pre[d] = inc - cnt[d];
    if (lane == 31) s_w[d][w] = inc;
  }
  __syncthreads();
  if (threadIdx.x < kRadix) {
    uint32_t run = 0;
    for (int j = 0; j < kT / 32; j++) {
      uint32_t t = s_w[threadIdx.x][j];
      s_w[threadIdx.x][j] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int d = 0; d < kRadix; d++) pre[d] += s_w[d][w] + offs[d * nblocks + blockIdx.x];
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    uint64_t i = b0 + k;
    if (i < n) {
      uint32_t d = (kk[k] >> shift) & (kRadix - 1);
      uint32_t p = 0;
#pragma unroll
      for (int e = 0; e < kRadix; e++)
        if (d == (uint32_t)e) p = pre[e]++;
      if (p < n) {  // always true for a consistent histogram; guards the write
        okeys[p] = kk[k];
        ovals[p] = vv[k];
      }
    }
  }
}

__global__ void __launch_bounds__(kT) k_sortkey_i64(const int64_t* key, const uint32_t* perm, uint64_t n, int desc,
                                                    uint64_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    uint64_t u = (uint64_t)key[perm ? perm[i] : i] ^ 0x8000000000000000ull;
    out[i] = desc ? ~u : u;
  }
}
__global__ void __launch_bounds__(kT) k_widen(const uint32_t* in, uint64_t n, int64_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) out[i] = in[i];
}
// Frame-of-reference re-encoding: the exact minimum and maximum (one pass), then the
// values less the minimum at the narrowest of 8/16/32/64 bits (a second pass).
__global__ void __launch_bounds__(kT) k_minmax_i64(const int64_t* in, uint64_t n, long long* mm) {
  long long lo = INT64_MAX, hi = INT64_MIN;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const long long v = in[i];
    lo = min(lo, v);
    hi = max(hi, v);
  }
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}
template <typename T>
__global__ void __launch_bounds__(kT) k_for_narrow(const int64_t* in, uint64_t n, const long long* mm, T* out) {
  const uint64_t lo = (uint64_t)mm[0];
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    out[i] = (T)((uint64_t)in[i] - lo);
}

__global__ void __launch_bounds__(kT) k_narrow(const int64_t* in, uint64_t n, uint32_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) out[i] = (uint32_t)in[i];
}
__global__ void __launch_bounds__(kT) k_iota(uint32_t* p, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) p[i] = (uint32_t)i;
}

// ------------------------------------------------------------ hash join
__global__ void __launch_bounds__(kT) k_join_build(const int64_t* keys, uint64_t n, uint64_t cap, int64_t* tkey,
                                                   uint32_t* trow, int* err) {
  const uint64_t mask = cap - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const int64_t k = keys[i];
    uint64_t h = murmur_u64((uint64_t)k) & mask;
    uint64_t probes = 0;
    while (true) {
      if (atomicCAS(trow + h, 0u, (uint32_t)(i + 1)) == 0u) {
        tkey[h] = k;
        break;
      }
      h = (h + 1) & mask;
      if (++probes > mask) {
        atomicExch(err, ALK_ERR_OVERFLOW);
        break;
      }
    }
  }
}

__global__ void __launch_bounds__(kT) k_join_probe(const int64_t* keys, uint64_t n, uint64_t cap, const int64_t* tkey,
                                                   const uint32_t* trow, uint32_t* out_l, uint32_t* out_r,
                                                   uint64_t out_cap, unsigned long long* count) {
  const uint64_t mask = cap - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const int64_t k = __ldg(keys + i);
    uint64_t h = murmur_u64((uint64_t)k) & mask;
    for (uint64_t probes = 0; probes <= mask; probes++) {
      const uint32_t r = __ldg(trow + h);
      if (r == 0) break;
      if (__ldg(tkey + h) == k) {
        unsigned long long pos = atomicAdd(count, 1ull);
        if (pos < out_cap) {
          out_l[pos] = (uint32_t)i;
          out_r[pos] = r - 1;
        }
      }
      h = (h + 1) & mask;
    }
  }
}

// Every operand of a program must name an existing register, column slot or constant:
// the device code indexes shared arrays with them unchecked.
bool program_ok(const alk_program* p, uint32_t ncols) {
  if (p->n_instr > ALK_MAX_INSTR || p->result >= ALK_MAX_REGS) return false;
  for (uint32_t i = 0; i < p->n_instr; i++) {
    const alk_instr& in = p->ins[i];
    if (in.dst >= ALK_MAX_REGS || in.op < ALK_OP_ADD || in.op > ALK_OP_INSET) return false;
    if (in.op == ALK_OP_INSET && in.kb != ALK_K_CONST) return false;  // the set's address
    const uint8_t k[2] = {in.ka, in.kb};
    const uint16_t x[2] = {in.a, in.b};
    for (int j = 0; j < 2; j++) {
      if (k[j] == ALK_K_REG && x[j] >= ALK_MAX_REGS) return false;
      if (k[j] == ALK_K_COL && x[j] >= ncols) return false;
      if (k[j] == ALK_K_CONST && x[j] >= ALK_MAX_CONST) return false;
      if (k[j] > ALK_K_CONST) return false;
    }
  }
  return true;
}

int grid_for(uint64_t n) {
  uint64_t b = (n + kT - 1) / kT;
  uint64_t lim = (uint64_t)sm_count() * 8;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, lim));
}


// ------------------------------------------------------------ sort-based group-by
// Rows in key order (the identity when the input already is, else a stable permutation)
// are cut into tiles of kSegTile rows; thread t of a tile owns rows t*kSegItems ..
// t*kSegItems + kSegItems - 1. A row heads a group when its key tuple differs from the
// previous row's. Group g = (heads up to and including the row) - 1.
constexpr int kSegItems = 8;
constexpr int kSegTile = kT * kSegItems;

struct SegGbArgs {
  const int64_t* const* keys;
  uint32_t nkeys;
  const int64_t* const* vals;
  const uint8_t* aggs;
  uint32_t nvals;
  uint64_t n;
  const uint32_t* perm;  // null: identity
  unsigned long long* tile_heads;  // [ntiles]: heads per tile, then their exclusive prefix
  unsigned long long* flags;       // [0] rows out of key order (the check), [1] groups
};

__device__ __forceinline__ uint64_t seg_row(const SegGbArgs& a, uint64_t i) { return a.perm ? a.perm[i] : i; }

__device__ __forceinline__ bool seg_head(const SegGbArgs& a, uint64_t i) {
  if (i == 0) return true;
  const uint64_t r = seg_row(a, i), q = seg_row(a, i - 1);
  for (uint32_t j = 0; j < a.nkeys; j++)
    if (__ldg(a.keys[j] + r) != __ldg(a.keys[j] + q)) return true;
  return false;
}

// Rows where the key tuple decreases (lexicographic, signed): zero means already in order.
__global__ void __launch_bounds__(kT) k_seg_check(const SegGbArgs a) {
  unsigned long long bad = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x + 1; i < a.n; i += (uint64_t)gridDim.x * kT) {
    for (uint32_t j = 0; j < a.nkeys; j++) {
      const int64_t x = __ldg(a.keys[j] + i - 1), y = __ldg(a.keys[j] + i);
      if (x != y) {
        bad += x > y;
        break;
      }
    }
  }
  for (int o = 16; o; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(a.flags, bad);
}

__global__ void __launch_bounds__(kT) k_seg_count(const SegGbArgs a) {
  __shared__ unsigned long long s_warp[kT / 32 + 1];
  const uint64_t t = blockIdx.x;
  const uint64_t i0 = t * kSegTile + (uint64_t)threadIdx.x * kSegItems;
  unsigned long long c = 0;
  for (int k = 0; k < kSegItems; k++)
    if (i0 + k < a.n && seg_head(a, i0 + k)) c++;
  unsigned long long tot;
  block_excl_scan<kT>(c, s_warp, &tot);
  if (threadIdx.x == 0) a.tile_heads[t] = tot;
}

// exclusive prefix of the tile counts, one block; flags[1] = groups
__global__ void __launch_bounds__(1024) k_seg_scan(const SegGbArgs a, uint64_t ntiles) {
  __shared__ unsigned long long s_warp[1024 / 32 + 1];
  unsigned long long carry = 0;
  for (uint64_t b = 0; b < ntiles; b += 1024) {
    const uint64_t i = b + threadIdx.x;
    const unsigned long long v = i < ntiles ? a.tile_heads[i] : 0;
    unsigned long long tot;
    const unsigned long long ex = block_excl_scan<1024>(v, s_warp, &tot);
    if (i < ntiles) a.tile_heads[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) a.flags[1] = carry;
}

__device__ __forceinline__ void seg_apply(int64_t* dst, uint8_t kind, int64_t v) {
  if (kind == ALK_AGG_MIN) atomicMin((long long*)dst, (long long)v);
  else if (kind == ALK_AGG_MAX) atomicMax((long long*)dst, (long long)v);
  else atomicAdd((unsigned long long*)dst, (unsigned long long)v);
}

// Group index of every row; head rows write their keys and first row; every row's values
// are folded in registers while the thread's group does not change, then applied with
// one atomic per (thread, group, value).
__global__ void __launch_bounds__(kT) k_seg_reduce(const SegGbArgs a, int64_t* const* out_keys,
                                                   int64_t* const* out_vals, uint32_t* out_first) {
  __shared__ unsigned long long s_warp[kT / 32 + 1];
  const uint64_t t = blockIdx.x;
  const uint64_t i0 = t * kSegTile + (uint64_t)threadIdx.x * kSegItems;
  uint32_t heads = 0;
  unsigned long long c = 0;
  for (int k = 0; k < kSegItems; k++)
    if (i0 + k < a.n && seg_head(a, i0 + k)) {
      heads |= 1u << k;
      c++;
    }
  unsigned long long tot;
  const unsigned long long ex = block_excl_scan<kT>(c, s_warp, &tot);
  // group of the thread's first row: heads before it, minus one
  long long g = (long long)(a.tile_heads[t] + ex) - 1;
  int64_t acc[kMaxVals];
  long long cur = -1;
  for (int k = 0; k < kSegItems; k++) {
    const uint64_t i = i0 + k;
    if (i >= a.n) break;
    const uint64_t r = seg_row(a, i);
    if ((heads >> k) & 1) {
      g++;
      for (uint32_t j = 0; j < a.nkeys; j++) out_keys[j][g] = __ldg(a.keys[j] + r);
      out_first[g] = (uint32_t)r;
    }
    if (g != cur) {
      if (cur >= 0)
        for (uint32_t v = 0; v < a.nvals; v++) seg_apply(out_vals[v] + cur, a.aggs[v], acc[v]);
      cur = g;
      for (uint32_t v = 0; v < a.nvals; v++)
        acc[v] = a.aggs[v] == ALK_AGG_COUNT ? 1 : __ldg(a.vals[v] + r);
      continue;
    }
    for (uint32_t v = 0; v < a.nvals; v++) {
      const uint8_t kind = a.aggs[v];
      if (kind == ALK_AGG_COUNT) {
        acc[v] += 1;
        continue;
      }
      const int64_t x = __ldg(a.vals[v] + r);
      acc[v] = kind == ALK_AGG_MIN ? min(acc[v], x)
             : kind == ALK_AGG_MAX ? max(acc[v], x)
                                   : (int64_t)((uint64_t)acc[v] + (uint64_t)x);
    }
  }
  if (cur >= 0)
    for (uint32_t v = 0; v < a.nvals; v++) seg_apply(out_vals[v] + cur, a.aggs[v], acc[v]);
}

__global__ void __launch_bounds__(kT) k_seg_init(int64_t* const* out_vals, const uint8_t* aggs, uint32_t nvals,
                                                 uint64_t g) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < g * nvals; i += (uint64_t)gridDim.x * kT) {
    const uint32_t v = (uint32_t)(i / g);
    const uint8_t k = aggs[v];
    out_vals[v][i - (uint64_t)v * g] = k == ALK_AGG_MIN ? INT64_MAX : k == ALK_AGG_MAX ? INT64_MIN : 0;
  }
}
}  // namespace

#define CK(x)                                           \
  do {                                                  \
    cudaError_t e_ = (x);                               \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_);   \
  } while (0)

namespace alk {
int cuda_fail(cudaError_t e) {
  set_last_cuda_error(e);
  return e == cudaErrorMemoryAllocation ? ALK_ERR_NOMEM : ALK_ERR_CUDA;
}
thread_local cudaError_t g_last_cuda = cudaSuccess;
void set_last_cuda_error(cudaError_t e) { g_last_cuda = e; }
const char* last_cuda_error() { return cudaGetErrorString(g_last_cuda); }
uint64_t g_kernel_launches = 0;

std::vector<void*>& capture_host_buffers() {
  static thread_local std::vector<void*> v;
  return v;
}

const void* upload_source(const void* host, size_t bytes, cudaStream_t s, cudaError_t* err) {
  *err = cudaSuccess;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusActive) return host;
  void* p = nullptr;
  *err = cudaMallocHost(&p, bytes ? bytes : 1);
  if (*err != cudaSuccess) return nullptr;
  std::memcpy(p, host, bytes);
  capture_host_buffers().push_back(p);
  return p;
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
}  // namespace alk

using alk::Scratch;

extern "C" {

int alk_device_info(int* sms, int* major, int* minor) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp p;
  CK(cudaGetDeviceProperties(&p, dev));
  if (sms) *sms = p.multiProcessorCount;
  if (major) *major = p.major;
  if (minor) *minor = p.minor;
  return ALK_OK;
}

int alk_decode_segment(const void* d_payload, uint32_t comp_type, uint32_t bits, uint32_t fit_count,
                       int64_t lower, int64_t start_val, uint32_t rows, int64_t* d_out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (rows == 0) return ALK_OK;
  if (!d_payload || !d_out) return ALK_ERR_ARG;
  if (comp_type == 0) {
    if (bits != 8 && bits != 16 && bits != 32 && bits != 64) return ALK_ERR_ARG;
    k_decode_for<<<grid_for(rows), kT, 0, s>>>(d_payload, bits, lower, rows, d_out);
    alk::g_kernel_launches++;
    CK(cudaGetLastError());
    return ALK_OK;
  }
  if (comp_type != 1 || bits == 0 || bits > 64 || fit_count != 64 / bits) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  // in 64 bits: rows + kTile - 1 wraps in 32 bits for rows near 2^32
  const uint32_t ntiles = (uint32_t)(((uint64_t)rows + kTile - 1) / kTile);
  uint32_t* flags = sc.get<uint32_t>(ntiles + 2, &e);
  CK(e);
  uint64_t* aggs = sc.get<uint64_t>(ntiles, &e);
  CK(e);
  uint64_t* incls = sc.get<uint64_t>(ntiles, &e);
  CK(e);
  int* err = (int*)(flags + ntiles + 1);
  CK(cudaMemsetAsync(flags, 0, (ntiles + 2) * sizeof(uint32_t), s));
  DeltaArgs a{(const unsigned long long*)d_payload, bits, fit_count, lower, start_val, rows, ntiles,
              flags, aggs, incls, flags + ntiles, err, d_out};
  int grid = std::min<int>(ntiles, sm_count() * 4);
  k_decode_delta<<<grid, kT, 0, s>>>(a);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  int h_err = 0;
  CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return h_err;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free decode
// Look-back state of alk_decode_segment_noalloc lives in this file-scope array instead of
// memory allocated per call: tile flags plus the tile counter and error word, then the
// per-tile aggregates and inclusive prefixes. Every device that loads the library holds
// it until the process exits.
namespace {
constexpr uint32_t kNoAllocMaxTiles = 32768;  // 32768 tiles x 2048 rows = 67,108,864 rows
constexpr size_t kNoAllocFlagBytes = ((kNoAllocMaxTiles + 2) * sizeof(uint32_t) + 255) / 256 * 256;
constexpr size_t kNoAllocScratchBytes = kNoAllocFlagBytes + 2 * (size_t)kNoAllocMaxTiles * sizeof(uint64_t);
static __device__ __align__(256) unsigned char g_decode_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_decode_scratch on the current device, looked up once per device
// (host code cannot use the array's name as a device address) and kept for the life of
// the process: a device reset (cudaDeviceReset) after the first call is not supported,
// because the array may then live at another address.
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return alk::cuda_fail(e);
  if (dev < 0 || dev >= kMaxDevices) return ALK_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_decode_scratch);
    if (e != cudaSuccess || !p) return alk::cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
    g_scratch_addr[dev] = p;
  }
  *out = (unsigned char*)g_scratch_addr[dev];
  return ALK_OK;
}
}  // namespace

extern "C" {

int alk_decode_segment_noalloc(const void* d_payload, uint32_t comp_type, uint32_t bits, uint32_t fit_count,
                               int64_t lower, int64_t start_val, uint32_t rows, int64_t* d_out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (rows == 0) return ALK_OK;
  if (!d_payload || !d_out) return ALK_ERR_ARG;
  if (comp_type == 0) {  // FOR widening needs no scratch
    if (bits != 8 && bits != 16 && bits != 32 && bits != 64) return ALK_ERR_ARG;
    k_decode_for<<<grid_for(rows), kT, 0, s>>>(d_payload, bits, lower, rows, d_out);
    alk::g_kernel_launches++;
    CK(cudaGetLastError());
    return ALK_OK;
  }
  if (comp_type != 1 || bits == 0 || bits > 64 || fit_count != 64 / bits) return ALK_ERR_ARG;
  // the row count is tested before any tile arithmetic, so no count wraps past the limit
  if ((uint64_t)rows > (uint64_t)kNoAllocMaxTiles * kTile) return ALK_ERR_TOO_LARGE;
  const uint32_t ntiles = (uint32_t)(((uint64_t)rows + kTile - 1) / kTile);
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  uint32_t* flags = (uint32_t*)base;
  uint64_t* aggs = (uint64_t*)(base + kNoAllocFlagBytes);
  uint64_t* incls = aggs + kNoAllocMaxTiles;
  int* err = (int*)(flags + ntiles + 1);
  // tile flags, the tile counter and the error word must start at zero
  CK(cudaMemsetAsync(flags, 0, (ntiles + 2) * sizeof(uint32_t), s));
  DeltaArgs a{(const unsigned long long*)d_payload, bits, fit_count, lower, start_val, rows, ntiles,
              flags, aggs, incls, flags + ntiles, err, d_out};
  int grid = std::min<int>(ntiles, sm_count() * 4);
  k_decode_delta<<<grid, kT, 0, s>>>(a);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  int h_err = 0;
  CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return h_err;
}

int alk_hash_tuples(const int64_t* const* d_cols, uint32_t k, uint64_t n, uint32_t seed, uint64_t* d_out,
                    alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return ALK_OK;
  if (k == 0 || k > kMaxKeys) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  const int64_t** dc = sc.get<const int64_t*>(k, &e);
  CK(e);
  CK(cudaMemcpyAsync(dc, d_cols, k * sizeof(void*), cudaMemcpyHostToDevice, s));
  k_hash_tuples<<<grid_for(n), kT, 0, s>>>(dc, k, n, seed, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_scan_filter(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                    const alk_program* pred, const uint32_t* out_cols, uint32_t nout, int64_t* const* d_out,
                    uint32_t* d_out_rowid, uint32_t* d_out_seg, uint64_t* d_seg_counts, uint64_t cap,
                    uint64_t* h_count, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_count || ncols == 0 || ncols > kMaxCols || nout > kMaxCols) return ALK_ERR_ARG;
  if (pred && !program_ok(pred, ncols)) return ALK_ERR_ARG;
  for (uint32_t o = 0; o < nout; o++)
    if (out_cols[o] >= ncols) return ALK_ERR_ARG;
  *h_count = 0;
  std::vector<uint32_t> tseg, trow;
  for (uint32_t g = 0; g < nseg; g++) {
    if (seg_mode[g] == 0) continue;
    uint32_t rows = cols[g].rows;
    for (uint32_t c = 1; c < ncols; c++)
      if (cols[c * nseg + g].rows != rows) return ALK_ERR_ARG;
    for (uint32_t r = 0; r < rows; r += kTile) {
      tseg.push_back(g);
      trow.push_back(r);
    }
  }
  if (d_seg_counts) CK(cudaMemsetAsync(d_seg_counts, 0, nseg * sizeof(uint64_t), s));
  if (tseg.empty()) return ALK_OK;
  const uint32_t ntiles = (uint32_t)tseg.size();
  // one packed upload: descriptors, modes, tiles, program, output pointers
  size_t off_cols = 0;
  size_t off_mode = off_cols + sizeof(alk_colseg) * ncols * nseg;
  size_t off_tseg = (off_mode + nseg + 15) & ~size_t(15);
  size_t off_trow = off_tseg + 4 * (size_t)ntiles;
  size_t off_prog = (off_trow + 4 * (size_t)ntiles + 15) & ~size_t(15);
  size_t off_ocol = off_prog + sizeof(alk_program);
  size_t off_optr = (off_ocol + 4 * (size_t)kMaxCols + 15) & ~size_t(15);
  size_t total = off_optr + sizeof(void*) * kMaxCols;
  std::vector<uint8_t> hb(total, 0);
  std::memcpy(&hb[off_cols], cols, sizeof(alk_colseg) * ncols * nseg);
  std::memcpy(&hb[off_mode], seg_mode, nseg);
  std::memcpy(&hb[off_tseg], tseg.data(), 4 * (size_t)ntiles);
  std::memcpy(&hb[off_trow], trow.data(), 4 * (size_t)ntiles);
  if (pred) std::memcpy(&hb[off_prog], pred, sizeof(alk_program));
  if (nout) {
    std::memcpy(&hb[off_ocol], out_cols, 4 * (size_t)nout);
    std::memcpy(&hb[off_optr], d_out, sizeof(void*) * nout);
  }
  Scratch sc(s);
  cudaError_t e;
  uint8_t* db = sc.get<uint8_t>(total, &e);
  CK(e);
  uint32_t* flags = sc.get<uint32_t>(ntiles + 4, &e);
  CK(e);
  uint64_t* lb = sc.get<uint64_t>(2 * (size_t)ntiles + 2, &e);
  CK(e);
  CK(cudaMemcpyAsync(db, hb.data(), total, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(flags, 0, (ntiles + 4) * sizeof(uint32_t), s));
  CK(cudaMemsetAsync(lb + 2 * (size_t)ntiles, 0, 2 * sizeof(uint64_t), s));
  ScanArgs a;
  a.cols = (const alk_colseg*)(db + off_cols);
  a.ncols = ncols;
  a.nseg = nseg;
  a.seg_mode = db + off_mode;
  a.tile_seg = (const uint32_t*)(db + off_tseg);
  a.tile_row0 = (const uint32_t*)(db + off_trow);
  a.ntiles = ntiles;
  a.prog = pred ? (const alk_program*)(db + off_prog) : nullptr;
  a.out_cols = (const uint32_t*)(db + off_ocol);
  a.nout = nout;
  a.out = (int64_t* const*)(db + off_optr);
  a.out_rowid = d_out_rowid;
  a.out_seg = d_out_seg;
  a.seg_counts = (unsigned long long*)d_seg_counts;
  a.cap = cap;
  a.flags = flags;
  a.ctr = flags + ntiles;
  a.err = (int*)(flags + ntiles + 1);
  a.aggs = lb;
  a.incls = lb + ntiles;
  a.total = (unsigned long long*)(lb + 2 * (size_t)ntiles);
  // one set test of one column and no output columns: the vector-load form
  bool set_form = pred && nout == 0 && pred->n_instr == 1 && pred->ins[0].op == ALK_OP_INSET &&
                  pred->ins[0].ka == ALK_K_COL && pred->ins[0].kb == ALK_K_CONST && pred->result == pred->ins[0].dst;
  const uint32_t set_slot = set_form ? pred->ins[0].a : 0;
  for (uint32_t g = 0; set_form && g < nseg; g++) {
    if (seg_mode[g] == 0) continue;
    const alk_colseg& d = cols[set_slot * nseg + g];
    if ((d.bits != 8 && d.bits != 16 && d.bits != 32) || ((uintptr_t)d.data & 15)) set_form = false;
  }
  int occ = 0;
  if (set_form) {
    const uint32_t* set = (const uint32_t*)(uintptr_t)pred->consts[pred->ins[0].b];
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_set_pass<true>, kT, 0);
    const int grid = std::max(1, std::min<int>((int)ntiles, sm_count() * std::max(occ, 1)));
    uint64_t* blk = sc.get<uint64_t>(grid, &e);
    CK(e);
    k_set_pass<false><<<grid, kT, 0, s>>>(a, set_slot, set, blk);
    k_block_offsets<<<1, kOffT, 0, s>>>(blk, (uint32_t)grid, a.total);
    k_set_pass<true><<<grid, kT, 0, s>>>(a, set_slot, set, blk);
    alk::g_kernel_launches += 2;
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_scan, kT, 0);
    int grid = std::max(1, std::min<int>((int)ntiles, sm_count() * std::max(occ, 1)));
    k_scan<<<grid, kT, 0, s>>>(a);
  }
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  uint64_t res[2];
  int h_err = 0;
  CK(cudaMemcpyAsync(res, lb + 2 * (size_t)ntiles, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&h_err, a.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *h_count = res[0];
  if (h_err) return h_err;
  return res[0] > cap ? ALK_ERR_OVERFLOW : ALK_OK;
}

int alk_eval(const int64_t* const* d_cols, uint32_t ncols, uint64_t n, const alk_program* prog, int64_t* d_out,
             alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return ALK_OK;
  if (!prog || ncols > kMaxCols || !program_ok(prog, ncols)) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  uint8_t* db = sc.get<uint8_t>(sizeof(alk_program) + sizeof(void*) * kMaxCols, &e);
  CK(e);
  std::vector<uint8_t> hb(sizeof(alk_program) + sizeof(void*) * kMaxCols, 0);
  std::memcpy(hb.data(), prog, sizeof(alk_program));
  if (ncols) std::memcpy(hb.data() + sizeof(alk_program), d_cols, sizeof(void*) * ncols);
  const void* src = alk::upload_source(hb.data(), hb.size(), s, &e);
  CK(e);
  CK(cudaMemcpyAsync(db, src, hb.size(), cudaMemcpyHostToDevice, s));
  k_eval<<<grid_for(n), kT, 0, s>>>((const int64_t* const*)(db + sizeof(alk_program)), ncols, n,
                                    (const alk_program*)db, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_gather(const int64_t* d_src, const uint32_t* d_idx, uint64_t n, int64_t* d_out, alk_stream stream) {
  if (n == 0) return ALK_OK;
  k_gather<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_src, d_idx, n, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_gather_u32(const uint32_t* d_src, const uint32_t* d_idx, uint64_t n, uint32_t* d_out, alk_stream stream) {
  if (n == 0) return ALK_OK;
  if (!d_src || !d_idx || !d_out) return ALK_ERR_ARG;
  k_gather_u32<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_src, d_idx, n, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_flags_compact(const uint64_t* d_flags, uint64_t n, uint32_t* d_out, uint64_t* h_count, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_count) return ALK_ERR_ARG;
  *h_count = 0;
  if (n == 0) return ALK_OK;
  if (!d_flags || !d_out || n > 0xffffffffull) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  const uint32_t ntiles = (uint32_t)((n + kTile - 1) / kTile);
  uint32_t* tflags = sc.get<uint32_t>(ntiles + 4, &e);
  CK(e);
  uint64_t* aggs = sc.get<uint64_t>(2 * (size_t)ntiles + 2, &e);
  CK(e);
  CK(cudaMemsetAsync(tflags, 0, (ntiles + 4) * sizeof(uint32_t), s));
  CompactArgs a{(const unsigned long long*)d_flags, n, ntiles, tflags, aggs, aggs + ntiles, tflags + ntiles,
                (int*)(tflags + ntiles + 1), d_out, (unsigned long long*)(aggs + 2 * ntiles)};
  k_flags_compact<<<std::min<int>(ntiles, sm_count() * 4), kT, 0, s>>>(a);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  unsigned long long res[2] = {0, 0};
  int h_err = 0;
  CK(cudaMemcpyAsync(res, aggs + 2 * ntiles, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&h_err, tflags + ntiles + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (h_err) return h_err;
  *h_count = res[0];
  return ALK_OK;
}

int alk_pair_match(const uint32_t* d_pl, const uint32_t* d_pr, uint64_t n, const int64_t* d_lcol,
                   const int64_t* d_rcol, int neq, uint64_t* d_flags, alk_stream stream) {
  if (n == 0) return ALK_OK;
  if (!d_pl || !d_pr || !d_lcol || !d_rcol || !d_flags) return ALK_ERR_ARG;
  k_pair_match<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_pl, d_pr, n, d_lcol, d_rcol, neq,
                                                             (unsigned long long*)d_flags);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_rows_mark(const uint32_t* d_rows, uint64_t n, uint64_t* d_flags, uint64_t value, alk_stream stream) {
  if (n == 0) return ALK_OK;
  if (!d_rows || !d_flags) return ALK_ERR_ARG;
  k_rows_mark<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_rows, n, (unsigned long long*)d_flags, value);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_seg_minmax(const int64_t* d_keys, const uint64_t* h_start, uint32_t nseg, int64_t* h_out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nseg == 0) return ALK_OK;
  if (!d_keys || !h_start || !h_out) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  uint64_t* d_start = sc.get<uint64_t>(nseg + 1, &e);
  CK(e);
  long long* d_out = sc.get<long long>(2 * (size_t)nseg, &e);
  CK(e);
  std::vector<long long> init(2 * (size_t)nseg);
  for (uint32_t g = 0; g < nseg; g++) {
    init[2 * g] = INT64_MAX;
    init[2 * g + 1] = INT64_MIN;
  }
  CK(cudaMemcpyAsync(d_start, h_start, (nseg + 1) * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_out, init.data(), init.size() * 8, cudaMemcpyHostToDevice, s));
  k_seg_minmax<<<grid_for(h_start[nseg]), kT, 0, s>>>(d_keys, d_start, nseg, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h_out, d_out, init.size() * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_groupby_sort(const int64_t* const* d_keys, uint32_t nkeys, const int64_t* const* d_vals,
                     const uint8_t* aggs, uint32_t nvals, uint64_t n, int64_t* const* d_out_keys,
                     int64_t* const* d_out_vals, uint32_t* d_out_first, uint64_t* h_groups, int* h_was_sorted,
                     alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_groups || nkeys == 0 || nkeys > kMaxKeys || nvals > kMaxVals || n > 0xffffffffull) return ALK_ERR_ARG;
  *h_groups = 0;
  if (h_was_sorted) *h_was_sorted = 1;
  if (n == 0) return ALK_OK;
  Scratch sc(s);
  cudaError_t e;
  const size_t ptr_bytes = sizeof(void*) * (kMaxKeys + kMaxVals) * 2 + 64;
  uint8_t* db = sc.get<uint8_t>(ptr_bytes, &e);
  CK(e);
  const uint64_t ntiles = (n + kSegTile - 1) / kSegTile;
  unsigned long long* tiles = sc.get<unsigned long long>(ntiles, &e);
  CK(e);
  unsigned long long* flags = sc.get<unsigned long long>(2, &e);
  CK(e);
  std::vector<uint8_t> hb(ptr_bytes, 0);
  const size_t o_keys = 0, o_vals = o_keys + sizeof(void*) * kMaxKeys, o_okeys = o_vals + sizeof(void*) * kMaxVals,
               o_ovals = o_okeys + sizeof(void*) * kMaxKeys, o_aggs = o_ovals + sizeof(void*) * kMaxVals;
  std::memcpy(&hb[o_keys], d_keys, sizeof(void*) * nkeys);
  if (nvals) {
    std::memcpy(&hb[o_vals], d_vals, sizeof(void*) * nvals);
    std::memcpy(&hb[o_ovals], d_out_vals, sizeof(void*) * nvals);
    std::memcpy(&hb[o_aggs], aggs, nvals);
  }
  std::memcpy(&hb[o_okeys], d_out_keys, sizeof(void*) * nkeys);
  CK(cudaMemcpyAsync(db, hb.data(), ptr_bytes, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(flags, 0, 16, s));
  SegGbArgs a{(const int64_t* const*)(db + o_keys), nkeys, (const int64_t* const*)(db + o_vals), db + o_aggs, nvals,
              n, nullptr, tiles, flags};
  // 1. already in key order?
  k_seg_check<<<grid_for(n), kT, 0, s>>>(a);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  unsigned long long bad = 0;
  CK(cudaMemcpyAsync(&bad, flags, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  uint32_t* perm = nullptr;
  if (bad) {  // 2. a stable sort on the key tuple
    if (h_was_sorted) *h_was_sorted = 0;
    perm = sc.get<uint32_t>(n, &e);
    CK(e);
    std::vector<uint8_t> desc(nkeys, 0);
    int rc = alk_sort_perm(d_keys, desc.data(), nkeys, n, perm, stream);
    if (rc) return rc;
    a.perm = perm;
  }
  // 3. heads per tile, their prefix, the group count
  k_seg_count<<<(unsigned)ntiles, kT, 0, s>>>(a);
  k_seg_scan<<<1, 1024, 0, s>>>(a, ntiles);
  alk::g_kernel_launches += 2;
  CK(cudaGetLastError());
  unsigned long long g = 0;
  CK(cudaMemcpyAsync(&g, flags + 1, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  // 4. identities, then the reduction
  if (nvals) {
    k_seg_init<<<grid_for(g * nvals), kT, 0, s>>>((int64_t* const*)(db + o_ovals), db + o_aggs, nvals, g);
    alk::g_kernel_launches++;
  }
  k_seg_reduce<<<(unsigned)ntiles, kT, 0, s>>>(a, (int64_t* const*)(db + o_okeys), (int64_t* const*)(db + o_ovals),
                                                d_out_first);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  *h_groups = g;
  return ALK_OK;
}

int alk_groupby_hash(const int64_t* const* d_keys, uint32_t nkeys, const int64_t* const* d_vals,
                     const uint8_t* aggs, uint32_t nvals, uint64_t n, int64_t* const* d_out_keys,
                     int64_t* const* d_out_vals, uint32_t* d_out_first, uint64_t* h_groups, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_groups || nkeys == 0 || nkeys > kMaxKeys || nvals > kMaxVals || n > 0xffffffffull) return ALK_ERR_ARG;
  *h_groups = 0;
  if (n == 0) return ALK_OK;
  uint64_t cap = 1024;
  while (cap < n + n / 2) cap <<= 1;
  Scratch sc(s);
  cudaError_t e;
  size_t ptr_bytes = sizeof(void*) * (kMaxKeys + kMaxVals) * 2 + 64;
  uint8_t* db = sc.get<uint8_t>(ptr_bytes, &e);
  CK(e);
  uint32_t* state = sc.get<uint32_t>(cap, &e);
  CK(e);
  uint32_t* first = sc.get<uint32_t>(cap, &e);
  CK(e);
  int64_t* tkeys = sc.get<int64_t>(cap * nkeys, &e);
  CK(e);
  int64_t* tvals = sc.get<int64_t>(cap * std::max<uint32_t>(nvals, 1), &e);
  CK(e);
  unsigned long long* ctr = sc.get<unsigned long long>(2, &e);
  CK(e);
  std::vector<uint8_t> hb(ptr_bytes, 0);
  size_t o_keys = 0, o_vals = o_keys + sizeof(void*) * kMaxKeys, o_okeys = o_vals + sizeof(void*) * kMaxVals,
         o_ovals = o_okeys + sizeof(void*) * kMaxKeys, o_aggs = o_ovals + sizeof(void*) * kMaxVals;
  std::memcpy(&hb[o_keys], d_keys, sizeof(void*) * nkeys);
  if (nvals) {
    std::memcpy(&hb[o_vals], d_vals, sizeof(void*) * nvals);
    std::memcpy(&hb[o_ovals], d_out_vals, sizeof(void*) * nvals);
    std::memcpy(&hb[o_aggs], aggs, nvals);
  }
  std::memcpy(&hb[o_okeys], d_out_keys, sizeof(void*) * nkeys);
  CK(cudaMemcpyAsync(db, hb.data(), ptr_bytes, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), s));
  GbArgs a{(const int64_t* const*)(db + o_keys), nkeys, (const int64_t* const*)(db + o_vals), db + o_aggs, nvals,
           n, cap, state, tkeys, tvals, first, ctr, (int*)(ctr + 1)};
  k_gb_init<<<grid_for(cap), kT, 0, s>>>(a);
  k_gb_insert<<<grid_for(n), kT, 0, s>>>(a);
  k_gb_compact<<<grid_for(cap), kT, 0, s>>>(a, (int64_t* const*)(db + o_okeys), (int64_t* const*)(db + o_ovals),
                                            d_out_first);
  alk::g_kernel_launches += 3;
  CK(cudaGetLastError());
  unsigned long long res[2];
  CK(cudaMemcpyAsync(res, ctr, sizeof(res), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *h_groups = res[0];
  return (int)res[1];
}

static int sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t n, uint64_t* k2, uint32_t* v2, uint32_t* hist,
                      unsigned long long* mm, cudaStream_t s) {
  // significant bits only: bits above the highest differing bit of min^max are equal
  unsigned long long h_mm[2] = {~0ull, 0ull};
  CK(cudaMemcpyAsync(mm, h_mm, sizeof(h_mm), cudaMemcpyHostToDevice, s));
  k_minmax_u64<<<grid_for(n), kT, 0, s>>>(keys, n, mm);
  alk::g_kernel_launches++;
  CK(cudaMemcpyAsync(h_mm, mm, sizeof(h_mm), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  uint64_t diff = h_mm[0] ^ h_mm[1];
  int hi = diff ? 64 - __builtin_clzll(diff) : 0;
  uint32_t nblocks = (uint32_t)((n + kTile - 1) / kTile);
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = k2;
  uint32_t* vb = v2;
  for (int shift = 0; shift < hi; shift += kRadixBits) {
    k_radix_hist<<<nblocks, kT, 0, s>>>(ka, n, shift, hist, nblocks);
    k_scan_small<<<1, 1024, 0, s>>>(hist, nblocks * kRadix);
    k_radix_scatter<<<nblocks, kT, 0, s>>>(ka, va, n, shift, hist, nblocks, kb, vb);
    alk::g_kernel_launches += 3;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  CK(cudaGetLastError());
  if (ka != keys) {
    CK(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  return ALK_OK;
}

int alk_sort_perm(const int64_t* const* d_keys, const uint8_t* desc, uint32_t nkeys, uint64_t n, uint32_t* d_perm,
                  alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return ALK_OK;
  if (n > 0xffffffffull || nkeys == 0) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  uint64_t* k1 = sc.get<uint64_t>(n, &e);
  CK(e);
  uint64_t* k2 = sc.get<uint64_t>(n, &e);
  CK(e);
  uint32_t* v2 = sc.get<uint32_t>(n, &e);
  CK(e);
  uint32_t nblocks = (uint32_t)((n + kTile - 1) / kTile);
  uint32_t* hist = sc.get<uint32_t>((size_t)nblocks * kRadix, &e);
  CK(e);
  unsigned long long* mm = sc.get<unsigned long long>(2, &e);
  CK(e);
  k_iota<<<grid_for(n), kT, 0, s>>>(d_perm, n);
  alk::g_kernel_launches++;
  for (uint32_t k = nkeys; k-- > 0;) {
    k_sortkey_i64<<<grid_for(n), kT, 0, s>>>(d_keys[k], k == nkeys - 1 ? nullptr : d_perm, n, desc ? desc[k] : 0, k1);
    alk::g_kernel_launches++;
    if (k != nkeys - 1) {
      // keys were gathered through the current permutation: sort (key, perm) pairs
    }
    int rc = sort_pairs(k1, d_perm, n, k2, v2, hist, mm, s);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_sort_perm_u64(const uint64_t* d_key, uint64_t n, uint32_t* d_perm, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return ALK_OK;
  if (n > 0xffffffffull) return ALK_ERR_ARG;
  Scratch sc(s);
  cudaError_t e;
  uint64_t* k1 = sc.get<uint64_t>(n, &e);
  CK(e);
  uint64_t* k2 = sc.get<uint64_t>(n, &e);
  CK(e);
  uint32_t* v2 = sc.get<uint32_t>(n, &e);
  CK(e);
  uint32_t nblocks = (uint32_t)((n + kTile - 1) / kTile);
  uint32_t* hist = sc.get<uint32_t>((size_t)nblocks * kRadix, &e);
  CK(e);
  unsigned long long* mm = sc.get<unsigned long long>(2, &e);
  CK(e);
  CK(cudaMemcpyAsync(k1, d_key, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  k_iota<<<grid_for(n), kT, 0, s>>>(d_perm, n);
  alk::g_kernel_launches++;
  int rc = sort_pairs(k1, d_perm, n, k2, v2, hist, mm, s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_widen_u32(const uint32_t* d_in, uint64_t n, int64_t* d_out, alk_stream stream) {
  if (n == 0) return ALK_OK;
  k_widen<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_in, n, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}
int alk_for_reencode(const int64_t* d_in, uint64_t n, void* d_out, size_t out_cap, int64_t* h_lower, uint32_t* h_bits,
                     alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_lower || !h_bits || (n && (!d_in || !d_out))) return ALK_ERR_ARG;
  *h_lower = 0;
  *h_bits = 8;
  if (n == 0) return ALK_OK;
  long long* mm = nullptr;
  CK(cudaMallocAsync((void**)&mm, 16, s));
  const long long init[2] = {INT64_MAX, INT64_MIN};
  CK(cudaMemcpyAsync(mm, init, 16, cudaMemcpyHostToDevice, s));
  k_minmax_i64<<<grid_for(n), kT, 0, s>>>(d_in, n, mm);
  alk::g_kernel_launches++;
  long long h[2];
  CK(cudaMemcpyAsync(h, mm, 16, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint64_t span = (uint64_t)h[1] - (uint64_t)h[0];
  const uint32_t bits = span < (1ull << 8) ? 8 : span < (1ull << 16) ? 16 : span < (1ull << 32) ? 32 : 64;
  if (out_cap < n * (bits / 8)) {
    cudaFreeAsync(mm, s);
    return ALK_ERR_OVERFLOW;
  }
  switch (bits) {
    case 8: k_for_narrow<uint8_t><<<grid_for(n), kT, 0, s>>>(d_in, n, mm, (uint8_t*)d_out); break;
    case 16: k_for_narrow<uint16_t><<<grid_for(n), kT, 0, s>>>(d_in, n, mm, (uint16_t*)d_out); break;
    case 32: k_for_narrow<uint32_t><<<grid_for(n), kT, 0, s>>>(d_in, n, mm, (uint32_t*)d_out); break;
    default: k_for_narrow<uint64_t><<<grid_for(n), kT, 0, s>>>(d_in, n, mm, (uint64_t*)d_out); break;
  }
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaFreeAsync(mm, s));
  *h_lower = h[0];
  *h_bits = bits;
  return ALK_OK;
}

int alk_narrow_u32(const int64_t* d_in, uint64_t n, uint32_t* d_out, alk_stream stream) {
  if (n == 0) return ALK_OK;
  k_narrow<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d_in, n, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

struct alk_join_table {
  uint64_t cap = 0, n = 0;
  int64_t* key = nullptr;
  uint32_t* row = nullptr;
};

int alk_join_build(const int64_t* d_keys, uint64_t n, alk_join_table** out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out || n >= 0xffffffffull) return ALK_ERR_ARG;
  auto* t = new alk_join_table();
  t->n = n;
  t->cap = 1024;
  while (t->cap < 2 * n) t->cap <<= 1;
  cudaError_t e = cudaMallocAsync((void**)&t->key, t->cap * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&t->row, (t->cap + 2) * sizeof(uint32_t), s);
  if (e != cudaSuccess) {
    alk_join_free(t, stream);
    return alk::cuda_fail(e);
  }
  CK(cudaMemsetAsync(t->row, 0, (t->cap + 2) * sizeof(uint32_t), s));
  int* err = (int*)(t->row + t->cap);
  if (n) {
    k_join_build<<<grid_for(n), kT, 0, s>>>(d_keys, n, t->cap, t->key, t->row, err);
    alk::g_kernel_launches++;
  }
  CK(cudaGetLastError());
  int h_err = 0;
  CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaMemsetAsync(err, 0, sizeof(int), s));
  if (h_err) {
    alk_join_free(t, stream);
    return h_err;
  }
  *out = t;
  return ALK_OK;
}

int alk_join_probe(const alk_join_table* t, const int64_t* d_keys, uint64_t n, uint32_t* d_left, uint32_t* d_right,
                   uint64_t cap, uint64_t* h_pairs, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!t || !h_pairs || n >= 0xffffffffull) return ALK_ERR_ARG;
  *h_pairs = 0;
  if (n == 0 || t->n == 0) return ALK_OK;
  Scratch sc(s);
  cudaError_t e;
  unsigned long long* cnt = sc.get<unsigned long long>(1, &e);
  CK(e);
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
  k_join_probe<<<grid_for(n), kT, 0, s>>>(d_keys, n, t->cap, t->key, t->row, d_left, d_right, cap, cnt);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *h_pairs = h;
  return h > cap ? ALK_ERR_OVERFLOW : ALK_OK;
}

void alk_join_free(alk_join_table* t, alk_stream stream) {
  if (!t) return;
  cudaStream_t s = (cudaStream_t)stream;
  if (t->key) cudaFreeAsync(t->key, s);
  if (t->row) cudaFreeAsync(t->row, s);
  delete t;
}

}  // extern "C"
