// Fused pipeline kernels: the filter -> join -> join -> group-by -> order chain that the
// reference runs as separate materialising operators (emit_filter, emit_multijoin x2,
// emit_select, emit_order, operators.cu) runs here as
//   build stage(s): scan + predicate [+ probe of the previous stage] -> insert the join
//                   key into a MurmurHash64A linear-probing table with payload columns,
//   probe-aggregate: scan + predicate + probe -> exact int64 aggregates per build row,
//   top-k: threshold selection for ORDER BY ... LIMIT.
#include <algorithm>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"
#include "pipeline.h"
#include "scan.cuh"

using namespace alkd;

namespace {
constexpr int kMaxCols = 16;

int sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Empty key marker: the byte pattern 0x80 repeated (a memset value). Tables whose key
// range contains it are refused at creation.
constexpr int64_t kEmptyKey = (int64_t)0x8080808080808080ULL;

struct HtView {
  uint64_t cap;  // power of two; keys[p] == kEmptyKey marks a free position
  int64_t* key;
  int64_t* payload;  // [npay][slot_cap]
  uint64_t slot_cap;
  uint32_t npay;
  unsigned long long* nslots;
  int* flags;  // [0] duplicate key, [1] slot overflow, [2] timeout, [3] key outside the bitmap range
  // Exact membership bitmap over [kmin, kmin + nbits) of the inserted keys (null when the
  // key range, known from the build column's zone maps, is too wide).
  uint32_t* bits;
  int64_t kmin;
  uint64_t nbits;
  // Dense (rank-addressed) table: a key's slot is its rank among the keys present, the
  // popcount of the bitmap below it (rank[w] = set bits in words < w). Keys and payload
  // are dense over slots [0, nslots); cap is then the slot capacity. Null: hash table.
  uint32_t* rank;
  // Dense tables only: 0 keys and payload stored at their ranks (build records, rank
  // prefix, scatter); 1 ranks only (bitmap and rank prefix: slots for accumulators, no
  // keys or payload stored); 2 membership only (the bitmap).
  uint32_t dense_mode;
};

__device__ __forceinline__ bool ht_member(const HtView& h, int64_t k) {
  const uint64_t o = (uint64_t)k - (uint64_t)h.kmin;
  if (o >= h.nbits) return false;
  return (__ldg(h.bits + (o >> 5)) >> (o & 31)) & 1u;
}

// Slot of a present key of a dense table (the caller knows the key is present).
__device__ __forceinline__ int64_t rank_slot(const HtView& h, int64_t k) {
  const uint64_t o = (uint64_t)k - (uint64_t)h.kmin;
  const uint32_t w = __ldg(h.bits + (o >> 5));
  return (int64_t)__ldg(h.rank + (o >> 5)) + __popc(w & ((1u << (o & 31)) - 1u));
}

__device__ __forceinline__ int64_t ht_probe(const HtView& h, int64_t k) {
  if (h.rank) {
    const uint64_t o = (uint64_t)k - (uint64_t)h.kmin;
    if (o >= h.nbits) return -1;
    const uint32_t w = __ldg(h.bits + (o >> 5));
    if (!((w >> (o & 31)) & 1u)) return -1;
    return (int64_t)__ldg(h.rank + (o >> 5)) + __popc(w & ((1u << (o & 31)) - 1u));
  }
  const uint64_t mask = h.cap - 1;
  uint64_t p = murmur_u64((uint64_t)k) & mask;
  for (uint64_t n = 0; n <= mask; n++) {
    const int64_t v = __ldg(h.key + p);
    if (v == kEmptyKey) return -1;
    if (v == k) return (int64_t)p;  // payload and accumulators are indexed by position
    p = (p + 1) & mask;
  }
  return -1;
}

// Inserts a unique key with one compare-and-swap on the key word itself; returns its
// position, or -1 for a duplicate or a full table (recorded in flags).
__device__ __forceinline__ int64_t ht_insert(const HtView& h, int64_t k) {
  const uint64_t mask = h.cap - 1;
  uint64_t p = murmur_u64((uint64_t)k) & mask;
  for (uint64_t n = 0; n <= mask; n++) {
    const int64_t old =
        (int64_t)atomicCAS((unsigned long long*)(h.key + p), (unsigned long long)kEmptyKey, (unsigned long long)k);
    if (old == kEmptyKey) {
      if (h.bits) {
        const uint64_t o = (uint64_t)k - (uint64_t)h.kmin;
        if (o < h.nbits) atomicOr(h.bits + (o >> 5), 1u << (o & 31));
        else atomicExch(h.flags + 3, 1);
      }
      return (int64_t)p;
    }
    if (old == k) {
      atomicExch(h.flags, 1);  // duplicate build key: the fused plan does not apply
      return -1;
    }
    p = (p + 1) & mask;
  }
  atomicExch(h.flags + 1, 1);
  return -1;
}

// Rows that survive a stage's scan are appended to a hit list as positions
// (segment << 32 | row within the segment). The scan kernels stream the columns every row
// needs; the hit kernel then does the per-row random work (hash probe, payload and
// aggregate-input loads, atomics) for all survivors in parallel, away from the scan's
// tile pipeline.
using Hit = uint64_t;

struct StageArgs {
  const alk_colseg* cols;  // [ncols][nseg]
  uint32_t ncols, nseg;
  const uint8_t* seg_mode;
  // Tiles of kTile rows, numbered across the scanned segments: segment g owns tiles
  // [seg_tile[g], seg_tile[g + 1]) (none when the zone maps skip it).
  const uint32_t* seg_tile;  // [nseg + 1]
  uint32_t ntiles;
  const alk_program* progs;  // [0] predicate (n_instr 0 = none), [1 + a] aggregate inputs
  uint32_t nprogs;
  int32_t probe_slot;  // fact column probed into probe_ht (-1: none)
  HtView probe;
  int need_slot;  // the stage reads the probed table's payload (else membership suffices)
  // build stage
  int32_t build_slot;
  HtView build;
  const int32_t* pay_src;  // per build payload column: < 32 scan slot, >= 32 probe payload
  // aggregate stage
  uint32_t nagg;
  const uint8_t* agg_kind;
  int64_t* acc;  // [nagg][acc_stride]
  uint64_t acc_stride;
  unsigned long long* cnt;  // rows per build slot (may be null)
  unsigned long long* rows_in;
  // survivors of the scan
  Hit* hits;                       // entries of hit_words words: [position, (key, payload...)]
  uint64_t hit_cap;                // entries
  uint32_t hit_words;              // 1: positions; 2 + npay: dense-build records
  unsigned long long* hit_count;   // entries reserved (whole chunks)
  unsigned long long* hit_rows;    // survivors appended
  int* err;
  // dense-build rank prefix over the key bitmap: per-tile set-bit counts and their
  // exclusive bases
  uint64_t* rk_aggs;
  uint64_t* rk_incls;
  uint32_t rk_tiles;
};

// Segment owning a tile: the g with seg_tile[g] <= tile < seg_tile[g + 1].
__device__ __forceinline__ uint32_t tile_segment(const uint32_t* seg_tile, uint32_t nseg, uint32_t tile) {
  uint32_t lo = 0, hi = nseg;  // seg_tile[lo] <= tile < seg_tile[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (seg_tile[mid] <= tile) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Warp-wide exclusive offsets of the lanes' hit counts; returns the warp total. Called by
// all 32 lanes.
__device__ __forceinline__ uint32_t warp_offsets(uint32_t n, uint32_t* excl) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  *excl = incl - n;
  return __shfl_sync(0xffffffffu, incl, 31);
}

// Each warp appends to chunks of kChunk entries that it reserves with one atomic, so the
// shared counter sees one atomic per kChunk survivors rather than one per warp and tile.
// The unused tail of a warp's last chunk holds kNoHit. Entries at or beyond hit_cap are
// counted but not written (the hit kernel then refuses the whole list), so a list needs
// room for the survivors plus kChunk entries per warp of the scan.
constexpr uint32_t kChunk = 128;
constexpr Hit kNoHit = ~0ull;

struct HitWriter {
  uint64_t base = 0;            // first entry of the warp's current chunk
  uint32_t fill = kChunk;       // entries used in it (a full chunk: none reserved yet)
  unsigned long long rows = 0;  // survivors the warp appended

  // Where the warp's next `total` entries go (total <= 2 * kChunk): entry i of them at
  // entry index i < avail ? b0 + i : nb + (i - avail). Warp-wide.
  struct Room {
    uint64_t b0;
    uint32_t avail;
    unsigned long long nb;
    __device__ __forceinline__ uint64_t at(uint32_t i) const { return i < avail ? b0 + i : nb + (i - avail); }
  };
  __device__ __forceinline__ Room reserve(const StageArgs& a, uint32_t total) {
    rows += total;
    Room r{base + fill, kChunk - fill, 0};
    if (total > r.avail) {  // at most two new chunks, contiguous
      if ((threadIdx.x & 31) == 0)
        r.nb = atomicAdd(a.hit_count, (unsigned long long)(total - r.avail > kChunk ? 2 * kChunk : kChunk));
      r.nb = __shfl_sync(0xffffffffu, r.nb, 0);
      const uint32_t used = total - r.avail;  // entries used of the new chunk(s)
      base = used > kChunk ? r.nb + kChunk : r.nb;
      fill = used > kChunk ? used - kChunk : used;
    } else {
      fill += total;
    }
    return r;
  }
  // Appends the lanes' live items as positions (rows base_row + k * kStride of segment
  // seg). Warp-wide.
  template <int kStride>
  __device__ __forceinline__ void append(const StageArgs& a, uint32_t live, uint32_t seg, uint64_t base_row) {
    if (!__any_sync(0xffffffffu, live)) return;
    uint32_t excl;
    const uint32_t total = warp_offsets(__popc(live), &excl);
    const Room r = reserve(a, total);
    const uint64_t pos0 = (uint64_t)seg << 32 | base_row;
    uint32_t i = excl;
    for (uint32_t m = live; m; m &= m - 1, i++) {
      const uint32_t k = __ffs(m) - 1;
      const uint64_t e = r.at(i);
      if (e < a.hit_cap) a.hits[e * a.hit_words] = pos0 + (uint64_t)k * kStride;
    }
  }
  // Appends the lanes' live items as positions row0 + k of segment seg, where each lane
  // owns the consecutive rows row0 .. row0 + 7 (blocked layout). Warp-wide.
  __device__ __forceinline__ void append_blocked(const StageArgs& a, uint32_t live, uint32_t seg, uint32_t row0) {
    if (!__any_sync(0xffffffffu, live)) return;
    uint32_t excl;
    const uint32_t total = warp_offsets(__popc(live), &excl);
    const Room r = reserve(a, total);
    const uint64_t pos0 = (uint64_t)seg << 32 | row0;
    uint32_t i = excl;
    for (uint32_t m = live; m; m &= m - 1, i++) {
      const uint64_t e = r.at(i);
      if (e < a.hit_cap) a.hits[e * a.hit_words] = pos0 + (uint32_t)(__ffs(m) - 1);
    }
  }
  // Marks the unused tail of the last chunk and publishes the warp's survivor count.
  // Warp-wide.
  __device__ __forceinline__ void finish(const StageArgs& a) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t i = fill + lane; i < kChunk; i += 32)
      if (base + i < a.hit_cap) a.hits[(base + i) * a.hit_words] = kNoHit;
    if (lane == 0 && rows) atomicAdd(a.hit_rows, rows);
  }
};

// Register-machine scan for predicates of any shape: the predicate runs per row, the
// probe key is tested against the probed table's key bitmap, survivors go to the hit list.
__global__ void __launch_bounds__(kT) k_stage_scan(const StageArgs a) {
  __shared__ alk_instr s_ins[ALK_MAX_INSTR];
  __shared__ int64_t s_consts[ALK_MAX_CONST];
  __shared__ uint32_t s_n, s_res;
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  __shared__ alk_colseg s_desc[kMaxCols];
  for (uint32_t i = threadIdx.x; i < a.progs[0].n_instr; i += kT) s_ins[i] = a.progs[0].ins[i];
  for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[i] = a.progs[0].consts[i];
  if (threadIdx.x == 0) {
    s_n = a.progs[0].n_instr;
    s_res = a.progs[0].result;
  }
  unsigned long long rows_seen = 0;
  HitWriter hw;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    __syncthreads();
    const uint32_t seg = tile_segment(a.seg_tile, a.nseg, tile);
    const uint32_t row0 = (tile - a.seg_tile[seg]) * kTile;
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
    const bool all = a.seg_mode[seg] == 1 || s_n == 0;
    const uint64_t base = (uint64_t)row0 + threadIdx.x;
    uint32_t live = 0;
#pragma unroll 1
    for (int k = 0; k < kItems; k++) {
      if (k * kT + threadIdx.x >= rows) continue;
      const uint64_t row = base + (uint64_t)k * kT;
      rows_seen++;
      auto col = [&](uint32_t slot) -> int64_t {
        const alk_colseg& d = s_desc[slot];
        return load_for(d.data, d.bits, d.lower, row);
      };
      if (!all && vm_eval<kT>(s_ins, s_n, s_res, s_consts, s_regs + threadIdx.x, col) == 0) continue;
      if (a.probe_slot >= 0 && a.probe.bits && !ht_member(a.probe, col((uint32_t)a.probe_slot))) continue;
      live |= 1u << k;
    }
    hw.append<kT>(a, live, seg, base);
  }
  hw.finish(a);
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
}

// Exact counts of one segment for the cardinality estimator's records (and the exact
// counting pass that replaces an estimate): rows passing the predicate, of those the rows
// whose probe key is in the probed table, and of those the distinct values of a key column
// (first settings of a bit in a bitmap over the key's range, cleared before the launch).
__global__ void __launch_bounds__(kT) k_card_count(const StageArgs a, uint32_t seg, int32_t key_slot, int64_t kmin,
                                                   uint64_t nbits, uint32_t* bitmap, unsigned long long* out) {
  __shared__ alk_instr s_ins[ALK_MAX_INSTR];
  __shared__ int64_t s_consts[ALK_MAX_CONST];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  __shared__ alk_colseg s_desc[kMaxCols];
  for (uint32_t i = threadIdx.x; i < a.progs[0].n_instr; i += kT) s_ins[i] = a.progs[0].ins[i];
  for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[i] = a.progs[0].consts[i];
  if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
  __syncthreads();
  const uint32_t n_ins = a.progs[0].n_instr, res = a.progs[0].result;
  const bool all = a.seg_mode[seg] == 1 || n_ins == 0;
  unsigned long long c_pass = 0, c_join = 0, c_new = 0;
  for (uint32_t tile = a.seg_tile[seg] + blockIdx.x; tile < a.seg_tile[seg + 1]; tile += gridDim.x) {
    const uint32_t row0 = (tile - a.seg_tile[seg]) * kTile;
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
#pragma unroll 1
    for (int k = 0; k < kItems; k++) {
      if (k * kT + threadIdx.x >= rows) continue;
      const uint64_t row = (uint64_t)row0 + threadIdx.x + (uint64_t)k * kT;
      auto col = [&](uint32_t slot) -> int64_t {
        const alk_colseg& d = s_desc[slot];
        return load_for(d.data, d.bits, d.lower, row);
      };
      if (!all && vm_eval<kT>(s_ins, n_ins, res, s_consts, s_regs + threadIdx.x, col) == 0) continue;
      c_pass++;
      if (a.probe_slot >= 0) {
        const int64_t pk = col((uint32_t)a.probe_slot);
        if (a.probe.bits ? !ht_member(a.probe, pk) : ht_probe(a.probe, pk) < 0) continue;
      }
      c_join++;
      if (key_slot >= 0 && nbits) {
        const uint64_t o = (uint64_t)col((uint32_t)key_slot) - (uint64_t)kmin;
        if (o < nbits) {
          const uint32_t bit = 1u << (o & 31);
          if (!(atomicOr(bitmap + (o >> 5), bit) & bit)) c_new++;
        }
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    c_pass += __shfl_xor_sync(0xffffffffu, c_pass, o);
    c_join += __shfl_xor_sync(0xffffffffu, c_join, o);
    c_new += __shfl_xor_sync(0xffffffffu, c_new, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (c_pass) atomicAdd(out, c_pass);
    if (c_join) atomicAdd(out + 1, c_join);
    if (c_new) atomicAdd(out + 2, c_new);
  }
}

// Per-survivor work of a stage, one thread per hit: the hash probe (for the payload
// position, or for membership when the probed table has no key bitmap), then either the
// build-side insert with its payload or the aggregate updates. A list that overflowed
// its capacity is refused as a whole (nothing is applied), so a rerun with a larger list
// starts from unchanged tables and accumulators.
// Per lane, the reduction of v over the lanes [lane, run_end): run_end is the end of the
// lane's run of equal slots. Warp-wide.
__device__ __forceinline__ int64_t run_reduce(int64_t v, uint32_t run_end, uint8_t kind) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (uint32_t off = 1; off < 32; off <<= 1) {
    const int64_t o = __shfl_down_sync(0xffffffffu, v, off);
    if (lane + off < run_end) v = kind == ALK_AGG_MIN ? min(v, o) : kind == ALK_AGG_MAX ? max(v, o) : v + o;
  }
  return v;
}

template <bool kBuild>
__global__ void __launch_bounds__(kT) k_stage_hits(const StageArgs a) {
  __shared__ alk_instr s_ins[8][ALK_MAX_INSTR];
  __shared__ int64_t s_consts[8][ALK_MAX_CONST];
  __shared__ uint32_t s_n[8], s_res[8];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  const uint64_t n = *(volatile unsigned long long*)a.hit_count;  // written by the scan kernel
  if (n > a.hit_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.err, ALK_ERR_OVERFLOW);
    return;
  }
  if (!kBuild) {
    for (uint32_t p = 1; p < a.nprogs; p++) {
      for (uint32_t i = threadIdx.x; i < a.progs[p].n_instr; i += kT) s_ins[p][i] = a.progs[p].ins[i];
      for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[p][i] = a.progs[p].consts[i];
      if (threadIdx.x == 0) {
        s_n[p] = a.progs[p].n_instr;
        s_res[p] = a.progs[p].result;
      }
    }
    __syncthreads();
  }
  if (!kBuild) {
    // Probe-aggregate: the warp takes 32 consecutive list entries, which a scan warp
    // appended in row order, so survivors of one build key (one slot) sit side by side.
    // Each run of equal slots is folded across its lanes, and its first lane applies it
    // with one atomic per aggregate.
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t i0 = blockIdx.x * (uint64_t)kT + (threadIdx.x & ~31u); i0 < n; i0 += (uint64_t)gridDim.x * kT) {
      const uint64_t i = i0 + lane;
      const Hit h = i < n ? a.hits[i * a.hit_words] : kNoHit;
      const uint32_t seg = (uint32_t)(h >> 32);
      const uint64_t row = h & 0xffffffffull;
      auto col = [&](uint32_t slot, int64_t j) -> int64_t {
        if (slot >= 32) return __ldg(a.probe.payload + (uint64_t)(slot - 32) * a.probe.slot_cap + j);
        const alk_colseg* d = a.cols + (uint64_t)slot * a.nseg + seg;
        const void* data = (const void*)__ldg((const unsigned long long*)&d->data);
        return load_for(data, __ldg(&d->bits), (int64_t)__ldg((const long long*)&d->lower), row);
      };
      int64_t j = -1;
      if (h != kNoHit) {
        j = ht_probe(a.probe, col((uint32_t)a.probe_slot, 0));
        // a dense table with more keys than slots flags it in its prefix pass; no slot
        // beyond the capacity is touched
        if ((uint64_t)j >= a.probe.cap) j = -1;
      }
      const bool use = j >= 0;
      const int64_t prev = __shfl_up_sync(0xffffffffu, j, 1);
      const uint32_t heads = __ballot_sync(0xffffffffu, use && (lane == 0 || prev != j));
      const uint32_t after = lane == 31 ? 0u : heads & (0xffffffffu << (lane + 1));
      const uint32_t run_end = after ? (uint32_t)__ffs(after) - 1 : 32u;
      const bool head = (heads >> lane) & 1u;
      for (uint32_t g = 0; g < a.nagg; g++) {
        const uint8_t kind = a.agg_kind[g];
        int64_t v = kind == ALK_AGG_MIN ? INT64_MAX : kind == ALK_AGG_MAX ? INT64_MIN : 0;
        if (use)
          v = kind == ALK_AGG_COUNT ? 1
                                    : vm_eval<kT>(s_ins[1 + g], s_n[1 + g], s_res[1 + g], s_consts[1 + g],
                                                  s_regs + threadIdx.x, [&](uint32_t sl) { return col(sl, j); });
        v = run_reduce(v, run_end, kind);
        if (!head) continue;
        unsigned long long* dst = (unsigned long long*)(a.acc + (uint64_t)g * a.acc_stride + j);
        if (kind == ALK_AGG_SUM || kind == ALK_AGG_COUNT) atomicAdd(dst, (unsigned long long)v);
        else if (kind == ALK_AGG_MIN) atomicMin((long long*)dst, (long long)v);
        else atomicMax((long long*)dst, (long long)v);
      }
      if (a.cnt) {
        const int64_t c = run_reduce(use ? 1 : 0, run_end, ALK_AGG_COUNT);
        if (head) atomicAdd(a.cnt + j, (unsigned long long)c);
      }
    }
    return;
  }
  // build stages: one survivor per thread
  unsigned long long inserted = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const Hit* e = a.hits + i * a.hit_words;
    const Hit h = e[0];
    if (h == kNoHit) continue;  // unused tail of a warp's last chunk
    const uint32_t seg = (uint32_t)(h >> 32);
    const uint64_t row = h & 0xffffffffull;
    int64_t j = -1;
    auto col = [&](uint32_t slot) -> int64_t {
      if (slot >= 32) return __ldg(a.probe.payload + (uint64_t)(slot - 32) * a.probe.slot_cap + j);
      const alk_colseg* d = a.cols + (uint64_t)slot * a.nseg + seg;
      const void* data = (const void*)__ldg((const unsigned long long*)&d->data);
      return load_for(data, __ldg(&d->bits), (int64_t)__ldg((const long long*)&d->lower), row);
    };
    if (kBuild && a.build.rank) {
      // dense build: the key's rank is its slot; the record carries key and payload, or
      // they are read at the survivor's position
      int64_t key, pv[8];
      if (a.hit_words > 1) {
        key = (int64_t)e[1];
#pragma unroll
        for (uint32_t p = 0; p < 8; p++)
          if (p < a.build.npay) pv[p] = (int64_t)e[2 + p];
      } else {
        if (a.probe_slot >= 0 && (a.need_slot || !a.probe.bits)) {  // as the bitmap pass did
          j = ht_probe(a.probe, col((uint32_t)a.probe_slot));
          if (j < 0 || (uint64_t)j >= a.probe.cap) continue;  // beyond the slots: flagged overflow
        }
        key = col((uint32_t)a.build_slot);
#pragma unroll
        for (uint32_t p = 0; p < 8; p++)
          if (p < a.build.npay) pv[p] = col((uint32_t)a.pay_src[p]);
      }
      const uint64_t o = (uint64_t)key - (uint64_t)a.build.kmin;
      if (o >= a.build.nbits) continue;  // flagged by the bitmap pass
      const int64_t sl = rank_slot(a.build, key);
      if ((uint64_t)sl >= a.build.cap) continue;  // more keys than slots: flagged by the prefix pass
      a.build.key[sl] = key;
#pragma unroll
      for (uint32_t p = 0; p < 8; p++)
        if (p < a.build.npay) a.build.payload[(uint64_t)p * a.build.slot_cap + sl] = pv[p];
      continue;
    }
    if (a.probe_slot >= 0 && (a.need_slot || !a.probe.bits)) {
      j = ht_probe(a.probe, col((uint32_t)a.probe_slot));
      // a dense table with more keys than slots flags it in its prefix pass; no slot
      // beyond the capacity is touched
      if (j < 0 || (uint64_t)j >= a.probe.cap) continue;
    }
    // the key and every payload value are loaded before the insert, so that one round
    // trip covers them all
    const int64_t key = col((uint32_t)a.build_slot);
    int64_t pv[8];
#pragma unroll
    for (uint32_t p = 0; p < 8; p++)
      if (p < a.build.npay) pv[p] = col((uint32_t)a.pay_src[p]);
    const int64_t sl = ht_insert(a.build, key);
    if (sl < 0) continue;
    inserted++;
#pragma unroll
    for (uint32_t p = 0; p < 8; p++)
      if (p < a.build.npay) a.build.payload[(uint64_t)p * a.build.slot_cap + sl] = pv[p];
  }
  for (int o = 16; o; o >>= 1) inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
  if ((threadIdx.x & 31) == 0 && inserted) atomicAdd(a.build.nslots, inserted);
}

// Dense build from a list of survivor positions: set each survivor's key bit (a bit found
// set already is a duplicate key; a key outside the bitmap range is flagged).
__global__ void __launch_bounds__(kT) k_rank_mark(const StageArgs a) {
  const uint64_t n = *(volatile unsigned long long*)a.hit_count;
  if (n > a.hit_cap) {
    // the scatter pass reports the overflow; a table that stores no keys has none
    if (a.build.dense_mode && blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.err, ALK_ERR_OVERFLOW);
    return;
  }
  unsigned long long inserted = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const Hit h = a.hits[i * a.hit_words];
    if (h == kNoHit) continue;
    const uint32_t seg = (uint32_t)(h >> 32);
    const uint64_t row = h & 0xffffffffull;
    auto col = [&](uint32_t slot) -> int64_t {
      const alk_colseg* d = a.cols + (uint64_t)slot * a.nseg + seg;
      const void* data = (const void*)__ldg((const unsigned long long*)&d->data);
      return load_for(data, __ldg(&d->bits), (int64_t)__ldg((const long long*)&d->lower), row);
    };
    if (a.probe_slot >= 0 && !a.probe.bits && ht_probe(a.probe, col((uint32_t)a.probe_slot)) < 0) continue;
    const int64_t key = col((uint32_t)a.build_slot);
    const uint64_t o = (uint64_t)key - (uint64_t)a.build.kmin;
    if (o >= a.build.nbits) {
      atomicExch(a.build.flags + 3, 1);
      continue;
    }
    const uint32_t bit = 1u << (o & 31);
    if (atomicOr(a.build.bits + (o >> 5), bit) & bit) atomicExch(a.build.flags, 1);
    else inserted++;
  }
  // the key count of a membership-only table (the rank prefix counts the others)
  if (a.build.dense_mode == 2) {
    for (int o = 16; o; o >>= 1) inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
    if ((threadIdx.x & 31) == 0 && inserted) atomicAdd(a.build.nslots, inserted);
  }
}

// rank[w] = set bits in words < w of the dense table's bitmap, as a three-pass scan over
// tiles of 2048 words: tile sums, one block's scan of the sums, then each tile's ranks.
// The total is the key count. A key count above the slot capacity is flagged, and, for
// survivors recorded by the scan (one record per survivor, every one a member), a key
// count below the survivor count means duplicate keys.
constexpr uint32_t kRankTile = kT * 8;
// The thread's 8 consecutive bitmap words (two 16-byte loads; the bitmap and the rank
// array of a dense table start on 16-byte boundaries) and their set-bit counts.
__device__ __forceinline__ uint64_t rank_tile_counts(const HtView& h, uint32_t tile, uint32_t (&c)[8]) {
  const uint64_t nwords = (h.nbits + 31) / 32;
  const uint64_t w0 = (uint64_t)tile * kRankTile + (uint64_t)threadIdx.x * 8;  // blocked
  uint32_t w[8];
  if (w0 + 8 <= nwords) {
    const uint4 p = ((const uint4*)(h.bits + w0))[0], q = ((const uint4*)(h.bits + w0))[1];
    w[0] = p.x, w[1] = p.y, w[2] = p.z, w[3] = p.w, w[4] = q.x, w[5] = q.y, w[6] = q.z, w[7] = q.w;
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) w[k] = w0 + k < nwords ? h.bits[w0 + k] : 0u;
  }
  uint64_t sum = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    c[k] = (uint32_t)__popc(w[k]);
    sum += c[k];
  }
  return sum;
}
__global__ void __launch_bounds__(kT) k_rank_sums(const StageArgs a) {
  __shared__ uint64_t s_warp[kT / 32 + 1];
  uint32_t c[8];
  const uint64_t sum = rank_tile_counts(a.build, blockIdx.x, c);
  uint64_t tot;
  block_excl_scan<kT>(sum, s_warp, &tot);
  if (threadIdx.x == 0) a.rk_aggs[blockIdx.x] = tot;
}
constexpr int kRankScanThreads = 1024;
__global__ void __launch_bounds__(kRankScanThreads) k_rank_scan_sums(const StageArgs a) {
  __shared__ uint64_t s_warp[kRankScanThreads / 32 + 1];
  const HtView& h = a.build;
  const uint32_t per = (a.rk_tiles + kRankScanThreads - 1) / kRankScanThreads;  // consecutive tiles per thread
  const uint32_t t0 = threadIdx.x * per;
  uint64_t sum = 0;
  for (uint32_t i = 0; i < per; i++)
    if (t0 + i < a.rk_tiles) sum += a.rk_aggs[t0 + i];
  uint64_t tot;
  uint64_t run = block_excl_scan<kRankScanThreads>(sum, s_warp, &tot);
  for (uint32_t i = 0; i < per; i++) {
    if (t0 + i >= a.rk_tiles) break;
    const uint64_t v = a.rk_aggs[t0 + i];
    a.rk_incls[t0 + i] = run;  // exclusive base of the tile
    run += v;
  }
  if (threadIdx.x == 0) {
    *h.nslots = tot;
    if (tot > h.cap) atomicExch(h.flags + 1, 1);
    if (a.hit_words > 1 && *(volatile unsigned long long*)a.hit_rows != tot) atomicExch(h.flags, 1);
  }
}
__global__ void __launch_bounds__(kT) k_rank_write(const StageArgs a) {
  __shared__ uint64_t s_warp[kT / 32 + 1];
  const HtView& h = a.build;
  const uint64_t nwords = (h.nbits + 31) / 32;
  uint32_t c[8];
  const uint64_t sum = rank_tile_counts(h, blockIdx.x, c);
  uint64_t tot;
  uint64_t r = a.rk_incls[blockIdx.x] + block_excl_scan<kT>(sum, s_warp, &tot);
  const uint64_t w0 = (uint64_t)blockIdx.x * kRankTile + (uint64_t)threadIdx.x * 8;
  uint32_t rk[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    rk[k] = (uint32_t)r;
    r += c[k];
  }
  if (w0 + 8 <= nwords) {
    ((uint4*)(h.rank + w0))[0] = make_uint4(rk[0], rk[1], rk[2], rk[3]);
    ((uint4*)(h.rank + w0))[1] = make_uint4(rk[4], rk[5], rk[6], rk[7]);
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (w0 + k < nwords) h.rank[w0 + k] = rk[k];
  }
}

__global__ void __launch_bounds__(kT) k_fill_i64(int64_t* p, uint64_t n, int64_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) p[i] = v;
}

// Top-k threshold: per block, the k largest ranking values among live slots.
__global__ void __launch_bounds__(kT) k_topk_local(const int64_t* rank, const unsigned long long* live, uint64_t n,
                                                   uint32_t k, int64_t* out) {
  __shared__ int64_t s_best[kT / 32];
  __shared__ int64_t s_prev;
  __shared__ uint32_t s_taken;
  const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = blockIdx.x * per, hi = min(n, lo + per);
  // k rounds of a block maximum over values strictly below the previous one, counting
  // multiplicity so that the k-th value is exact.
  int64_t prev = INT64_MAX;
  uint32_t taken = 0;
  bool first = true;
  uint32_t written = 0;
  while (written < k) {
    int64_t best = INT64_MIN;
    bool any = false;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kT) {
      if (!live[i]) continue;
      const int64_t v = rank[i];
      if (first ? true : v < prev) {
        if (!any || v > best) best = v;
        any = true;
      }
    }
    unsigned anyb = __ballot_sync(0xffffffffu, any);
    for (int o = 16; o; o >>= 1) {
      int64_t x = __shfl_xor_sync(0xffffffffu, best, o);
      best = x > best ? x : best;
    }
    if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = anyb ? best : INT64_MIN;
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    if (anyb && (threadIdx.x & 31) == 0) atomicOr(&s_any, 1);
    __syncthreads();
    if (!s_any) break;
    if (threadIdx.x == 0) {
      int64_t b = INT64_MIN;
      for (int w = 0; w < kT / 32; w++) b = s_best[w] > b ? s_best[w] : b;
      s_prev = b;
    }
    __syncthreads();
    const int64_t v = s_prev;
    // multiplicity of v in the slice
    uint32_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kT)
      if (live[i] && rank[i] == v) c++;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (threadIdx.x == 0) s_taken = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_taken, c);
    __syncthreads();
    taken = s_taken;
    for (uint32_t t = 0; t < taken && written < k; t++, written++)
      if (threadIdx.x == 0) out[(uint64_t)blockIdx.x * k + written] = v;
    prev = v;
    first = false;
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (; written < k; written++) out[(uint64_t)blockIdx.x * k + written] = INT64_MIN;
}

// Top-k threshold in one pass for k <= 16: every thread keeps its 16 largest ranking
// values (with multiplicity) in registers, then the block sorts the 4096 candidates in
// shared memory and writes its k largest.
constexpr int kTopK = 16;

// Inserts v into a descending register list, dropping the smallest.
__device__ __forceinline__ void top16_insert(int64_t (&t)[kTopK], int64_t v) {
  if (v <= t[kTopK - 1]) return;
#pragma unroll
  for (int q = kTopK - 1; q > 0; q--) {
    const int64_t up = t[q - 1];
    t[q] = v > up ? up : (v > t[q] ? v : t[q]);
  }
  t[0] = v > t[0] ? v : t[0];
}

// The warp's 16 largest values (with multiplicity) out of its lanes' descending lists:
// 16 rounds of a warp maximum over the list heads, the winning lane popping its head.
// Lane r < 16 returns the r-th largest. Warp-wide.
__device__ __forceinline__ int64_t warp_top16(int64_t (&t)[kTopK]) {
  const uint32_t lane = threadIdx.x & 31;
  int64_t mine = INT64_MIN;
#pragma unroll 1
  for (int r = 0; r < kTopK; r++) {
    int64_t m = t[0];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const int64_t x = __shfl_xor_sync(0xffffffffu, m, o);
      m = x > m ? x : m;
    }
    const uint32_t win = __ffs(__ballot_sync(0xffffffffu, t[0] == m)) - 1;
    if (lane == (uint32_t)r) mine = m;
    if (lane == win) {
#pragma unroll
      for (int q = 0; q < kTopK - 1; q++) t[q] = t[q + 1];
      t[kTopK - 1] = INT64_MIN;
    }
  }
  return mine;
}

// The block's 16 largest: warp lists through shared memory, merged by warp 0.
template <int kThreads>
__device__ __forceinline__ void block_top16(int64_t (&t)[kTopK], int64_t* s_w, int64_t* out16) {
  constexpr int kWarps = kThreads / 32;
  static_assert(kWarps * kTopK <= 32 * kTopK, "warp 0 holds at most 16 values per lane");
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t w = warp_top16(t);
  if (lane < (uint32_t)kTopK) s_w[warp * kTopK + lane] = w;
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
    for (int i = lane; i < kWarps * kTopK; i += 32) top16_insert(t, s_w[i]);
    const int64_t b = warp_top16(t);
    if (lane < (uint32_t)kTopK) out16[lane] = b;
  }
}

__global__ void __launch_bounds__(kT) k_topk_local16(const int64_t* rank, const unsigned long long* live, uint64_t n,
                                                     uint32_t k, int64_t* out) {
  __shared__ int64_t s_w[(kT / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  // kU slots per thread and round, all loads issued before any is used
  constexpr int kU = 4;
  const uint64_t step = (uint64_t)gridDim.x * kT * kU;
  for (uint64_t i0 = blockIdx.x * (uint64_t)kT * kU + threadIdx.x; i0 < n; i0 += step) {
    unsigned long long l[kU];
    int64_t r[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const uint64_t i = i0 + (uint64_t)u * kT;
      l[u] = i < n ? __ldg(live + i) : 0ull;
      r[u] = i < n ? __ldg(rank + i) : 0;
    }
#pragma unroll
    for (int u = 0; u < kU; u++)
      if (l[u]) top16_insert(t, r[u]);
  }
  block_top16<kT>(t, s_w, s_best);
  __syncthreads();
  if (threadIdx.x < k) out[(uint64_t)blockIdx.x * k + threadIdx.x] = s_best[threadIdx.x];
}

// Collect live slots whose ranking value is at least the threshold.
__global__ void __launch_bounds__(kT) k_topk_collect(const int64_t* rank, const unsigned long long* live, uint64_t n,
                                                     int64_t thr, uint32_t* out, uint64_t cap,
                                                     unsigned long long* count) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    if (!live[i] || rank[i] < thr) continue;
    unsigned long long p = atomicAdd(count, 1ull);
    if (p < cap) out[p] = (uint32_t)i;
  }
}

// Threshold on the device: the k-th largest of the per-block candidate lists (m values,
// m <= kMergeMax).
constexpr int kMergeThreads = 256;
constexpr int kMergeMax = 4096;
// slots the sampled top-k selection collects at or above its threshold, at most
constexpr uint64_t kTopKCollect = 1 << 16;
__global__ void __launch_bounds__(kMergeThreads) k_topk_merge(const int64_t* best, uint32_t m, uint32_t k,
                                                              int64_t* thr) {
  __shared__ int64_t s_w[(kMergeThreads / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  for (uint32_t i = threadIdx.x; i < m; i += kMergeThreads) top16_insert(t, best[i]);
  block_top16<kMergeThreads>(t, s_w, s_best);
  __syncthreads();
  if (threadIdx.x == 0) *thr = s_best[k - 1];
}

// Collect live slots whose ranking value is at least the device-side threshold.
__global__ void __launch_bounds__(kT) k_topk_collect_dev(const int64_t* rank, const unsigned long long* live,
                                                         uint64_t n, const int64_t* thr_p, uint32_t* out,
                                                         uint64_t cap, unsigned long long* count) {
  const int64_t thr = *thr_p;
  constexpr int kU = 4;
  const uint64_t step = (uint64_t)gridDim.x * kT * kU;
  for (uint64_t i0 = blockIdx.x * (uint64_t)kT * kU + threadIdx.x; i0 < n; i0 += step) {
    unsigned long long l[kU];
    int64_t r[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const uint64_t i = i0 + (uint64_t)u * kT;
      l[u] = i < n ? __ldg(live + i) : 0ull;
      r[u] = i < n ? __ldg(rank + i) : 0;
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      if (!l[u] || r[u] < thr) continue;
      const unsigned long long p = atomicAdd(count, 1ull);
      if (p < cap) out[p] = (uint32_t)(i0 + (uint64_t)u * kT);
    }
  }
}

// Sampled threshold for the top-k selection: per block, the k largest ranking values
// among the live slots i * kSampleStride (a thread holds a few samples, so its list
// inserts are few). The k-th largest of a sample is at most the k-th largest of all
// slots, so every slot at or above the true threshold is at or above the sample's.
constexpr uint32_t kSampleStride = 64;
__global__ void __launch_bounds__(kT) k_topk_sample(const int64_t* rank, const unsigned long long* live, uint64_t n,
                                                    uint32_t k, int64_t* out) {
  __shared__ int64_t s_w[(kT / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  const uint64_t ns = (n + kSampleStride - 1) / kSampleStride;
  for (uint64_t j = blockIdx.x * (uint64_t)kT + threadIdx.x; j < ns; j += (uint64_t)gridDim.x * kT) {
    const uint64_t i = j * kSampleStride;
    if (__ldg(live + i)) top16_insert(t, __ldg(rank + i));
  }
  block_top16<kT>(t, s_w, s_best);
  __syncthreads();
  if (threadIdx.x < k) out[(uint64_t)blockIdx.x * k + threadIdx.x] = s_best[threadIdx.x];
}

// Exact selection among the slots collected at or above the sampled threshold: their k-th
// largest value is the true threshold (they include every slot at or above it), and the
// ones at or above it are the result. When more slots were collected than fit (ties at
// the sampled threshold), *fallback is set and the exact full pass runs instead.
__global__ void __launch_bounds__(kMergeThreads) k_topk_refine(const int64_t* rank, const uint32_t* cand,
                                                               const unsigned long long* ncand, uint64_t cap,
                                                               uint32_t k, uint32_t* out, uint64_t out_cap,
                                                               unsigned long long* count, int* fallback) {
  __shared__ int64_t s_w[(kMergeThreads / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  const unsigned long long m = *ncand;
  if (m > cap) {
    if (threadIdx.x == 0) *fallback = 1;
    return;
  }
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  for (uint64_t i = threadIdx.x; i < m; i += kMergeThreads) top16_insert(t, rank[cand[i]]);
  block_top16<kMergeThreads>(t, s_w, s_best);
  __syncthreads();
  const int64_t thr = s_best[k - 1];
  for (uint64_t i = threadIdx.x; i < m; i += kMergeThreads) {
    const uint32_t c = cand[i];
    if (rank[c] < thr) continue;
    const unsigned long long p = atomicAdd(count, 1ull);
    if (p < out_cap) out[p] = c;
  }
}

// The exact full pass, run only when the sampled selection fell back (the flag is set on
// the device, so the sequence needs no host round trip and can be captured in a graph).
__global__ void __launch_bounds__(kT) k_topk_local16_if(const int* fallback, const int64_t* rank,
                                                        const unsigned long long* live, uint64_t n, uint32_t k,
                                                        int64_t* out) {
  if (!*fallback) return;
  __shared__ int64_t s_w[(kT / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT)
    if (__ldg(live + i)) top16_insert(t, __ldg(rank + i));
  block_top16<kT>(t, s_w, s_best);
  __syncthreads();
  if (threadIdx.x < k) out[(uint64_t)blockIdx.x * k + threadIdx.x] = s_best[threadIdx.x];
}
__global__ void __launch_bounds__(kMergeThreads) k_topk_merge_if(const int* fallback, const int64_t* best, uint32_t m,
                                                                 uint32_t k, int64_t* thr) {
  if (!*fallback) return;
  __shared__ int64_t s_w[(kMergeThreads / 32) * kTopK];
  __shared__ int64_t s_best[kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  for (uint32_t i = threadIdx.x; i < m; i += kMergeThreads) top16_insert(t, best[i]);
  block_top16<kMergeThreads>(t, s_w, s_best);
  __syncthreads();
  if (threadIdx.x == 0) *thr = s_best[k - 1];
}
__global__ void __launch_bounds__(kT) k_topk_collect_if(const int* fallback, const int64_t* rank,
                                                        const unsigned long long* live, uint64_t n,
                                                        const int64_t* thr_p, uint32_t* out, uint64_t cap,
                                                        unsigned long long* count) {
  if (!*fallback) return;
  const int64_t thr = *thr_p;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    if (!__ldg(live + i) || __ldg(rank + i) < thr) continue;
    const unsigned long long p = atomicAdd(count, 1ull);
    if (p < cap) out[p] = (uint32_t)i;
  }
}

// Rows idx[0 .. min(*count, cap)) of up to kGatherCols int64 columns, column-major into
// out[c * cap + r].
constexpr int kGatherCols = 32;
struct GatherCols {
  const int64_t* col[kGatherCols];
};
__global__ void __launch_bounds__(kT) k_gather_rows(const __grid_constant__ GatherCols g, uint32_t ncols,
                                                    const uint32_t* idx, const unsigned long long* count,
                                                    uint64_t cap, int64_t* out) {
  const uint64_t n = min((uint64_t)*count, cap);
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n * ncols; t += (uint64_t)gridDim.x * kT) {
    const uint64_t c = t / n, r = t - c * n;
    out[c * cap + r] = g.col[c][idx[r]];
  }
}

__global__ void __launch_bounds__(kT) k_live_compact(const unsigned long long* live, uint64_t n, uint32_t* out,
                                                     unsigned long long* count) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    if (!live[i]) continue;
    out[atomicAdd(count, 1ull)] = (uint32_t)i;
  }
}

// ---------------------------------------------------------------- conjunctive fast path
// Predicates of the shape AND_i (column_i * mul_i OP const_i), which is what the host
// compiles for the reference's "column OP constant" filters (filter.cu:473-590), run as
// straight-line tests over values loaded for the whole item batch at once; probes test
// the table's exact key bitmap before touching the hash table.
struct FastArgs {
  StageArgs a;
  Conj conj[kMaxConj];
  uint32_t nconj;
  // Per conjunct and segment ([nconj][nseg]), the test rewritten on the stored value x
  // (value = x + lower): most conjuncts become one unsigned range test on x.
  const struct ConjSeg* cseg;
  // Per segment ([nseg]): whether the scan may run in 32-bit arithmetic, and the probe
  // key's stored-value offset into the probed table's key bitmap.
  const struct SegPlan* splan;
};

struct SegPlan {
  uint32_t narrow;  // every staged column stores <= 32 bits: 32-bit evaluation
  // probe key x (stored value) against the key bitmap, in 32 bits: member when
  // x - xlo <= xspan (unsigned) and bit (x - xlo + boff) is set; kmember 0: no stored
  // value of the segment lies in the bitmap's key range
  uint32_t kmember;
  uint32_t xlo, xspan, boff, pad;
};

// Drops the thread's items whose probe key (stored value x + lower) is absent from the
// probed table's key bitmap.
// The key-bitmap tests load all of the thread's bitmap words before testing any: the
// loads are independent round trips to L2, issued back to back (an item already dropped
// reads word 0 and is not tested).
__device__ __forceinline__ uint32_t probe_filter(const HtView& h, int64_t lower, const uint64_t (&x)[kItems],
                                                 uint32_t live) {
  uint64_t o[kItems];
  uint32_t w[kItems];
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    o[k] = x[k] + (uint64_t)lower - (uint64_t)h.kmin;
    if (!(((live >> k) & 1) && o[k] < h.nbits)) {
      live &= ~(1u << k);
      o[k] = 0;
    }
  }
#pragma unroll
  for (int k = 0; k < kItems; k++) w[k] = __ldg(h.bits + (o[k] >> 5));
#pragma unroll
  for (int k = 0; k < kItems; k++)
    if (!((w[k] >> (o[k] & 31)) & 1u)) live &= ~(1u << k);
  return live;
}

__device__ __forceinline__ uint32_t probe_filter32(const HtView& h, const SegPlan& sp, const uint32_t (&x)[kItems],
                                                   uint32_t live) {
  if (!sp.kmember) return 0;
  uint32_t o[kItems], w[kItems];
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    const uint32_t d = x[k] - sp.xlo;
    o[k] = d + sp.boff;
    if (d > sp.xspan) live &= ~(1u << k);
  }
  // only live items load their word (predicated loads: no memory access for the others)
#pragma unroll
  for (int k = 0; k < kItems; k++) w[k] = ((live >> k) & 1) ? __ldg(h.bits + (o[k] >> 5)) : 0u;
#pragma unroll
  for (int k = 0; k < kItems; k++)
    if (!((w[k] >> (o[k] & 31)) & 1u)) live &= ~(1u << k);
  return live;
}
__global__ void __launch_bounds__(kT) k_stage_fast(const __grid_constant__ FastArgs f) {
  const StageArgs& a = f.a;
  __shared__ alk_colseg s_desc[kMaxCols];
  __shared__ ConjSeg s_cs[kMaxConj];
  unsigned long long rows_seen = 0;
  HitWriter hw;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    __syncthreads();
    const uint32_t seg = tile_segment(a.seg_tile, a.nseg, tile);
    const uint32_t row0 = (tile - a.seg_tile[seg]) * kTile;
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    if (threadIdx.x < f.nconj) s_cs[threadIdx.x] = f.cseg[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
    const uint64_t base = (uint64_t)row0 + threadIdx.x;
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (k * kT + threadIdx.x < rows) live |= 1u << k;
    rows_seen += __popc(live);
    uint64_t x[kItems];
    if (a.seg_mode[seg] != 1) {
      for (uint32_t c = 0; c < f.nconj; c++) {
        const alk_colseg& d = s_desc[f.conj[c].slot];
        load_raw<true>(d.data, d.bits, base, live, x);
        live = conj_filter(f.conj[c], s_cs[c], d.lower, x, live);
      }
    }
    if (live && a.probe_slot >= 0 && a.probe.bits) {
      const alk_colseg& d = s_desc[a.probe_slot];
      load_raw<true>(d.data, d.bits, base, live, x);
      live = probe_filter(a.probe, d.lower, x, live);
    }
    hw.append<kT>(a, live, seg, base);
  }
  hw.finish(a);
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
}

// ---------------------------------------------------------------- TMA-staged stage
// The conjunctive scan with the columns every row needs (conjunct columns and the probe
// key) brought into shared memory by bulk asynchronous copies (cp.async.bulk, completion
// on a "full" mbarrier). One producer warp keeps kStages tiles in flight per block; kCW
// consumer warps each evaluate a 256-row slice of a tile and release the stage through
// an "empty" mbarrier, so no block-wide barrier sits in the loop and a warp waiting on
// its key-bitmap loads or its hit-list atomic does not hold the others back. Columns read
// only for surviving rows (payload, aggregate inputs) are left to the hit kernel.
constexpr int kStaged = 6;          // staged columns at most
constexpr int kCW = kTile / (32 * kItems);   // consumer warps
constexpr int kTmaThreads = (kCW + 1) * 32;  // + one producer warp

constexpr uint32_t kMaxStages = 4;  // tiles in flight per block, at most

struct TmaArgs {
  FastArgs f;
  uint32_t nstaged;
  uint32_t staged_slot[kStaged];  // scan slot of each staged column
  uint32_t col_off[kStaged];      // byte offset of each staged column in a stage buffer
  uint32_t stage_bytes;           // shared bytes of one stage (all staged columns, kTile rows)
  uint32_t nst;                   // stages in flight (2 .. kMaxStages)
  uint32_t conj_st[kMaxConj];     // staged index of each conjunct's column
  int32_t probe_st;               // staged index of the probe key (-1: no probe)
  // Build stage whose key and payload are all scan columns: the consumers insert their
  // survivors straight from the staged tile (no hit list).
  uint32_t inline_build;
  uint32_t key_st;     // staged index of the build key
  uint32_t pay_st[8];  // staged index of each payload column
};

// Dynamic shared memory of k_stage_tma: nst stage buffers, then the segment tile prefix,
// the staged columns' per-segment descriptors, the conjuncts' per-segment raw-domain
// tests and the per-segment plans, so that issuing and evaluating a tile read shared
// memory only.
__host__ __device__ inline uint32_t tma_tile_table_off(uint32_t stage_bytes, uint32_t nst) {
  return nst * stage_bytes;
}
__host__ __device__ inline uint32_t tma_desc_off(uint32_t stage_bytes, uint32_t nst, uint32_t nseg) {
  return (tma_tile_table_off(stage_bytes, nst) + (nseg + 1) * 4 + 15) & ~15u;
}
__host__ __device__ inline uint32_t tma_cseg_off(uint32_t stage_bytes, uint32_t nst, uint32_t nseg, uint32_t nstaged) {
  return tma_desc_off(stage_bytes, nst, nseg) + nstaged * nseg * (uint32_t)sizeof(alk_colseg);
}
__host__ __device__ inline uint32_t tma_splan_off(uint32_t stage_bytes, uint32_t nst, uint32_t nseg,
                                                  uint32_t nstaged, uint32_t nconj) {
  return tma_cseg_off(stage_bytes, nst, nseg, nstaged) + nconj * nseg * (uint32_t)sizeof(ConjSeg);
}
__host__ __device__ inline uint32_t tma_smem_bytes(uint32_t stage_bytes, uint32_t nst, uint32_t nseg,
                                                   uint32_t nstaged, uint32_t nconj) {
  return tma_splan_off(stage_bytes, nst, nseg, nstaged, nconj) + nseg * (uint32_t)sizeof(SegPlan);
}

// Decoded value of row r of a staged column.
__device__ __forceinline__ int64_t staged_value(const unsigned char* p, const alk_colseg& d, uint32_t r) {
  uint64_t x;
  switch (d.bits) {
    case 8: x = p[r]; break;
    case 16: x = ((const uint16_t*)p)[r]; break;
    case 32: x = ((const uint32_t*)p)[r]; break;
    default: x = ((const unsigned long long*)p)[r]; break;
  }
  return (int64_t)(x + (uint64_t)d.lower);
}

__global__ void __launch_bounds__(kTmaThreads) k_stage_tma(const __grid_constant__ TmaArgs t) {
  const FastArgs& f = t.f;
  const StageArgs& a = f.a;
  const uint32_t nst = t.nst;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ __align__(8) uint64_t s_full[kMaxStages], s_empty[kMaxStages];
  __shared__ int s_abort;
  __shared__ uint16_t s_rows[kCW * 32 * kItems];  // per consumer warp: survivors of its slice (inline build)
  uint32_t* s_tile = (uint32_t*)(s_dyn + tma_tile_table_off(t.stage_bytes, nst));
  alk_colseg* s_cd = (alk_colseg*)(s_dyn + tma_desc_off(t.stage_bytes, nst, a.nseg));  // [nstaged][nseg]
  ConjSeg* s_cs = (ConjSeg*)(s_dyn + tma_cseg_off(t.stage_bytes, nst, a.nseg, t.nstaged));  // [nconj][nseg]
  for (uint32_t i = threadIdx.x; i <= a.nseg; i += kTmaThreads) s_tile[i] = a.seg_tile[i];
  for (uint32_t i = threadIdx.x; i < t.nstaged * a.nseg; i += kTmaThreads)
    s_cd[i] = a.cols[t.staged_slot[i / a.nseg] * a.nseg + i % a.nseg];
  for (uint32_t i = threadIdx.x; i < f.nconj * a.nseg; i += kTmaThreads) s_cs[i] = f.cseg[i];
  SegPlan* s_sp = (SegPlan*)(s_dyn + tma_splan_off(t.stage_bytes, nst, a.nseg, t.nstaged, f.nconj));  // [nseg]
  for (uint32_t i = threadIdx.x; i < a.nseg; i += kTmaThreads) s_sp[i] = f.splan[i];
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (uint32_t i = 0; i < nst; i++) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], kCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int* abort_flag = &s_abort;

  if (warp == kCW) {
    // ---- producer: one thread issues the bulk copies of the block's tiles
    if (lane != 0) return;
    uint32_t issued = 0;
    for (uint32_t it = 0;; it++) {
      const uint32_t tile = blockIdx.x + it * gridDim.x;
      if (tile >= a.ntiles || *abort_flag) break;
      const uint32_t st = it % nst;
      if (it >= nst && !mbar_wait(&s_empty[st], (it / nst - 1) & 1)) {
        atomicExch(a.err, ALK_ERR_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      const uint32_t seg = tile_segment(s_tile, a.nseg, tile);
      const uint32_t row0 = (tile - s_tile[seg]) * kTile;
      const uint32_t rows = min((uint32_t)kTile, s_cd[seg].rows - row0);
      uint32_t total = 0;
      for (uint32_t i = 0; i < t.nstaged; i++) total += (rows * (s_cd[i * a.nseg + seg].bits / 8) + 15) & ~15u;
      unsigned char* buf = s_dyn + st * t.stage_bytes;
      mbar_expect_tx(&s_full[st], total);
      for (uint32_t i = 0; i < t.nstaged; i++) {
        const alk_colseg& d = s_cd[i * a.nseg + seg];
        const uint32_t w = d.bits / 8;
        bulk_g2s(buf + t.col_off[i], (const unsigned char*)d.data + (uint64_t)row0 * w, (rows * w + 15) & ~15u,
                 &s_full[st]);
      }
      issued = it + 1;
    }
    // every copy issued has landed before the block may exit (bounded)
    for (uint32_t it = issued > nst ? issued - nst : 0; it < issued; it++)
      mbar_wait(&s_full[it % nst], (it / nst) & 1);
    return;
  }

  // ---- consumers: warp `warp` owns rows warp * 256 + k * 32 + lane of every tile
  unsigned long long rows_seen = 0, inserted = 0, survivors = 0;  // survivors: inline builds
  HitWriter hw;
  const uint32_t r0 = warp * (32 * kItems) + lane;
  for (uint32_t it = 0;; it++) {
    const uint32_t tile = blockIdx.x + it * gridDim.x;
    if (tile >= a.ntiles || __any_sync(0xffffffffu, *abort_flag)) break;
    const uint32_t st = it % nst;
    if (!mbar_wait_warp(&s_full[st], (it / nst) & 1)) {
      if (lane == 0) {
        atomicExch(a.err, ALK_ERR_TIMEOUT);
        *abort_flag = 1;
      }
      break;
    }
    const uint32_t seg = tile_segment(s_tile, a.nseg, tile);
    const uint32_t row0 = (tile - s_tile[seg]) * kTile;
    const uint32_t rows = min((uint32_t)kTile, s_cd[seg].rows - row0);
    const unsigned char* buf = s_dyn + st * t.stage_bytes;
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (r0 + k * 32 < rows) live |= 1u << k;
    rows_seen += __popc(live);
    const SegPlan sp = s_sp[seg];
    if (sp.narrow) {
      uint32_t x[kItems];
      for (uint32_t c = 0; c < f.nconj; c++) {
        const alk_colseg& d = s_cd[t.conj_st[c] * a.nseg + seg];
        load_raw32<32>(buf + t.col_off[t.conj_st[c]], d.bits, r0, x);
        live = conj_filter32(f.conj[c], s_cs[c * a.nseg + seg], d.lower, x, live);
      }
      if (t.probe_st >= 0 && a.probe.bits) {
        const alk_colseg& d = s_cd[t.probe_st * a.nseg + seg];
        load_raw32<32>(buf + t.col_off[t.probe_st], d.bits, r0, x);
        live = probe_filter32(a.probe, sp, x, live);
      }
    } else {
      uint64_t x[kItems];
      for (uint32_t c = 0; c < f.nconj; c++) {
        const alk_colseg& d = s_cd[t.conj_st[c] * a.nseg + seg];
        load_raw<false, 32>(buf + t.col_off[t.conj_st[c]], d.bits, r0, live, x);
        live = conj_filter(f.conj[c], s_cs[c * a.nseg + seg], d.lower, x, live);
      }
      if (t.probe_st >= 0 && a.probe.bits) {
        const alk_colseg& d = s_cd[t.probe_st * a.nseg + seg];
        load_raw<false, 32>(buf + t.col_off[t.probe_st], d.bits, r0, live, x);
        live = probe_filter(a.probe, d.lower, x, live);
      }
    }
    if (t.inline_build) {
      // insert the survivors from the staged tile, then release it; the warp's survivors
      // are first compacted so that all lanes insert at once (one compare-and-swap round
      // trip per 32 survivors). A dense table takes records instead: the key's bit is set
      // and [position, key, payload] goes to the survivor list, for the rank passes.
      const bool dense = a.build.rank != nullptr;
      if (!dense) survivors += __popc(live);
      uint32_t excl;
      const uint32_t total = __any_sync(0xffffffffu, live) ? warp_offsets(__popc(live), &excl) : 0;
      uint16_t* wl = s_rows + warp * (32 * kItems);
      uint32_t q = excl;
      for (uint32_t m = total ? live : 0; m; m &= m - 1, q++) wl[q] = (uint16_t)(r0 + (__ffs(m) - 1) * 32);
      __syncwarp();
      if (dense) {
        const HitWriter::Room room = total ? hw.reserve(a, total) : HitWriter::Room{0, 0, 0};
        for (uint32_t j = lane; j < total; j += 32) {
          const uint32_t r = wl[j];
          const int64_t key = staged_value(buf + t.col_off[t.key_st], s_cd[t.key_st * a.nseg + seg], r);
          const uint64_t o = (uint64_t)key - (uint64_t)a.build.kmin;
          if (o < a.build.nbits) atomicOr(a.build.bits + (o >> 5), 1u << (o & 31));
          else atomicExch(a.build.flags + 3, 1);
          const uint64_t e = room.at(j);
          if (e >= a.hit_cap) continue;
          Hit* rec = a.hits + e * a.hit_words;
          rec[0] = (uint64_t)seg << 32 | (uint64_t)(row0 + r);
          rec[1] = (uint64_t)key;
#pragma unroll
          for (uint32_t p = 0; p < 8; p++)
            if (p < a.build.npay)
              rec[2 + p] = (uint64_t)staged_value(buf + t.col_off[t.pay_st[p]], s_cd[t.pay_st[p] * a.nseg + seg], r);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_empty[st]);
        continue;
      }
      // rounds of 32 survivors; the last round's values are read into registers and the
      // stage is released before its inserts, so the producer refills it meanwhile
      for (uint32_t j0 = 0; j0 < total; j0 += 32) {
        const uint32_t j = j0 + lane;
        const bool mine = j < total;
        int64_t key = 0, pv[8];
        if (mine) {
          const uint32_t r = wl[j];
          key = staged_value(buf + t.col_off[t.key_st], s_cd[t.key_st * a.nseg + seg], r);
#pragma unroll
          for (uint32_t p = 0; p < 8; p++)
            if (p < a.build.npay)
              pv[p] = staged_value(buf + t.col_off[t.pay_st[p]], s_cd[t.pay_st[p] * a.nseg + seg], r);
        }
        if (j0 + 32 >= total) {
          __syncwarp();
          if (lane == 0) mbar_arrive(&s_empty[st]);
        }
        const int64_t sl = mine ? ht_insert(a.build, key) : -1;
        if (sl >= 0) {
          inserted++;
#pragma unroll
          for (uint32_t p = 0; p < 8; p++)
            if (p < a.build.npay) a.build.payload[(uint64_t)p * a.build.slot_cap + sl] = pv[p];
        }
        __syncwarp();
      }
      __syncwarp();  // the survivor list is rewritten by the next tile
      if (total == 0 && lane == 0) mbar_arrive(&s_empty[st]);
      continue;
    }
    // the slice's values are in registers: release the stage to the producer
    __syncwarp();
    if (lane == 0) mbar_arrive(&s_empty[st]);
    hw.append<32>(a, live, seg, (uint64_t)row0 + r0);
  }
  hw.finish(a);
  for (int o = 16; o; o >>= 1) {
    rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
    inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
    survivors += __shfl_xor_sync(0xffffffffu, survivors, o);
  }
  if (lane == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
  if (lane == 0 && inserted) atomicAdd(a.build.nslots, inserted);
  if (lane == 0 && survivors) atomicAdd(a.hit_rows, survivors);
}

// ---------------------------------------------------------------- blocked vector-load stage
// The conjunctive scan when every scanned segment stores its tested columns in at most 32
// bits. Each thread owns 8 consecutive rows of a 2048-row tile and reads every column it
// tests with one or two 16-byte loads (one 8-byte load for an 8-bit column), so a warp's
// loads cover whole sectors, there is no staging copy or handshake, and a row costs a few
// instructions: the shipdate-and-key-bitmap scan of a 600M-row fact table reads at about
// the copy bandwidth of HBM. Survivors are appended to the hit list as positions, or, for
// an inline build, go straight to the build table (a hash insert, or a dense table's key
// bit and record); their key and payload values are read per survivor.
constexpr uint32_t kVecRows = kItems;  // consecutive rows per thread per tile
static_assert(kT * kVecRows == kTile, "a tile is one block of rows per thread");

// Stored values of rows row0 .. row0 + n - 1 (n <= 8) of a column of at most 32 bits; the
// full block reads 8 rows with vector loads (row0 is a multiple of 8, so the addresses
// are aligned when the column's base is), a segment's last partial block reads row by row.
__device__ __forceinline__ void load8_narrow(const void* p, uint32_t bits, uint32_t row0, uint32_t n,
                                             uint32_t (&x)[kVecRows]) {
  if (n == kVecRows) {
    if (bits == 8) {
      const uint2 v = __ldcs((const uint2*)((const uint8_t*)p + row0));
#pragma unroll
      for (int k = 0; k < 4; k++) {
        x[k] = (v.x >> (8 * k)) & 0xffu;
        x[4 + k] = (v.y >> (8 * k)) & 0xffu;
      }
    } else if (bits == 16) {
      const uint4 v = __ldcs((const uint4*)((const uint16_t*)p + row0));
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        x[2 * k] = w[k] & 0xffffu;
        x[2 * k + 1] = w[k] >> 16;
      }
    } else {
      const uint4* q = (const uint4*)((const uint32_t*)p + row0);
      const uint4 u = __ldcs(q), v = __ldcs(q + 1);
      x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w;
      x[4] = v.x, x[5] = v.y, x[6] = v.z, x[7] = v.w;
    }
    return;
  }
#pragma unroll
  for (uint32_t k = 0; k < kVecRows; k++) {
    x[k] = 0;
    if (k < n) {
      const uint32_t r = row0 + k;
      x[k] = bits == 8 ? __ldg((const uint8_t*)p + r) : bits == 16 ? __ldg((const uint16_t*)p + r)
                                                                   : __ldg((const uint32_t*)p + r);
    }
  }
}

// Hint to the copy engine: bring [p, p + bytes) into L2 (p 16-byte aligned, bytes a
// multiple of 16; no register or completion is involved).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
// The part of a column's rows [r0, r0 + nr) that starts and ends on 16-byte boundaries
// inside the rows, prefetched into L2.
__device__ __forceinline__ void prefetch_rows(const alk_colseg& d, uint32_t r0, uint32_t nr) {
  const uint32_t w = d.bits / 8;
  const uintptr_t b = (uintptr_t)d.data + (uintptr_t)r0 * w;
  const uintptr_t e = (uintptr_t)d.data + (uintptr_t)(r0 + nr) * w;
  const uintptr_t b16 = (b + 15) & ~(uintptr_t)15, e16 = e & ~(uintptr_t)15;
  if (e16 > b16) prefetch_l2((const void*)b16, (uint32_t)(e16 - b16));
}

// Resident blocks of 256 threads per SM that each form of k_stage_vec is compiled for
// (at most 65536 / (256 x blocks) registers a thread), the most that compile without
// spills. The loop is latency-bound: with one conjunct, 8 blocks at 32 registers against
// 6 at 40 took the 600M-row query from 2.12 to 2.09 ms; left to itself the compiler gave
// the forms with more conjuncts 76-110 registers (2-3 blocks).
constexpr int vec_min_blocks(int mode, int conj) {
  return mode == 2 ? (conj <= 2 ? 4 : 3) : conj <= 1 ? 8 : conj == 2 ? 5 : 4;
}

// kMode: 0 survivors to the hit list, 1 inline dense build (records), 2 inline hash build,
// 3 inline dense build of a table that stores no keys (bits only).
// kConj: the predicate's conjuncts. A block's tiles advance by gridDim.x, so each thread
// follows its segment incrementally and keeps the segment's column descriptors, conjunct
// tests and probe plan in registers (no per-tile table lookups).
template <int kMode, int kConj>
__global__ void __launch_bounds__(kT, vec_min_blocks(kMode, kConj)) k_stage_vec(const __grid_constant__ TmaArgs t) {
  const FastArgs& f = t.f;
  const StageArgs& a = f.a;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  // the per-segment tables of k_stage_tma's layout, with no stage buffers in front
  uint32_t* s_tile = (uint32_t*)(s_dyn + tma_tile_table_off(0, 0));
  alk_colseg* s_cd = (alk_colseg*)(s_dyn + tma_desc_off(0, 0, a.nseg));  // [nstaged][nseg]
  ConjSeg* s_cs = (ConjSeg*)(s_dyn + tma_cseg_off(0, 0, a.nseg, t.nstaged));  // [nconj][nseg]
  SegPlan* s_sp = (SegPlan*)(s_dyn + tma_splan_off(0, 0, a.nseg, t.nstaged, f.nconj));  // [nseg]
  for (uint32_t i = threadIdx.x; i <= a.nseg; i += kT) s_tile[i] = a.seg_tile[i];
  for (uint32_t i = threadIdx.x; i < t.nstaged * a.nseg; i += kT)
    s_cd[i] = a.cols[t.staged_slot[i / a.nseg] * a.nseg + i % a.nseg];
  for (uint32_t i = threadIdx.x; i < f.nconj * a.nseg; i += kT) s_cs[i] = f.cseg[i];
  for (uint32_t i = threadIdx.x; i < a.nseg; i += kT) s_sp[i] = f.splan[i];
  __syncthreads();
  // per warp: its survivors' rows within the tile (inline builds), so that the warp then
  // handles them 32 at a time, one per lane, whatever lanes they came from
  __shared__ uint16_t s_rows[kMode == 0 ? 1 : kT * kVecRows];
  unsigned long long rows_seen = 0, inserted = 0, survivors = 0;
  HitWriter hw;
  const uint32_t lane = threadIdx.x & 31;
  const bool probe = t.probe_st >= 0 && a.probe.bits;
  // the current segment, in registers
  uint32_t seg = 0, seg_end = 0, tile0 = 0, nrows = 0;
  const void* cdata[kConj > 0 ? kConj : 1];
  uint32_t cbits[kConj > 0 ? kConj : 1];
  int64_t clower[kConj > 0 ? kConj : 1];
  ConjSeg ccs[kConj > 0 ? kConj : 1];
  const void* pdata = nullptr;
  uint32_t pbits = 0;
  SegPlan sp{};
  bool first = true;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    if (first || tile >= seg_end) {
      if (first) seg = tile_segment(s_tile, a.nseg, tile);
      while (tile >= s_tile[seg + 1]) seg++;
      first = false;
      tile0 = s_tile[seg];
      seg_end = s_tile[seg + 1];
#pragma unroll
      for (int c = 0; c < kConj; c++) {
        const alk_colseg& d = s_cd[t.conj_st[c] * a.nseg + seg];
        cdata[c] = d.data;
        cbits[c] = d.bits;
        clower[c] = d.lower;
        ccs[c] = s_cs[c * a.nseg + seg];
      }
      nrows = s_cd[seg].rows;
      if (probe) {
        const alk_colseg& d = s_cd[t.probe_st * a.nseg + seg];
        pdata = d.data;
        pbits = d.bits;
        sp = s_sp[seg];
      }
    }
    // the columns every row reads, for this block's next tile: into L2 while this tile
    // is worked on, so that their loads meet L2 latency rather than DRAM's
    if (threadIdx.x == 0 && tile + gridDim.x < a.ntiles && (kConj > 0 || probe)) {
      const uint32_t nt = tile + gridDim.x;
      uint32_t sg = seg;
      while (nt >= s_tile[sg + 1]) sg++;
      const uint32_t r0 = (nt - s_tile[sg]) * kTile;
      const uint32_t nr = min(kTile, s_cd[sg].rows - r0);
#pragma unroll
      for (int c = 0; c < kConj; c++) prefetch_rows(s_cd[t.conj_st[c] * a.nseg + sg], r0, nr);
      if (probe) prefetch_rows(s_cd[t.probe_st * a.nseg + sg], r0, nr);
    }
    const uint32_t row0 = (tile - tile0) * kTile + threadIdx.x * kVecRows;
    const uint32_t n = row0 < nrows ? min(kVecRows, nrows - row0) : 0u;
    uint32_t live = (1u << n) - 1u;
    rows_seen += n;
    uint32_t x[kVecRows];
#pragma unroll
    for (int c = 0; c < kConj; c++) {
      if (live) {
        load8_narrow(cdata[c], cbits[c], row0, n, x);
        live = conj_filter32(f.conj[c], ccs[c], clower[c], x, live);
      }
    }
    if (live && probe) {
      load8_narrow(pdata, pbits, row0, n, x);
      live = probe_filter32(a.probe, sp, x, live);
    }
    if (kMode == 0) {
      hw.append_blocked(a, live, seg, row0);
      continue;
    }
    // inline build: the warp's survivors are listed, then handled one per lane; key and
    // payload are read at each survivor's row
    uint32_t excl;
    const uint32_t total = __any_sync(0xffffffffu, live) ? warp_offsets(__popc(live), &excl) : 0;
    if (!total) continue;
    uint16_t* wl = s_rows + (threadIdx.x & ~31u) * kVecRows;
    {
      uint32_t q = excl;
      for (uint32_t m = live; m; m &= m - 1, q++) wl[q] = (uint16_t)(threadIdx.x * kVecRows + (__ffs(m) - 1));
    }
    __syncwarp();
    const uint32_t tile_row0 = (tile - tile0) * kTile;
    const alk_colseg& kd = s_cd[t.key_st * a.nseg + seg];
    if (kMode == 3) {
      // dense table without stored keys: the key's bit; a bit found set already is a
      // duplicate key, a new one counts as an inserted key
      for (uint32_t j = lane; j < total; j += 32) {
        const uint32_t r = tile_row0 + wl[j];
        const int64_t key = load_for(kd.data, kd.bits, kd.lower, r);
        const uint64_t o = (uint64_t)key - (uint64_t)a.build.kmin;
        if (o >= a.build.nbits) {
          atomicExch(a.build.flags + 3, 1);
          continue;
        }
        const uint32_t bit = 1u << (o & 31);
        if (atomicOr(a.build.bits + (o >> 5), bit) & bit) atomicExch(a.build.flags, 1);
        else inserted++;
      }
    } else if (kMode == 1) {
      // dense table: the key's bit, and the record [position, key, payload...]
      const HitWriter::Room room = hw.reserve(a, total);
      for (uint32_t j = lane; j < total; j += 32) {
        const uint32_t r = tile_row0 + wl[j];
        const int64_t key = load_for(kd.data, kd.bits, kd.lower, r);
        const uint64_t o = (uint64_t)key - (uint64_t)a.build.kmin;
        if (o < a.build.nbits) atomicOr(a.build.bits + (o >> 5), 1u << (o & 31));
        else atomicExch(a.build.flags + 3, 1);
        const uint64_t e = room.at(j);
        if (e >= a.hit_cap) continue;
        Hit* rec = a.hits + e * a.hit_words;
        rec[0] = (uint64_t)seg << 32 | (uint64_t)r;
        rec[1] = (uint64_t)key;
#pragma unroll
        for (uint32_t p = 0; p < 8; p++)
          if (p < a.build.npay) {
            const alk_colseg& pd = s_cd[t.pay_st[p] * a.nseg + seg];
            rec[2 + p] = (uint64_t)load_for(pd.data, pd.bits, pd.lower, r);
          }
      }
    } else {
      // hash table: insert, then the payload at the key's position
      if (lane == 0) survivors += total;
      for (uint32_t j = lane; j < total; j += 32) {
        const uint32_t r = tile_row0 + wl[j];
        const int64_t key = load_for(kd.data, kd.bits, kd.lower, r);
        int64_t pv[8];
#pragma unroll
        for (uint32_t p = 0; p < 8; p++)
          if (p < a.build.npay) {
            const alk_colseg& pd = s_cd[t.pay_st[p] * a.nseg + seg];
            pv[p] = load_for(pd.data, pd.bits, pd.lower, r);
          }
        const int64_t sl = ht_insert(a.build, key);
        if (sl < 0) continue;
        inserted++;
#pragma unroll
        for (uint32_t p = 0; p < 8; p++)
          if (p < a.build.npay) a.build.payload[(uint64_t)p * a.build.slot_cap + sl] = pv[p];
      }
    }
    __syncwarp();  // the list is rewritten by the warp's next tile
  }
  hw.finish(a);
  for (int o = 16; o; o >>= 1) {
    rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
    inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
    survivors += __shfl_xor_sync(0xffffffffu, survivors, o);
  }
  if (lane == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
  if (lane == 0 && inserted) atomicAdd(a.build.nslots, inserted);
  if (lane == 0 && survivors) atomicAdd(a.hit_rows, survivors);
}

// The blocked kernel for a mode and conjunct count (0 .. kMaxConj).
template <int kMode>
using VecKernel = void (*)(const TmaArgs);
template <int kMode>
VecKernel<kMode> vec_kernel_for(uint32_t nconj) {
  switch (nconj) {
    case 0: return k_stage_vec<kMode, 0>;
    case 1: return k_stage_vec<kMode, 1>;
    case 2: return k_stage_vec<kMode, 2>;
    case 3: return k_stage_vec<kMode, 3>;
    default: return k_stage_vec<kMode, 4>;
  }
}
static_assert(kMaxConj == 4, "one blocked kernel per conjunct count");

// Host: recognise an AND of (column * mul OP constant) tests in a compiled predicate.
bool as_conjuncts(const alk_program& p, Conj* out, uint32_t* n) {
  *n = 0;
  if (p.n_instr == 0) return true;
  struct R {
    int kind = 0;  // 0 unknown, 1 scaled column, 2 conjunct list
    uint32_t slot = 0;
    int64_t mul = 1;
    std::vector<Conj> cj;
  } r[ALK_MAX_REGS];
  struct Opd {
    int kind;  // 0 unknown, 1 scaled column, 2 conjuncts, 3 constant
    uint32_t slot;
    int64_t mul, c;
    const std::vector<Conj>* cj;
  };
  auto opd = [&](uint8_t k, uint16_t x) -> Opd {
    if (k == ALK_K_COL) return {x < 32 ? 1 : 0, x, 1, 0, nullptr};
    if (k == ALK_K_CONST) return {3, 0, 1, p.consts[x], nullptr};
    const R& q = r[x];
    return {q.kind, q.slot, q.mul, 0, &q.cj};
  };
  auto mirror = [](uint8_t op) -> uint8_t {
    switch (op) {
      case ALK_OP_LT: return ALK_OP_GT;
      case ALK_OP_GT: return ALK_OP_LT;
      case ALK_OP_LE: return ALK_OP_GE;
      case ALK_OP_GE: return ALK_OP_LE;
      default: return op;
    }
  };
  for (uint32_t i = 0; i < p.n_instr; i++) {
    const alk_instr& in = p.ins[i];
    Opd x = opd(in.ka, in.a), y = opd(in.kb, in.b);
    R res;
    if (in.op == ALK_OP_MUL && ((x.kind == 1 && y.kind == 3) || (x.kind == 3 && y.kind == 1))) {
      const Opd& c = x.kind == 1 ? x : y;
      const Opd& k = x.kind == 3 ? x : y;
      res.kind = 1;
      res.slot = c.slot;
      res.mul = (int64_t)((uint64_t)c.mul * (uint64_t)k.c);
    } else if (in.op >= ALK_OP_LT && in.op <= ALK_OP_NE && x.kind == 1 && y.kind == 3) {
      res.kind = 2;
      res.cj.push_back({x.mul, y.c, x.slot, in.op});
    } else if (in.op >= ALK_OP_LT && in.op <= ALK_OP_NE && x.kind == 3 && y.kind == 1) {
      res.kind = 2;
      res.cj.push_back({y.mul, x.c, y.slot, mirror(in.op)});
    } else if (in.op == ALK_OP_AND && x.kind == 2 && y.kind == 2) {
      res.kind = 2;
      res.cj = *x.cj;
      res.cj.insert(res.cj.end(), y.cj->begin(), y.cj->end());
    } else if (in.op == ALK_OP_MOV && (x.kind == 1 || x.kind == 2)) {
      res.kind = x.kind;
      res.slot = x.slot;
      res.mul = x.mul;
      if (x.cj) res.cj = *x.cj;
    } else {
      return false;
    }
    r[in.dst] = res;
  }
  const R& fin = r[p.result];
  if (fin.kind != 2 || fin.cj.size() > (size_t)kMaxConj) return false;
  for (size_t i = 0; i < fin.cj.size(); i++) out[i] = fin.cj[i];
  *n = (uint32_t)fin.cj.size();
  return true;
}

int grid_for(uint64_t n) {
  uint64_t b = (n + kT - 1) / kT;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sms() * 8));
}

// Static shared memory of k_stage_tma (barriers) next to its dynamic stage buffers and
// tables; the SM offers 227 KB per block.
constexpr size_t kTmaStaticSmem = 6 * 1024;
constexpr size_t kSmemPerBlock = 227 * 1024;
constexpr size_t kSmemPerSM = 228 * 1024;

// Launch a stage as two kernels on one stream: the scan (the TMA-staged kernel when the
// predicate is a conjunction and the staged columns fit in shared memory, else the
// conjunctive kernel with direct loads, else the register-machine kernel), then the hit
// kernel over its survivors. cols is the host descriptor array [ncols][nseg]; fa holds
// the device arguments and, when conj, the predicate's conjuncts.
template <bool kBuild>
cudaError_t launch_stage(FastArgs fa, bool conj, bool narrow_all, const alk_colseg* cols, const uint8_t* seg_mode,
                         const int32_t* h_pay_src, cudaStream_t s, alk_event_timer* timer) {
  StageArgs& a = fa.a;
  if (!a.ntiles) return cudaSuccess;
  TmaArgs t{};
  bool tma = false, vec = false;
  uint32_t tma_smem = 0, vec_smem = 0;
  // The columns every row needs (conjunct columns and the probe key) and, for an inline
  // build, the key and payload: their descriptors go to shared memory.
  std::vector<uint32_t> st;
  auto plan_cols = [&](bool with_build) -> bool {
    t = TmaArgs{};
    t.f = fa;
    st.clear();
    auto add = [&](uint32_t sl) -> uint32_t {
      auto it = std::find(st.begin(), st.end(), sl);
      if (it != st.end()) return (uint32_t)(it - st.begin());
      st.push_back(sl);
      return (uint32_t)st.size() - 1;
    };
    for (uint32_t c = 0; c < fa.nconj; c++) t.conj_st[c] = add(fa.conj[c].slot);
    t.probe_st = a.probe_slot >= 0 ? (int32_t)add((uint32_t)a.probe_slot) : -1;
    if (with_build) {
      t.inline_build = 1;
      t.key_st = add((uint32_t)a.build_slot);
      for (uint32_t p = 0; p < a.build.npay; p++) t.pay_st[p] = add((uint32_t)h_pay_src[p]);
    }
    if (st.empty() || st.size() > (size_t)kStaged) return false;
    for (size_t i = 0; i < st.size(); i++) t.staged_slot[i] = st[i];
    t.nstaged = (uint32_t)st.size();
    return true;
  };
  // Blocked vector loads: every scanned segment narrow, and the columns read for every
  // row aligned for 16-byte (8-bit columns: 8-byte) loads.
  auto plan_vec = [&](bool with_build) -> bool {
    if (!plan_cols(with_build)) return false;
    std::vector<uint32_t> tested;
    for (uint32_t c = 0; c < fa.nconj; c++) tested.push_back(t.conj_st[c]);
    if (t.probe_st >= 0 && a.probe.bits) tested.push_back((uint32_t)t.probe_st);
    for (uint32_t i : tested)
      for (uint32_t g = 0; g < a.nseg; g++) {
        if (!seg_mode[g]) continue;
        const alk_colseg& d = cols[st[i] * a.nseg + g];
        if (d.bits > 32 || ((uintptr_t)d.data & (d.bits == 8 ? 7u : 15u))) return false;
      }
    vec_smem = tma_smem_bytes(0, 0, a.nseg, t.nstaged, fa.nconj);
    return vec_smem + kTmaStaticSmem <= kSmemPerBlock;
  };
  // Staged tiles, with as many tiles in flight as keep 3 blocks per SM (2 at least).
  auto plan = [&](bool with_build) -> bool {
    if (!plan_cols(with_build)) return false;
    // bulk copies need 16-byte aligned sources (row0 * width is a multiple of kTile)
    uint32_t bytes = 0;
    for (size_t i = 0; i < st.size(); i++) {
      uint32_t w = 1;
      for (uint32_t g = 0; g < a.nseg; g++) {
        if (!seg_mode[g]) continue;
        const alk_colseg& d = cols[st[i] * a.nseg + g];
        w = std::max<uint32_t>(w, d.bits / 8);
        if ((uintptr_t)d.data & 15) return false;
      }
      t.col_off[i] = bytes;
      bytes += (kTile * w + 127) & ~127u;
    }
    t.stage_bytes = bytes;
    for (t.nst = kMaxStages; t.nst >= 2; t.nst--) {
      const size_t need = kTmaStaticSmem + tma_smem_bytes(bytes, t.nst, a.nseg, t.nstaged, fa.nconj);
      const bool three_fit = 3 * (need + 1024) <= kSmemPerSM;  // 1 KB per block is reserved
      if (need <= kSmemPerBlock && (three_fit || t.nst == 2)) {
        tma_smem = tma_smem_bytes(bytes, t.nst, a.nseg, t.nstaged, fa.nconj);
        return true;
      }
    }
    return false;
  };
  if (conj) {
    // an inline build needs every payload value from the scan and the probe (if any)
    // settled by the exact key bitmap
    const bool can_inline = kBuild && h_pay_src && !a.need_slot && (a.probe_slot < 0 || a.probe.bits);
    if (narrow_all) vec = (can_inline && plan_vec(true)) || plan_vec(false);
    // the staged kernel's inline dense build writes records: tables that store no keys
    // take the survivor list and the bit-marking pass instead
    const bool tma_inline = can_inline && !(a.build.rank && a.build.dense_mode);
    if (!vec) tma = (tma_inline && plan(true)) || plan(false);
  }
  const bool inline_build = (tma || vec) && t.inline_build;
  const bool dense = kBuild && a.build.rank != nullptr;
  // a dense build staged inline records [position, key, payload] per survivor
  a.hit_words = dense && inline_build && !a.build.dense_mode ? 2 + a.build.npay : 1;
  t.f.a.hit_words = a.hit_words;
  int occ = 0;
  // the blocked kernel's mode: hit list, inline builds
  void (*vec_kernel)(const TmaArgs) = !inline_build               ? vec_kernel_for<0>(fa.nconj)
                                      : dense && a.build.dense_mode ? vec_kernel_for<3>(fa.nconj)
                                      : dense                       ? vec_kernel_for<1>(fa.nconj)
                                                                    : vec_kernel_for<2>(fa.nconj);
  if (vec) {
    cudaFuncSetAttribute(vec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, vec_smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, vec_kernel, kT, vec_smem);
  } else if (tma) {
    cudaFuncSetAttribute(k_stage_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem);
    cudaFuncSetAttribute(k_stage_tma, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_tma, kTmaThreads, tma_smem);
  } else if (conj) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_fast, kT, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_scan, kT, 0);
  }
  // at most 8 blocks per SM of 8 appending warps each: the hit list's chunk slack assumes it
  const int grid = std::min<int>((int)a.ntiles, sms() * std::min(std::max(occ, 1), 8));
  int occ_hits = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_hits, k_stage_hits<kBuild>, kT, 0);
  // inside a stream capture the timing events become event-record nodes of the graph
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  if (timer && timer->on) cudaStreamIsCapturing(s, &cst);
  const unsigned evflags = cst == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  if (timer && timer->on) cudaEventRecordWithFlags((cudaEvent_t)timer->ev0, s, evflags);
  if (vec) vec_kernel<<<grid, kT, vec_smem, s>>>(t);
  else if (tma) k_stage_tma<<<grid, kTmaThreads, tma_smem, s>>>(t);
  else if (conj) k_stage_fast<<<grid, kT, 0, s>>>(fa);
  else k_stage_scan<<<grid, kT, 0, s>>>(a);
  uint32_t launches = 1;
  const int hits_grid = sms() * std::max(occ_hits, 1);
  if (dense) {
    // dense build: key bits (from positions, when the scan did not set them), the rank
    // prefix (unless the table is membership only), then the scatter of keys and payload
    // to their ranks (only for a table that stores them)
    if (!inline_build) {
      k_rank_mark<<<hits_grid, kT, 0, s>>>(a);
      launches++;
    }
    if (a.build.dense_mode != 2) {
      k_rank_sums<<<a.rk_tiles, kT, 0, s>>>(a);
      k_rank_scan_sums<<<1, kRankScanThreads, 0, s>>>(a);
      k_rank_write<<<a.rk_tiles, kT, 0, s>>>(a);
      launches += 3;
    }
    if (a.build.dense_mode == 0) {
      k_stage_hits<kBuild><<<hits_grid, kT, 0, s>>>(a);
      launches++;
    }
  } else if (!inline_build) {
    k_stage_hits<kBuild><<<hits_grid, kT, 0, s>>>(a);
    launches++;
  }
  if (timer && timer->on) cudaEventRecordWithFlags((cudaEvent_t)timer->ev1, s, evflags);
  alk::g_kernel_launches += launches;
  return cudaGetLastError();
}

// Late payload of a ranks-only dense table (keys and payload fetched for a few candidate
// slots after the aggregation, instead of stored for every key during the build).
struct LateArgs {
  HtView h;
  const uint32_t* cand;             // candidate slots
  const unsigned long long* count;  // their number (device)
  uint32_t cap;                     // at most this many are handled
  uint32_t nseg, npay;
  const alk_colseg* cols;   // [1 + npay][nseg]: the key column (ascending), then payload
  const int64_t* seg_lo;    // [nseg] zone bounds of the key column
  const int64_t* seg_hi;
  const uint8_t* seg_mode;  // [nseg] segments the build stage scanned
  int64_t* const* out;      // [1 + npay] slot-indexed columns: key, payload
  int* status;              // set: a candidate matched no row or more than one
};

// First index in [lo, hi) whose value is >= key (hi if none), for values nondecreasing
// in the index; 32-ary: each round the warp tests 32 pivots, so a range of n values takes
// ceil(log32 n) dependent loads instead of log2 n. Called by all 32 lanes.
template <class F>
__device__ __forceinline__ uint64_t warp_lower_bound(uint64_t lo, uint64_t hi, int64_t key, F value) {
  const uint32_t lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + lane * step;
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, p < hi && value(p) < key));
    if (c == 0) return lo;
    // the answer lies after pivot c - 1 and at or before pivot c (or hi)
    const uint64_t nlo = lo + (uint64_t)(c - 1) * step + 1;
    hi = min(hi, lo + (uint64_t)c * step);
    lo = nlo;
  }
  return lo + __popc(__ballot_sync(0xffffffffu, lo + lane < hi && value(lo + lane) < key));
}

// One warp per candidate: its key from the rank prefix (the last bitmap word whose rank
// is <= slot, then the (slot - rank)-th set bit), then the key's rows by binary search
// in each scanned segment whose zone holds the key. Exactly one row: its payload is the
// candidate's; none or several: status.
__global__ void __launch_bounds__(kT) k_late_rows(const LateArgs a) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = (uint32_t)min((unsigned long long)a.cap, *(volatile const unsigned long long*)a.count);
  const uint64_t nkeys = *(volatile const unsigned long long*)a.h.nslots;
  const uint64_t nwords = (a.h.nbits + 31) / 32;
  const uint32_t warps = gridDim.x * (kT / 32);
  for (uint32_t i = blockIdx.x * (kT / 32) + (threadIdx.x >> 5); i < n; i += warps) {
    const uint32_t slot = a.cand[i];
    if (slot >= nkeys || slot >= a.h.slot_cap) {
      if (lane == 0) atomicExch(a.status, 1);
      continue;
    }
    const uint64_t w =
        warp_lower_bound(0, nwords, (int64_t)slot + 1, [&](uint64_t x) { return (int64_t)a.h.rank[x]; }) - 1;
    uint32_t m = a.h.bits[w];
    for (uint32_t r = slot - a.h.rank[w]; r && m; r--) m &= m - 1;
    if (!m) {  // the rank prefix and the bitmap disagree
      if (lane == 0) atomicExch(a.status, 1);
      continue;
    }
    const int64_t key = (int64_t)((uint64_t)a.h.kmin + w * 32 + (uint64_t)(__ffs(m) - 1));
    if (lane == 0) a.out[0][slot] = key;
    uint32_t found = 0, fg = 0;
    uint64_t frow = 0;
    for (uint32_t g0 = 0; g0 < a.nseg && found < 2; g0 += 32) {
      const uint32_t g = g0 + lane;
      uint32_t hit = __ballot_sync(0xffffffffu, g < a.nseg && a.seg_mode[g] && key >= a.seg_lo[g] &&
                                                    key <= a.seg_hi[g]);
      for (; hit && found < 2; hit &= hit - 1) {
        const uint32_t sg = g0 + __ffs(hit) - 1;
        const alk_colseg kd = a.cols[sg];
        auto v = [&](uint64_t x) { return load_for(kd.data, kd.bits, kd.lower, x); };
        const uint64_t lb = warp_lower_bound(0, kd.rows, key, v);
        uint32_t c = 0;
        if (lb < kd.rows && v(lb) == key) c = (lb + 1 < kd.rows && v(lb + 1) == key) ? 2 : 1;
        if (c && !found) {
          fg = sg;
          frow = lb;
        }
        found += c;
      }
    }
    if (lane != 0) continue;
    if (found != 1) {
      atomicExch(a.status, 1);
      continue;
    }
    for (uint32_t p = 0; p < a.npay; p++) {
      const alk_colseg& pd = a.cols[(uint64_t)(1 + p) * a.nseg + fg];
      a.out[1 + p][slot] = load_for(pd.data, pd.bits, pd.lower, frow);
    }
  }
}

// Per segment: 1 when a row's value is below its predecessor's.
__global__ void __launch_bounds__(kT) k_seg_unsorted(const alk_colseg* segs, uint32_t* flags) {
  const uint32_t g = blockIdx.y;
  const alk_colseg d = segs[g];
  int bad = 0;
  for (uint64_t r = 1 + blockIdx.x * (uint64_t)kT + threadIdx.x; r < d.rows && !bad; r += (uint64_t)gridDim.x * kT)
    bad = load_for(d.data, d.bits, d.lower, r) < load_for(d.data, d.bits, d.lower, r - 1);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags + g, 1u);
}

// ---- Fused filter + hash GROUP BY over resident segments (emit_select's group-by,
// select.cu:359-952, with the filter of filter.cu:133-643 in the same pass): each row's
// predicate, group keys and aggregate inputs are read at their stored widths, the group's
// slot is found or claimed in an open-addressing table, and lanes of a warp that land on
// the same slot fold their values before one atomic per aggregate.
struct GroupTable {
  uint64_t cap;            // power of two (hash forms); the key space's size (direct form)
  // One record of rw words per slot: the key columns (hash forms; one key: kEmptyKey
  // marks a free slot), then the accumulators. A group's key and accumulators share a
  // record, so its random updates touch one 32-byte sector when rw <= 4.
  int64_t* rec;
  uint32_t rw, kw;         // words per record; key words in front (0 in the direct form)
  uint32_t* state;         // several keys: 0 free, 1 being written, 2 full
  // direct form: slot = sum over j of (key_j - kmin_j) * kstride_j, a slot's presence a bit
  int64_t kmin[4];
  uint64_t kspan[4], kstride[4];
  uint32_t* occ;
  uint32_t nkeys;
  int32_t key_slot[4];
  int generic;             // the predicate is not a conjunction: run it per row
  unsigned long long* seg_rows;  // [nseg] surviving rows per segment
  unsigned long long* groups;    // groups written by the compaction
  int64_t* const* out_keys;      // [nkeys] compacted keys (device array of addresses)
  int64_t* const* out_vals;      // [nagg]
  uint64_t out_cap;
};

// One conjunct on one stored value x (value = x + lower).
__device__ __forceinline__ bool conj_pass(const Conj& cj, const ConjSeg& cs, int64_t lower, uint64_t x) {
  switch (cs.mode) {
    case kCjAlways: return true;
    case kCjNever: return false;
    case kCjIn: return x - cs.lo <= cs.span;
    case kCjOut: return x - cs.lo > cs.span;
    default: {
      const int64_t v = wrap_mul((int64_t)(x + (uint64_t)lower), cj.mul);
      switch (cj.op) {
        case ALK_OP_LT: return v < cj.k;
        case ALK_OP_GT: return v > cj.k;
        case ALK_OP_LE: return v <= cj.k;
        case ALK_OP_GE: return v >= cj.k;
        case ALK_OP_EQ: return v == cj.k;
        default: return v != cj.k;
      }
    }
  }
}

// Slot of a one-column group key: found, or claimed with one compare-and-swap on the key
// word. -1 when the table is full or the key is the free-slot marker (err set).
__device__ __forceinline__ int64_t group_slot1(const GroupTable& g, int64_t key, int* err) {
  if (key == kEmptyKey) {
    atomicExch(err, ALK_ERR_UNSUPPORTED);
    return -1;
  }
  const uint64_t mask = g.cap - 1;
  uint64_t p = murmur_u64((uint64_t)key) & mask;
  for (uint64_t n = 0; n <= mask; n++) {
    const int64_t v = __ldcg(g.rec + p * g.rw);  // keys only go from free to set
    if (v == key) return (int64_t)p;
    if (v == kEmptyKey) {
      const int64_t old = (int64_t)atomicCAS((unsigned long long*)(g.rec + p * g.rw), (unsigned long long)kEmptyKey,
                                             (unsigned long long)key);
      if (old == kEmptyKey || old == key) return (int64_t)p;
    }
    p = (p + 1) & mask;
  }
  atomicCAS(err, 0, ALK_ERR_OVERFLOW);
  return -1;
}

// Slot of a multi-column group key: a slot's state goes 0 -> 1 (claimed) -> 2 (keys
// written); a reader that meets 1 waits, with a bound.
__device__ __forceinline__ int64_t group_slot(const GroupTable& g, const int64_t (&key)[4], int* err) {
  const uint64_t mask = g.cap - 1;
  uint64_t h = kSeed ^ ((uint64_t)(8 * g.nkeys) * kMurmurM);
#pragma unroll
  for (int j = 0; j < 4; j++)
    if (j < (int)g.nkeys) h = mm_block(h, (uint64_t)key[j]);
  uint64_t p = mm_final(h) & mask;
  uint32_t spins = 0;
  for (uint64_t n = 0; n <= mask;) {
    const uint32_t st = *((volatile uint32_t*)g.state + p);
    if (st == 0) {
      if (atomicCAS(g.state + p, 0u, 1u) == 0u) {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (j < (int)g.nkeys) g.rec[p * g.rw + j] = key[j];
        __threadfence();
        atomicExch(g.state + p, 2u);
        return (int64_t)p;
      }
      continue;  // claimed meanwhile: look again
    }
    if (st == 1) {
      if (++spins > kSpinLimit) {
        atomicExch(err, ALK_ERR_TIMEOUT);
        return -1;
      }
      continue;
    }
    __threadfence();
    bool eq = true;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (j < (int)g.nkeys && __ldcg(g.rec + p * g.rw + j) != key[j]) eq = false;
    if (eq) return (int64_t)p;
    p = (p + 1) & mask;
    n++;
  }
  atomicCAS(err, 0, ALK_ERR_OVERFLOW);
  return -1;
}

// Slot of a group key in the direct form (keys within the zone maps' ranges); -1 with err
// set for a key outside them.
__device__ __forceinline__ int64_t group_slot_direct(const GroupTable& g, const int64_t (&key)[4], int* err) {
  uint64_t slot = 0;
#pragma unroll
  for (int j = 0; j < 4; j++)
    if (j < (int)g.nkeys) {
      const uint64_t o = (uint64_t)key[j] - (uint64_t)g.kmin[j];
      if (o >= g.kspan[j]) {
        atomicExch(err, ALK_ERR_UNSUPPORTED);
        return -1;
      }
      slot += o * g.kstride[j];
    }
  return (int64_t)slot;
}

// Position of the n-th (from 0) set bit of m; 32 when m has fewer.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t n) {
  for (uint32_t i = 0; i < n && m; i++) m &= m - 1;
  return m ? (uint32_t)__ffs(m) - 1 : 32u;
}

// Reduction of v over the lanes of `peers` (this lane's group, from __match_any_sync),
// delivered to the group's lowest lane: a tree over the group's ranks. Warp-wide.
__device__ __forceinline__ int64_t peer_reduce(int64_t v, uint32_t peers, uint8_t kind) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t rank = __popc(peers & ((1u << lane) - 1u)), cnt = __popc(peers);
  for (uint32_t s = 1; s < 32; s <<= 1) {
    if (!__any_sync(0xffffffffu, cnt > s)) break;
    const bool take = (rank & (2 * s - 1)) == 0 && rank + s < cnt;
    const uint32_t src = take ? nth_set_bit(peers, rank + s) : lane;
    const int64_t o = __shfl_sync(0xffffffffu, v, src);
    if (take) v = kind == ALK_AGG_MIN ? min(v, o) : kind == ALK_AGG_MAX ? max(v, o) : v + o;
  }
  return v;
}

// kForm: 0 hash table on one key column, 1 hash table on several, 2 direct (the key
// space, from the zone maps, indexes the accumulators).
template <int kForm>
__global__ void __launch_bounds__(kT, 6) k_group_scan(const __grid_constant__ FastArgs f,
                                                   const __grid_constant__ GroupTable g) {
  const StageArgs& a = f.a;
  __shared__ alk_instr s_ins[8][ALK_MAX_INSTR];
  __shared__ int64_t s_consts[8][ALK_MAX_CONST];
  __shared__ uint32_t s_n[8], s_res[8];
  __shared__ uint8_t s_kind[8];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  for (uint32_t p = 0; p < a.nprogs; p++) {
    for (uint32_t i = threadIdx.x; i < a.progs[p].n_instr; i += kT) s_ins[p][i] = a.progs[p].ins[i];
    for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[p][i] = a.progs[p].consts[i];
    if (threadIdx.x == 0) {
      s_n[p] = a.progs[p].n_instr;
      s_res[p] = a.progs[p].result;
      s_kind[p] = p ? a.agg_kind[p - 1] : 0;
    }
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  unsigned long long rows_seen = 0;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const uint32_t seg = tile_segment(a.seg_tile, a.nseg, tile);
    const uint32_t rows = a.cols[seg].rows;
    const uint32_t row0 = (tile - a.seg_tile[seg]) * kTile;
    const bool test = a.seg_mode[seg] == 2;
    unsigned long long kept = 0;
    for (int k = 0; k < kItems; k++) {
      // rows strided by the block: a warp's lanes read consecutive rows
      const uint32_t r = row0 + k * kT + threadIdx.x;
      bool live = r < rows;
      rows_seen += live;
      auto col = [&](uint32_t sl) -> int64_t {
        const alk_colseg* d = a.cols + (uint64_t)sl * a.nseg + seg;
        const void* data = (const void*)__ldg((const unsigned long long*)&d->data);
        return load_for(data, __ldg(&d->bits), (int64_t)__ldg((const long long*)&d->lower), r);
      };
      if (live && test) {
        if (g.generic) {
          live = vm_eval<kT>(s_ins[0], s_n[0], s_res[0], s_consts[0], s_regs + threadIdx.x, col) != 0;
        } else {
          for (uint32_t c = 0; c < f.nconj && live; c++) {
            const Conj& cj = f.conj[c];
            const int64_t lower = (int64_t)__ldg((const long long*)&a.cols[(uint64_t)cj.slot * a.nseg + seg].lower);
            live = conj_pass(cj, f.cseg[c * a.nseg + seg], lower, (uint64_t)(col(cj.slot) - lower));
          }
        }
      }
      kept += __popc(__ballot_sync(0xffffffffu, live));
      int64_t slot = -1;
      if (live) {
        if (kForm == 0) {
          slot = group_slot1(g, col((uint32_t)g.key_slot[0]), a.err);
        } else {
          int64_t key[4] = {0, 0, 0, 0};
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (j < (int)g.nkeys) key[j] = col((uint32_t)g.key_slot[j]);
          slot = kForm == 1 ? group_slot(g, key, a.err) : group_slot_direct(g, key, a.err);
        }
      }
      const bool use = slot >= 0;
      // lanes on the same slot: fold their values, then the group's lowest lane applies them
      const uint32_t peers = __match_any_sync(0xffffffffu, use ? (unsigned long long)slot : ~0ull);
      const bool share = __any_sync(0xffffffffu, use && __popc(peers) > 1);
      const bool leader = use && (uint32_t)(__ffs(peers) - 1) == lane;
      if (kForm == 2) {
        // presence bits: the warp's groups in one word (keys in order put them side by
        // side) are or-ed together first, and one lane applies the word; a word already
        // showing every bit is left alone
        const uint64_t word = leader ? (uint64_t)slot >> 5 : ~0ull;
        const uint32_t wpeers = __match_any_sync(0xffffffffu, word);
        const uint32_t bits = __reduce_or_sync(wpeers, leader ? 1u << (slot & 31) : 0u);
        if (leader && (uint32_t)(__ffs(wpeers) - 1) == lane && (__ldcg(g.occ + word) & bits) != bits)
          atomicOr(g.occ + word, bits);
      }
      for (uint32_t v = 0; v < a.nagg; v++) {
        const uint8_t kind = s_kind[1 + v];
        int64_t x = kind == ALK_AGG_MIN ? INT64_MAX : kind == ALK_AGG_MAX ? INT64_MIN : 0;
        if (use)
          x = kind == ALK_AGG_COUNT
                  ? 1
                  : vm_eval<kT>(s_ins[1 + v], s_n[1 + v], s_res[1 + v], s_consts[1 + v], s_regs + threadIdx.x, col);
        if (share) x = peer_reduce(x, peers, kind);
        if (!leader) continue;
        unsigned long long* dst = (unsigned long long*)(g.rec + (uint64_t)slot * g.rw + g.kw + v);
        if (kind == ALK_AGG_SUM || kind == ALK_AGG_COUNT) atomicAdd(dst, (unsigned long long)x);
        else if (kind == ALK_AGG_MIN) atomicMin((long long*)dst, (long long)x);
        else atomicMax((long long*)dst, (long long)x);
      }
    }
    if (lane == 0 && kept) atomicAdd(g.seg_rows + seg, kept);
  }
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if (lane == 0 && rows_seen) atomicAdd(a.rows_in, rows_seen);
}

// Every record: free key words (kEmptyKey for the one-key table), accumulators at their
// kind's identity.
__global__ void __launch_bounds__(kT) k_group_init(const GroupTable g, uint32_t nagg, uint64_t kinds) {
  const uint64_t words = g.cap * g.rw;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < words; i += (uint64_t)gridDim.x * kT) {
    const uint32_t w = (uint32_t)(i % g.rw);
    int64_t v = 0;
    if (w < g.kw) v = kEmptyKey;
    else if (w - g.kw < nagg) {
      const uint8_t kind = (uint8_t)(kinds >> (8 * (w - g.kw)));
      v = kind == ALK_AGG_MIN ? INT64_MAX : kind == ALK_AGG_MAX ? INT64_MIN : 0;
    }
    g.rec[i] = v;
  }
}

// Direct form: present slots to the output columns, one presence word per thread; the keys
// are recovered from the slot.
__global__ void __launch_bounds__(kT) k_group_compact_direct(const GroupTable g, uint32_t nagg) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nwords = (g.cap + 31) / 32;
  for (uint64_t w0 = blockIdx.x * (uint64_t)kT + (threadIdx.x & ~31u); w0 < nwords; w0 += (uint64_t)gridDim.x * kT) {
    const uint64_t w = w0 + lane;
    uint32_t bits = w < nwords ? g.occ[w] : 0u;
    const uint32_t n = __popc(bits);
    uint32_t excl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, excl, o);
      if (lane >= (uint32_t)o) excl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, excl, 31);
    excl -= n;
    if (!total) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(g.groups, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 0);
    uint64_t pos = base + excl;
    for (; bits; bits &= bits - 1, pos++) {
      const uint64_t slot = w * 32 + (uint32_t)(__ffs(bits) - 1);
      if (pos >= g.out_cap) continue;
      for (uint32_t j = 0; j < g.nkeys; j++)
        g.out_keys[j][pos] = (int64_t)((uint64_t)g.kmin[j] + (slot / g.kstride[j]) % g.kspan[j]);
      for (uint32_t v = 0; v < nagg; v++) g.out_vals[v][pos] = g.rec[slot * g.rw + v];
    }
  }
}

// Occupied slots to the output columns (in slot order within a warp, warps in any order).
__global__ void __launch_bounds__(kT) k_group_compact(const GroupTable g, uint32_t nagg) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint64_t h0 = blockIdx.x * (uint64_t)kT + (threadIdx.x & ~31u); h0 < g.cap; h0 += (uint64_t)gridDim.x * kT) {
    const uint64_t h = h0 + lane;
    const bool full = h < g.cap && (g.state ? g.state[h] == 2 : g.rec[h * g.rw] != kEmptyKey);
    const uint32_t m = __ballot_sync(0xffffffffu, full);
    if (!m) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(g.groups, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (!full) continue;
    const uint64_t pos = base + __popc(m & ((1u << lane) - 1u));
    if (pos >= g.out_cap) continue;  // counted: the caller sees the total and sizes again
    for (uint32_t j = 0; j < g.nkeys; j++) g.out_keys[j][pos] = g.rec[h * g.rw + j];
    for (uint32_t v = 0; v < nagg; v++) g.out_vals[v][pos] = g.rec[h * g.rw + g.kw + v];
  }
}

bool prog_ok(const alk_program& p, uint32_t ncols, uint32_t npay) {
  if (p.n_instr > ALK_MAX_INSTR || p.result >= ALK_MAX_REGS) return false;
  for (uint32_t i = 0; i < p.n_instr; i++) {
    const alk_instr& in = p.ins[i];
    if (in.dst >= ALK_MAX_REGS || in.op < ALK_OP_ADD || in.op > ALK_OP_INSET) return false;
    if (in.op == ALK_OP_INSET && in.kb != ALK_K_CONST) return false;  // the set's address
    const uint8_t k[2] = {in.ka, in.kb};
    const uint16_t x[2] = {in.a, in.b};
    for (int j = 0; j < 2; j++) {
      if (k[j] == ALK_K_REG && x[j] >= ALK_MAX_REGS) return false;
      if (k[j] == ALK_K_COL && !((x[j] < ncols) || (x[j] >= 32 && x[j] < 32 + npay))) return false;
      if (k[j] == ALK_K_CONST && x[j] >= ALK_MAX_CONST) return false;
      if (k[j] > ALK_K_CONST) return false;
    }
  }
  return true;
}
}  // namespace

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

struct alk_ht {
  HtView v{};
  void* mem = nullptr;
  size_t bytes = 0;  // device bytes held
};

extern "C" {

int alk_ht_create_range(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, alk_ht** out,
                        alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out || npay > 8 || max_keys >= 0xffffffffull) return ALK_ERR_ARG;
  auto* h = new alk_ht();
  uint64_t cap = 1024;
  while (cap < 2 * max_keys) cap <<= 1;
  const uint64_t slot_cap = cap;  // payload is indexed by table position
  // exact key bitmap when the key range is below 2^32 values (at most 512 MB); bit
  // offsets then fit the 32-bit probe path
  uint64_t nbits = 0;
  if (key_max >= key_min) {
    uint64_t span = (uint64_t)key_max - (uint64_t)key_min + 1;
    if (span != 0 && span <= ALK_DENSE_MAX_SPAN) nbits = span;
  }
  // the empty marker must not be a possible key
  if (key_max >= key_min && kEmptyKey >= key_min && kEmptyKey <= key_max) {
    delete h;
    return ALK_ERR_UNSUPPORTED;
  }
  size_t words = (nbits + 31) / 32;
  size_t bytes = cap * 8 + slot_cap * 8 * npay + 64 + words * 4;
  cudaError_t e = cudaMallocAsync(&h->mem, bytes, s);
  if (e != cudaSuccess) {
    delete h;
    return alk::cuda_fail(e);
  }
  h->bytes = bytes;
  uint8_t* p = (uint8_t*)h->mem;
  h->v.cap = cap;
  h->v.key = (int64_t*)p;
  p += cap * 8;
  h->v.payload = (int64_t*)p;
  p += slot_cap * 8 * npay;
  h->v.nslots = (unsigned long long*)p;
  h->v.flags = (int*)(p + 8);
  h->v.slot_cap = slot_cap;
  h->v.npay = npay;
  CK(cudaMemsetAsync(h->v.key, 0x80, cap * 8, s));  // every key word = kEmptyKey
  CK(cudaMemsetAsync(p, 0, 64, s));
  if (nbits) {
    h->v.bits = (uint32_t*)(p + 64);
    h->v.kmin = key_min;
    h->v.nbits = nbits;
    CK(cudaMemsetAsync(h->v.bits, 0, words * 4, s));
  }
  *out = h;
  return ALK_OK;
}

int alk_ht_create_dense_mode(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, int mode,
                             alk_ht** out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out || npay > 8 || max_keys >= 0xffffffffull || key_max < key_min) return ALK_ERR_ARG;
  if (mode < ALK_DENSE_FULL || mode > ALK_DENSE_BITS || (mode != ALK_DENSE_FULL && npay)) return ALK_ERR_ARG;
  const uint64_t span = (uint64_t)key_max - (uint64_t)key_min + 1;
  if (span == 0 || span > ALK_DENSE_MAX_SPAN) return ALK_ERR_UNSUPPORTED;  // no exact bitmap
  const uint64_t cap = std::max<uint64_t>(max_keys, 1);  // slots are ranks: no spare room
  const size_t words = (span + 31) / 32;
  // keys and payload only for a table that stores them
  const size_t off_pay = mode == ALK_DENSE_FULL ? cap * 8 : 0;
  const size_t off_ctr = off_pay + (mode == ALK_DENSE_FULL ? cap * 8 * npay : 0);
  const size_t off_bits = (off_ctr + 64 + 15) & ~size_t(15);  // 16-byte aligned (vector loads)
  const size_t off_rank = off_bits + ((words * 4 + 15) & ~size_t(15));
  // a membership-only table keeps a one-word rank array: probes of it never ask for slots
  const size_t rank_bytes = mode == ALK_DENSE_BITS ? 16 : words * 4;
  auto* h = new alk_ht();
  cudaError_t e = cudaMallocAsync(&h->mem, off_rank + rank_bytes, s);
  if (e != cudaSuccess) {
    delete h;
    return alk::cuda_fail(e);
  }
  h->bytes = off_rank + rank_bytes;
  uint8_t* p = (uint8_t*)h->mem;
  h->v.cap = cap;
  h->v.key = mode == ALK_DENSE_FULL ? (int64_t*)p : nullptr;
  h->v.payload = mode == ALK_DENSE_FULL ? (int64_t*)(p + off_pay) : nullptr;
  h->v.slot_cap = cap;
  h->v.npay = npay;
  h->v.nslots = (unsigned long long*)(p + off_ctr);
  h->v.flags = (int*)(p + off_ctr + 8);
  h->v.bits = (uint32_t*)(p + off_bits);
  h->v.kmin = key_min;
  h->v.nbits = span;
  h->v.rank = (uint32_t*)(p + off_rank);
  h->v.dense_mode = (uint32_t)mode;
  CK(cudaMemsetAsync(p + off_ctr, 0, off_rank - off_ctr, s));  // counters and bitmap
  *out = h;
  return ALK_OK;
}

int alk_ht_create_dense(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, alk_ht** out,
                        alk_stream stream) {
  return alk_ht_create_dense_mode(max_keys, npay, key_min, key_max, ALK_DENSE_FULL, out, stream);
}

int alk_ht_create(uint64_t max_keys, uint32_t npay, alk_ht** out, alk_stream stream) {
  return alk_ht_create_range(max_keys, npay, 1, 0, out, stream);
}

void alk_ht_free(alk_ht* h, alk_stream stream) {
  if (!h) return;
  if (h->mem) cudaFreeAsync(h->mem, (cudaStream_t)stream);
  delete h;
}

int alk_ht_info(const alk_ht* h, uint64_t* nslots, int* flags, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h) return ALK_ERR_ARG;
  unsigned long long n = 0;
  int f[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(&n, h->v.nslots, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(f, h->v.flags, sizeof(f), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (nslots) *nslots = std::min<uint64_t>(n, h->v.slot_cap);
  if (flags) *flags = (f[0] ? 1 : 0) | (f[1] ? 2 : 0) | (f[2] ? 4 : 0) | (f[3] ? 8 : 0);
  return ALK_OK;
}

uint64_t alk_ht_slots(const alk_ht* h) { return h ? h->v.slot_cap : 0; }

uint64_t alk_ht_bytes(const alk_ht* h) { return h ? h->bytes : 0; }

const int64_t* alk_ht_keys(const alk_ht* h) { return h ? h->v.key : nullptr; }

const int64_t* alk_ht_payload(const alk_ht* h, uint32_t p) {
  if (!h || p >= h->v.npay) return nullptr;
  return h->v.payload + (uint64_t)p * h->v.slot_cap;
}

static int stage_common(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                        const alk_program* progs, uint32_t nprogs, std::vector<uint8_t>& hb, StageArgs& a,
                        size_t extra_bytes, size_t* off_extra) {
  if (nseg == 0) return ALK_ERR_ARG;
  std::vector<uint32_t> seg_tile(nseg + 1, 0);
  uint64_t ntiles = 0;
  for (uint32_t g = 0; g < nseg; g++) {
    seg_tile[g] = (uint32_t)ntiles;
    if (seg_mode[g] == 0) continue;
    const uint32_t rows = cols[g].rows;
    for (uint32_t c = 0; c < ncols; c++) {
      const alk_colseg& d = cols[c * nseg + g];
      if (d.rows != rows || !(d.bits == 8 || d.bits == 16 || d.bits == 32 || d.bits == 64)) return ALK_ERR_ARG;
      if (rows && !d.data) return ALK_ERR_ARG;
    }
    ntiles += (rows + kTile - 1) / kTile;
  }
  if (ntiles >= 0xffffffffull) return ALK_ERR_TOO_LARGE;
  seg_tile[nseg] = (uint32_t)ntiles;
  a.ntiles = (uint32_t)ntiles;
  size_t off_cols = 0;
  size_t off_mode = off_cols + sizeof(alk_colseg) * ncols * nseg;
  size_t off_tile = (off_mode + nseg + 15) & ~size_t(15);
  size_t off_prog = (off_tile + 4 * (nseg + 1) + 15) & ~size_t(15);
  size_t off_x = (off_prog + sizeof(alk_program) * nprogs + 15) & ~size_t(15);
  hb.assign(off_x + extra_bytes + 16, 0);
  std::memcpy(&hb[off_cols], cols, sizeof(alk_colseg) * ncols * nseg);
  std::memcpy(&hb[off_mode], seg_mode, nseg);
  std::memcpy(&hb[off_tile], seg_tile.data(), 4 * (nseg + 1));
  std::memcpy(&hb[off_prog], progs, sizeof(alk_program) * nprogs);
  a.ncols = ncols;
  a.nseg = nseg;
  a.nprogs = nprogs;
  *off_extra = off_x;
  // device offsets are patched by the caller once the buffer exists
  a.cols = (const alk_colseg*)(uintptr_t)off_cols;
  a.seg_mode = (const uint8_t*)(uintptr_t)off_mode;
  a.seg_tile = (const uint32_t*)(uintptr_t)off_tile;
  a.progs = (const alk_program*)(uintptr_t)off_prog;
  return ALK_OK;
}

static void patch(StageArgs& a, uint8_t* db) {
  a.cols = (const alk_colseg*)(db + (uintptr_t)a.cols);
  a.seg_mode = db + (uintptr_t)a.seg_mode;
  a.seg_tile = (const uint32_t*)(db + (uintptr_t)a.seg_tile);
  a.progs = (const alk_program*)(db + (uintptr_t)a.progs);
}

// Uploads a stage's arguments with its counters and hit list in one stream-ordered
// allocation, runs scan + hit kernels, reads the counters back (one synchronisation).
// hit_cap 0 (or above the rows scanned) means the rows scanned, which cannot overflow.
}  // extern "C"
template <bool kBuild>
static int run_stage(StageArgs& a, const alk_program& pred, const alk_colseg* cols, const uint8_t* seg_mode,
                     const std::vector<uint8_t>& hb, size_t off_x, uint64_t hit_cap, uint64_t* h_rows_in,
                     uint64_t* h_hits, alk_stage_status* h_status, cudaStream_t s, alk_event_timer* timer) {
  uint64_t upper = 0;
  for (uint32_t g = 0; g < a.nseg; g++)
    if (seg_mode[g]) upper += cols[g].rows;
  if (hit_cap == 0 || hit_cap > upper) hit_cap = upper;
  // room for the survivors plus the unused tail of every scan warp's last chunk
  hit_cap += std::min<uint64_t>(a.ntiles, (uint64_t)sms() * 8) * 8 * kChunk;
  // conjunctive predicates: per conjunct and segment, the raw-domain test (segments the
  // zone maps pass whole need none)
  FastArgs fa{};
  const bool conj = as_conjuncts(pred, fa.conj, &fa.nconj);
  std::vector<ConjSeg> cs;
  if (conj) {
    cs.resize((size_t)fa.nconj * a.nseg);
    for (uint32_t c = 0; c < fa.nconj; c++)
      for (uint32_t g = 0; g < a.nseg; g++)
        cs[c * a.nseg + g] = seg_mode[g] == 1 ? ConjSeg{0, 0, kCjAlways, 0}
                                              : conj_seg(fa.conj[c], cols[fa.conj[c].slot * a.nseg + g]);
  }
  // per segment: 32-bit evaluation when every staged column stores <= 32 bits and the
  // stored probe key maps to its bitmap index without leaving 32-bit arithmetic
  std::vector<SegPlan> sp(a.nseg, SegPlan{0, 0, 0, 0, 0, 0});
  for (uint32_t g = 0; g < a.nseg; g++) {
    bool narrow = conj;
    for (uint32_t c = 0; conj && c < fa.nconj; c++)
      if (cols[fa.conj[c].slot * a.nseg + g].bits > 32) narrow = false;
    if (a.probe_slot >= 0) {
      const alk_colseg& d = cols[a.probe_slot * a.nseg + g];
      if (d.bits > 32) narrow = false;
      if (narrow && a.probe.bits) {
        // stored values x in [0, 2^bits) whose key x + lower lies in [kmin, kmin + nbits)
        const __int128 blo = (__int128)a.probe.kmin - d.lower;  // x of the first bitmap key
        const __int128 xmax = ((__int128)1 << d.bits) - 1;
        const __int128 lo = std::max<__int128>(blo, 0);
        const __int128 hi = std::min<__int128>(blo + (__int128)a.probe.nbits - 1, xmax);
        if (lo <= hi) {
          sp[g].kmember = 1;
          sp[g].xlo = (uint32_t)lo;
          sp[g].xspan = (uint32_t)(hi - lo);
          sp[g].boff = (uint32_t)(lo - blo);  // < nbits < 2^32
        }
      }
    }
    sp[g].narrow = narrow ? 1 : 0;
  }
  const size_t off_cs = (hb.size() + 15) & ~size_t(15);
  const size_t off_sp = (off_cs + cs.size() * sizeof(ConjSeg) + 15) & ~size_t(15);
  // zeroed tail: the stage counters, then (dense build) the look-back state of the rank
  // prefix; the survivor list follows, in entries of up to wmax words
  const bool dense = kBuild && a.build.rank != nullptr;
  const uint32_t wmax = dense ? 2 + a.build.npay : 1;
  const uint32_t rk_tiles = dense ? (uint32_t)(((a.build.nbits + 31) / 32 + kRankTile - 1) / kRankTile) : 0;
  const size_t off_tail = (off_sp + sp.size() * sizeof(SegPlan) + 15) & ~size_t(15);
  const size_t off_rk_aggs = 32;
  const size_t off_rk_incls = off_rk_aggs + 8 * (size_t)rk_tiles;
  const size_t tail_bytes = off_rk_incls + 8 * (size_t)rk_tiles;
  const size_t off_hits = (off_tail + tail_bytes + 255) & ~size_t(255);
  std::vector<uint8_t> up(off_tail, 0);
  std::memcpy(up.data(), hb.data(), hb.size());
  if (!cs.empty()) std::memcpy(up.data() + off_cs, cs.data(), cs.size() * sizeof(ConjSeg));
  std::memcpy(up.data() + off_sp, sp.data(), sp.size() * sizeof(SegPlan));
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, off_hits + std::max<uint64_t>(hit_cap, 1) * wmax * sizeof(Hit), s));
  cudaError_t ue;
  const void* src = alk::upload_source(up.data(), up.size(), s, &ue);
  CK(ue);
  CK(cudaMemcpyAsync(db, src, up.size(), cudaMemcpyHostToDevice, s));
  uint8_t* tail = db + off_tail;
  CK(cudaMemsetAsync(tail, 0, tail_bytes, s));
  patch(a, db);
  if (kBuild) a.pay_src = (const int32_t*)(db + off_x);
  else a.agg_kind = db + off_x;
  a.rows_in = (unsigned long long*)tail;
  a.hit_count = (unsigned long long*)(tail + 8);
  a.err = (int*)(tail + 16);
  a.hit_rows = (unsigned long long*)(tail + 24);
  a.rk_aggs = (uint64_t*)(tail + off_rk_aggs);
  a.rk_incls = (uint64_t*)(tail + off_rk_incls);
  a.rk_tiles = rk_tiles;
  a.hits = (Hit*)(db + off_hits);
  a.hit_cap = hit_cap;
  a.hit_words = 1;
  fa.a = a;
  fa.cseg = (const ConjSeg*)(db + off_cs);
  fa.splan = (const SegPlan*)(db + off_sp);
  bool narrow_all = true;
  for (uint32_t g = 0; g < a.nseg; g++)
    if (seg_mode[g] && !sp[g].narrow) narrow_all = false;
  CK(launch_stage<kBuild>(fa, conj, narrow_all, cols, seg_mode, kBuild ? (const int32_t*)(hb.data() + off_x) : nullptr,
                          s, timer));
  static_assert(sizeof(alk_stage_status) == 32, "status mirrors the counters after the arguments");
  if (h_status) {  // asynchronous: the counters land in the caller's (pinned) status
    if (timer && timer->on && a.ntiles) timer->launches++;
    CK(cudaMemcpyAsync(h_status, tail, 32, cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(db, s));
    return ALK_OK;
  }
  unsigned long long back[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(back, tail, 32, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  if (timer && timer->on && a.ntiles) {
    float ms = 0;
    cudaEventElapsedTime(&ms, (cudaEvent_t)timer->ev0, (cudaEvent_t)timer->ev1);
    timer->ms += ms;
    timer->launches++;
  }
  if (h_rows_in) *h_rows_in = back[0];
  if (h_hits) *h_hits = back[3];
  return (int)(uint32_t)back[2];
}
extern "C" {

static int pipeline_build(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                          const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                          int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap, uint64_t* h_rows_in,
                          uint64_t* h_hits, alk_stage_status* h_status, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!build || ncols == 0 || ncols > kMaxCols || build_slot < 0 || (uint32_t)build_slot >= ncols) return ALK_ERR_ARG;
  if ((probe_slot >= 0) != (probe != nullptr) || (probe_slot >= 0 && (uint32_t)probe_slot >= ncols))
    return ALK_ERR_ARG;
  uint32_t npay_probe = probe ? probe->v.npay : 0;
  for (uint32_t p = 0; p < build->v.npay; p++) {
    int32_t src = pay_src[p];
    if (!((src >= 0 && (uint32_t)src < ncols) || (src >= 32 && (uint32_t)(src - 32) < npay_probe))) return ALK_ERR_ARG;
  }
  alk_program prog{};
  if (pred) prog = *pred;
  if (!prog_ok(prog, ncols, 0)) return ALK_ERR_ARG;  // the predicate reads scan columns only
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, &prog, 1, hb, a, 4 * 8, &off_x);
  if (rc) return rc;
  if (build->v.npay) std::memcpy(&hb[off_x], pay_src, 4 * build->v.npay);
  a.probe_slot = probe_slot;
  if (probe) a.probe = probe->v;
  a.build_slot = build_slot;
  a.build = build->v;
  for (uint32_t p = 0; p < build->v.npay; p++)
    if (pay_src[p] >= 32) a.need_slot = 1;
  if (probe && probe->v.dense_mode == ALK_DENSE_BITS && a.need_slot) return ALK_ERR_ARG;  // no slots
  return run_stage<true>(a, prog, cols, seg_mode, hb, off_x, hit_cap, h_rows_in, h_hits, h_status, s, nullptr);
}

int alk_pipeline_build(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                       const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                       int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap, uint64_t* h_rows_in,
                       uint64_t* h_hits, alk_stream stream) {
  return pipeline_build(cols, ncols, nseg, seg_mode, pred, probe, probe_slot, build, build_slot, pay_src, hit_cap,
                        h_rows_in, h_hits, nullptr, stream);
}

int alk_pipeline_build_async(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                             const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                             int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap,
                             alk_stage_status* h_status, alk_stream stream) {
  if (!h_status) return ALK_ERR_ARG;
  return pipeline_build(cols, ncols, nseg, seg_mode, pred, probe, probe_slot, build, build_slot, pay_src, hit_cap,
                        nullptr, nullptr, h_status, stream);
}

static int pipeline_probe_agg(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                              const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                              const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, int64_t* d_acc,
                              uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap, uint64_t* h_rows_in,
                              uint64_t* h_hits, alk_stage_status* h_status, alk_stream stream,
                              alk_event_timer* timer) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!probe || probe_slot < 0 || (uint32_t)probe_slot >= ncols || ncols == 0 || ncols > kMaxCols || nagg > 7)
    return ALK_ERR_ARG;
  if (acc_stride < probe->v.slot_cap) return ALK_ERR_ARG;  // accumulators indexed by table position
  if (probe->v.dense_mode == ALK_DENSE_BITS) return ALK_ERR_ARG;  // a membership-only table has no slots

  std::vector<alk_program> progs(1 + nagg);
  std::memset(progs.data(), 0, sizeof(alk_program) * progs.size());
  if (pred) progs[0] = *pred;
  for (uint32_t g = 0; g < nagg; g++) {
    if (agg_kind[g] > ALK_AGG_MAX) return ALK_ERR_ARG;
    if (agg_kind[g] != ALK_AGG_COUNT) progs[1 + g] = agg_progs[g];
  }
  for (size_t p = 0; p < progs.size(); p++)
    if (!prog_ok(progs[p], ncols, p ? probe->v.npay : 0)) return ALK_ERR_ARG;
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, progs.data(), (uint32_t)progs.size(), hb, a, 16, &off_x);
  if (rc) return rc;
  std::memcpy(&hb[off_x], agg_kind, nagg);
  a.probe_slot = probe_slot;
  a.probe = probe->v;
  a.need_slot = 1;  // accumulators are indexed by the probed key's position
  a.build_slot = -1;
  a.nagg = nagg;
  a.acc = d_acc;
  a.acc_stride = acc_stride;
  a.cnt = (unsigned long long*)d_cnt;
  return run_stage<false>(a, progs[0], cols, seg_mode, hb, off_x, hit_cap, h_rows_in, h_hits, h_status, s, timer);
}

int alk_pipeline_probe_agg(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                           const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                           const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, int64_t* d_acc,
                           uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap, uint64_t* h_rows_in,
                           uint64_t* h_hits, alk_stream stream, alk_event_timer* timer) {
  return pipeline_probe_agg(cols, ncols, nseg, seg_mode, pred, probe, probe_slot, agg_progs, agg_kind, nagg, d_acc,
                            acc_stride, d_cnt, hit_cap, h_rows_in, h_hits, nullptr, stream, timer);
}

int alk_pipeline_probe_agg_async(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                                 const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                                 const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg,
                                 int64_t* d_acc, uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap,
                                 alk_stage_status* h_status, alk_stream stream, alk_event_timer* timer) {
  if (!h_status) return ALK_ERR_ARG;
  return pipeline_probe_agg(cols, ncols, nseg, seg_mode, pred, probe, probe_slot, agg_progs, agg_kind, nagg, d_acc,
                            acc_stride, d_cnt, hit_cap, nullptr, nullptr, h_status, stream, timer);
}

int alk_ht_info_async(const alk_ht* h, alk_ht_status* h_out, alk_stream stream) {
  if (!h || !h_out) return ALK_ERR_ARG;
  static_assert(sizeof(alk_ht_status) == 24, "inserted count followed by the four flags");
  CK(cudaMemcpyAsync(h_out, h->v.nslots, 24, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  return ALK_OK;
}

int alk_fill_i64(int64_t* d, uint64_t n, int64_t v, alk_stream stream) {
  if (n == 0) return ALK_OK;
  k_fill_i64<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(d, n, v);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_topk_candidates(const int64_t* d_rank, const uint64_t* d_live, uint64_t n, uint32_t k, uint32_t* d_out,
                        uint64_t cap, uint64_t* h_count, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_count || k == 0 || k > 4096) return ALK_ERR_ARG;
  *h_count = 0;
  if (n == 0) return ALK_OK;
  const bool one_pass = k <= (uint32_t)kTopK;
  const int blocks = one_pass ? (int)std::min<uint64_t>((n + kT - 1) / kT, (uint64_t)sms() * 2)
                              : (int)std::min<uint64_t>((n + 1023) / 1024, (uint64_t)sms() * 2);
  std::vector<int64_t> best((size_t)blocks * k);
  void* db = nullptr;
  CK(cudaMallocAsync(&db, best.size() * 8 + 16, s));
  if (one_pass) {
    k_topk_local16<<<blocks, kT, 0, s>>>(d_rank, (const unsigned long long*)d_live, n, k, (int64_t*)db);
  } else {
    k_topk_local<<<blocks, kT, 0, s>>>(d_rank, (const unsigned long long*)d_live, n, k, (int64_t*)db);
  }
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(best.data(), db, best.size() * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::sort(best.begin(), best.end(), [](int64_t x, int64_t y) { return x > y; });
  int64_t thr = best[std::min<size_t>(k, best.size()) - 1];
  unsigned long long* cnt = (unsigned long long*)db;
  CK(cudaMemsetAsync(cnt, 0, 8, s));
  k_topk_collect<<<grid_for(n), kT, 0, s>>>(d_rank, (const unsigned long long*)d_live, n, thr, d_out, cap, cnt);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  unsigned long long c = 0;
  CK(cudaMemcpyAsync(&c, cnt, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  *h_count = c;
  return c > cap ? ALK_ERR_OVERFLOW : ALK_OK;
}

int alk_topk_select(const int64_t* d_rank, const uint64_t* d_live, uint64_t n, uint32_t k, uint32_t* d_out,
                    uint64_t cap, uint64_t* d_count, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!d_count || !d_out || k == 0 || k > (uint32_t)kTopK) return ALK_ERR_ARG;
  CK(cudaMemsetAsync(d_count, 0, 8, s));
  if (n == 0) return ALK_OK;
  const unsigned long long* live = (const unsigned long long*)d_live;
  // 1. the sampled threshold: per-block lists over every kSampleStride-th slot, merged
  const uint64_t ns = (n + kSampleStride - 1) / kSampleStride;
  const int sblocks = (int)std::min<uint64_t>(std::min<uint64_t>((ns + kT - 1) / kT, (uint64_t)kMergeMax / k),
                                              (uint64_t)sms() * 4);
  // 2. the exact full pass's per-block lists, should the sampled selection fall back
  const int blocks = (int)std::min<uint64_t>(std::min<uint64_t>((n + kT - 1) / kT, (uint64_t)kMergeMax / k),
                                             (uint64_t)sms() * 4);
  const uint64_t ccap = kTopKCollect;  // slots collected at or above the sampled threshold
  const size_t off_sthr = (size_t)sblocks * k, off_lists = off_sthr + 1, off_thr = off_lists + (size_t)blocks * k;
  const size_t off_ctr = off_thr + 1, off_cand = off_ctr + 2;  // [ncand, fallback flag]
  int64_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, (off_cand * 8 + ccap * 4 + 15) & ~size_t(15), s));
  unsigned long long* ncand = (unsigned long long*)(db + off_ctr);
  int* fallback = (int*)(db + off_ctr + 1);
  uint32_t* cand = (uint32_t*)(db + off_cand);
  CK(cudaMemsetAsync(db + off_ctr, 0, 16, s));
  k_topk_sample<<<sblocks, kT, 0, s>>>(d_rank, live, n, k, db);
  k_topk_merge<<<1, kMergeThreads, 0, s>>>(db, (uint32_t)sblocks * k, k, db + off_sthr);
  k_topk_collect_dev<<<grid_for(n), kT, 0, s>>>(d_rank, live, n, db + off_sthr, cand, ccap, ncand);
  k_topk_refine<<<1, kMergeThreads, 0, s>>>(d_rank, cand, ncand, ccap, k, d_out, cap,
                                           (unsigned long long*)d_count, fallback);
  k_topk_local16_if<<<blocks, kT, 0, s>>>(fallback, d_rank, live, n, k, db + off_lists);
  k_topk_merge_if<<<1, kMergeThreads, 0, s>>>(fallback, db + off_lists, (uint32_t)blocks * k, k, db + off_thr);
  k_topk_collect_if<<<grid_for(n), kT, 0, s>>>(fallback, d_rank, live, n, db + off_thr, d_out, cap,
                                               (unsigned long long*)d_count);
  alk::g_kernel_launches += 7;
  CK(cudaGetLastError());
  CK(cudaFreeAsync(db, s));
  return ALK_OK;
}

int alk_gather_rows(const int64_t* const* d_cols, uint32_t ncols, const uint32_t* d_idx, const uint64_t* d_count,
                    uint64_t cap, int64_t* d_out, alk_stream stream) {
  if (ncols == 0 || ncols > (uint32_t)kGatherCols || !d_idx || !d_count || !d_out) return ALK_ERR_ARG;
  if (cap == 0) return ALK_OK;
  GatherCols g{};
  for (uint32_t c = 0; c < ncols; c++) {
    if (!d_cols[c]) return ALK_ERR_ARG;
    g.col[c] = d_cols[c];
  }
  k_gather_rows<<<grid_for(cap * ncols), kT, 0, (cudaStream_t)stream>>>(
      g, ncols, d_idx, (const unsigned long long*)d_count, cap, d_out);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

int alk_ht_late_rows(const alk_ht* h, const uint32_t* d_cand, const uint64_t* d_count, uint32_t cap,
                     const alk_colseg* cols, uint32_t npay, uint32_t nseg, const uint8_t* seg_mode,
                     const int64_t* seg_lo, const int64_t* seg_hi, int64_t* const* d_out, int32_t* d_status,
                     alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h || h->v.dense_mode != ALK_DENSE_RANKS || !d_cand || !d_count || !cols || !seg_mode || !seg_lo ||
      !seg_hi || !d_out || !d_status || npay > 8 || nseg == 0)
    return ALK_ERR_ARG;
  for (uint32_t c = 0; c <= npay; c++)
    if (!d_out[c]) return ALK_ERR_ARG;
  for (uint32_t c = 0; c <= npay; c++)
    for (uint32_t g = 0; g < nseg; g++) {
      const alk_colseg& d = cols[(size_t)c * nseg + g];
      if (d.rows != cols[g].rows || !(d.bits == 8 || d.bits == 16 || d.bits == 32 || d.bits == 64)) return ALK_ERR_ARG;
      if (seg_mode[g] && d.rows && !d.data) return ALK_ERR_ARG;
    }
  if (cap == 0) return ALK_OK;
  // one upload: descriptors, zone bounds, output addresses, segment verdicts
  const size_t n_cols = (size_t)(1 + npay) * nseg;
  const size_t off_lo = (n_cols * sizeof(alk_colseg) + 15) & ~size_t(15);
  const size_t off_hi = off_lo + 8 * (size_t)nseg;
  const size_t off_out = off_hi + 8 * (size_t)nseg;
  const size_t off_mode = off_out + 8 * (size_t)(1 + npay);
  const size_t up_bytes = (off_mode + nseg + 15) & ~size_t(15);
  std::vector<uint8_t> up(up_bytes, 0);
  std::memcpy(up.data(), cols, n_cols * sizeof(alk_colseg));
  std::memcpy(up.data() + off_lo, seg_lo, 8 * (size_t)nseg);
  std::memcpy(up.data() + off_hi, seg_hi, 8 * (size_t)nseg);
  std::memcpy(up.data() + off_out, d_out, 8 * (size_t)(1 + npay));
  std::memcpy(up.data() + off_mode, seg_mode, nseg);
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, up_bytes, s));
  cudaError_t ue;
  const void* src = alk::upload_source(up.data(), up.size(), s, &ue);
  CK(ue);
  CK(cudaMemcpyAsync(db, src, up.size(), cudaMemcpyHostToDevice, s));
  LateArgs a{};
  a.h = h->v;
  a.cand = d_cand;
  a.count = (const unsigned long long*)d_count;
  a.cap = cap;
  a.nseg = nseg;
  a.npay = npay;
  a.cols = (const alk_colseg*)db;
  a.seg_lo = (const int64_t*)(db + off_lo);
  a.seg_hi = (const int64_t*)(db + off_hi);
  a.out = (int64_t* const*)(db + off_out);
  a.seg_mode = db + off_mode;
  a.status = d_status;
  const uint32_t blocks = std::min<uint32_t>((cap + kT / 32 - 1) / (kT / 32), (uint32_t)sms() * 2);
  k_late_rows<<<blocks, kT, 0, s>>>(a);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaFreeAsync(db, s));
  return ALK_OK;
}

int alk_seg_sorted(const alk_colseg* segs, uint32_t nseg, uint8_t* h_sorted, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nseg == 0) return ALK_OK;
  if (!segs || !h_sorted || nseg > 65535) return ALK_ERR_ARG;
  uint64_t most = 0;
  for (uint32_t g = 0; g < nseg; g++) {
    if (!(segs[g].bits == 8 || segs[g].bits == 16 || segs[g].bits == 32 || segs[g].bits == 64)) return ALK_ERR_ARG;
    if (segs[g].rows && !segs[g].data) return ALK_ERR_ARG;
    most = std::max<uint64_t>(most, segs[g].rows);
  }
  const size_t off_flags = (sizeof(alk_colseg) * (size_t)nseg + 15) & ~size_t(15);
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, off_flags + 4 * (size_t)nseg, s));
  CK(cudaMemcpyAsync(db, segs, sizeof(alk_colseg) * nseg, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(db + off_flags, 0, 4 * (size_t)nseg, s));
  const uint32_t bx = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((most + kT * 16 - 1) / (kT * 16), 512));
  k_seg_unsorted<<<dim3(bx, nseg), kT, 0, s>>>((const alk_colseg*)db, (uint32_t*)(db + off_flags));
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  std::vector<uint32_t> f(nseg);
  CK(cudaMemcpyAsync(f.data(), db + off_flags, 4 * (size_t)nseg, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  for (uint32_t g = 0; g < nseg; g++) h_sorted[g] = f[g] ? 0 : 1;
  return ALK_OK;
}

int alk_pipeline_groupby(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                         const alk_program* pred, const int32_t* key_slots, uint32_t nkeys,
                         const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, uint64_t max_groups,
                         const int64_t* key_min, const int64_t* key_max, int64_t* const* d_out_keys,
                         int64_t* const* d_out_vals, uint64_t out_cap, uint64_t* h_groups, uint64_t* h_seg_rows,
                         uint64_t* h_rows_in, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_groups || ncols == 0 || ncols > kMaxCols || nkeys == 0 || nkeys > 4 || nagg > 7 || !key_slots ||
      (nagg && (!agg_kind || !d_out_vals)) || !d_out_keys)
    return ALK_ERR_ARG;
  *h_groups = 0;
  for (uint32_t j = 0; j < nkeys; j++)
    if (key_slots[j] < 0 || (uint32_t)key_slots[j] >= ncols || !d_out_keys[j]) return ALK_ERR_ARG;
  std::vector<alk_program> progs(1 + nagg);
  std::memset(progs.data(), 0, sizeof(alk_program) * progs.size());
  if (pred) progs[0] = *pred;
  for (uint32_t v = 0; v < nagg; v++) {
    if (agg_kind[v] > ALK_AGG_MAX || !d_out_vals[v]) return ALK_ERR_ARG;
    if (agg_kind[v] != ALK_AGG_COUNT) progs[1 + v] = agg_progs[v];
  }
  for (auto& p : progs)
    if (!prog_ok(p, ncols, 0)) return ALK_ERR_ARG;  // scan columns only
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, progs.data(), (uint32_t)progs.size(), hb, a,
                        16 + 8 * (size_t)(nkeys + nagg), &off_x);
  if (rc) return rc;
  std::memcpy(&hb[off_x], agg_kind, nagg);
  const size_t off_outp = off_x + 16;
  std::memcpy(&hb[off_outp], d_out_keys, 8 * (size_t)nkeys);
  if (nagg) std::memcpy(&hb[off_outp + 8 * (size_t)nkeys], d_out_vals, 8 * (size_t)nagg);
  FastArgs fa{};
  const bool conj = as_conjuncts(progs[0], fa.conj, &fa.nconj);
  std::vector<ConjSeg> cs;
  if (conj)
    for (uint32_t c = 0; c < fa.nconj; c++)
      for (uint32_t g = 0; g < nseg; g++)
        cs.push_back(seg_mode[g] == 1 ? ConjSeg{0, 0, kCjAlways, 0} : conj_seg(fa.conj[c], cols[fa.conj[c].slot * nseg + g]));
  // Direct form when the key ranges are known and their product is small: at most 2^32
  // slots, no more than 16 per scanned row, and records within 24 GB. Otherwise a
  // hash table at most 0.7 full at max_groups.
  uint64_t rows = 0;
  for (uint32_t g = 0; g < nseg; g++)
    if (seg_mode[g]) rows += cols[g].rows;
  bool direct = key_min && key_max;
  uint64_t space = 1, span[4] = {1, 1, 1, 1};
  for (uint32_t j = 0; direct && j < nkeys; j++) {
    if (key_max[j] < key_min[j]) {
      span[j] = 1;  // nothing scanned: any key lies outside, which the kernel reports
      continue;
    }
    span[j] = (uint64_t)key_max[j] - (uint64_t)key_min[j] + 1;
    if (span[j] == 0 || span[j] > (1ull << 32) || space > (1ull << 32) / span[j]) direct = false;
    else space *= span[j];
  }
  uint32_t dw = 1;  // record words of the direct form (accumulators, padded)
  while (dw < nagg) dw <<= 1;
  if (direct && (space > 16 * std::max<uint64_t>(rows, 1024) || (long double)space * 8.0L * dw > 24.0L * (1ull << 30)))
    direct = false;
  uint64_t cap = 1024;
  if (direct) cap = space;
  else
    while ((long double)cap * 0.7L < (long double)std::max<uint64_t>(max_groups, 1)) cap <<= 1;
  const bool one = nkeys == 1 && !direct;
  const size_t off_cs = (hb.size() + 15) & ~size_t(15);
  const size_t off_ctr = (off_cs + cs.size() * sizeof(ConjSeg) + 255) & ~size_t(255);
  const size_t ctr_bytes = 32 + 8 * (size_t)nseg;  // rows_in, groups, err, pad, seg_rows
  const size_t off_keys = (off_ctr + ctr_bytes + 255) & ~size_t(255);
  // record: key words (hash forms), accumulators; padded to 1, 2, 4 or 8 words when that fits
  const uint32_t kw = direct ? 0 : nkeys;
  uint32_t rw = std::max<uint32_t>(kw + nagg, 1);
  if (rw <= 8) rw = rw <= 1 ? 1 : rw <= 2 ? 2 : rw <= 4 ? 4 : 8;
  const size_t off_state = (off_keys + 8 * (size_t)rw * cap + 15) & ~size_t(15);  // state words or presence bits
  const size_t state_bytes = direct ? 4 * ((cap + 31) / 32) : one ? 0 : 4 * (size_t)cap;
  const size_t total = off_state + state_bytes;
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, total, s));
  std::vector<uint8_t> up(off_ctr, 0);
  std::memcpy(up.data(), hb.data(), hb.size());
  if (!cs.empty()) std::memcpy(up.data() + off_cs, cs.data(), cs.size() * sizeof(ConjSeg));
  cudaError_t ue;
  const void* src = alk::upload_source(up.data(), up.size(), s, &ue);
  CK(ue);
  CK(cudaMemcpyAsync(db, src, up.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(db + off_ctr, 0, ctr_bytes, s));
  if (state_bytes) CK(cudaMemsetAsync(db + off_state, 0, state_bytes, s));
  patch(a, db);
  a.agg_kind = db + off_x;
  a.nagg = nagg;
  a.rows_in = (unsigned long long*)(db + off_ctr);
  a.err = (int*)(db + off_ctr + 16);
  fa.a = a;
  fa.cseg = (const ConjSeg*)(db + off_cs);
  GroupTable g{};
  g.cap = cap;
  g.rec = (int64_t*)(db + off_keys);
  g.rw = rw;
  g.kw = kw;
  g.state = one || direct ? nullptr : (uint32_t*)(db + off_state);
  g.occ = direct ? (uint32_t*)(db + off_state) : nullptr;
  g.nkeys = nkeys;
  if (direct) {
    uint64_t stride = 1;
    for (int j = (int)nkeys - 1; j >= 0; j--) {  // the last key column varies fastest
      g.kmin[j] = key_min[j];
      g.kspan[j] = span[j];
      g.kstride[j] = stride;
      stride *= span[j];
    }
  }
  for (uint32_t j = 0; j < nkeys; j++) g.key_slot[j] = key_slots[j];
  g.generic = progs[0].n_instr && !conj;
  g.seg_rows = (unsigned long long*)(db + off_ctr + 32);
  g.groups = (unsigned long long*)(db + off_ctr + 8);
  g.out_keys = (int64_t* const*)(db + off_outp);
  g.out_vals = (int64_t* const*)(db + off_outp + 8 * (size_t)nkeys);
  g.out_cap = out_cap;
  uint64_t kinds = 0;
  for (uint32_t v = 0; v < nagg; v++) kinds |= (uint64_t)agg_kind[v] << (8 * v);
  k_group_init<<<grid_for(cap * rw), kT, 0, s>>>(g, nagg, kinds);
  alk::g_kernel_launches++;
  if (a.ntiles) {
    void (*kern)(const FastArgs, const GroupTable) = direct ? k_group_scan<2> : one ? k_group_scan<0> : k_group_scan<1>;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kT, 0);
    const int grid = std::min<int>((int)a.ntiles, sms() * std::max(occ, 1));
    kern<<<grid, kT, 0, s>>>(fa, g);
    alk::g_kernel_launches++;
  }
  if (direct) k_group_compact_direct<<<grid_for((cap + 31) / 32), kT, 0, s>>>(g, nagg);
  else k_group_compact<<<grid_for(cap), kT, 0, s>>>(g, nagg);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  std::vector<unsigned long long> back(4 + nseg);
  CK(cudaMemcpyAsync(back.data(), db + off_ctr, ctr_bytes, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  *h_groups = back[1];
  if (h_rows_in) *h_rows_in = back[0];
  if (h_seg_rows)
    for (uint32_t g2 = 0; g2 < nseg; g2++) h_seg_rows[g2] = back[4 + g2];
  const int err = (int)(uint32_t)back[2];
  if (err) return err;
  return back[1] > out_cap ? ALK_ERR_OVERFLOW : ALK_OK;
}

int alk_live_compact(const uint64_t* d_live, uint64_t n, uint32_t* d_out, uint64_t* h_count, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_count) return ALK_ERR_ARG;
  *h_count = 0;
  if (n == 0) return ALK_OK;
  void* db = nullptr;
  CK(cudaMallocAsync(&db, 16, s));
  CK(cudaMemsetAsync(db, 0, 16, s));
  k_live_compact<<<grid_for(n), kT, 0, s>>>((const unsigned long long*)d_live, n, d_out, (unsigned long long*)db);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  unsigned long long c = 0;
  CK(cudaMemcpyAsync(&c, db, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  *h_count = c;
  return ALK_OK;
}

}  // extern "C"

namespace alk {
bool program_conjuncts(const alk_program& p, std::vector<CardConj>& out) {
  Conj cj[kMaxConj];
  uint32_t n = 0;
  out.clear();
  if (!as_conjuncts(p, cj, &n)) return false;
  for (uint32_t i = 0; i < n; i++) out.push_back({cj[i].mul, cj[i].k, cj[i].slot, cj[i].op});
  return true;
}
}  // namespace alk

extern "C" {

int alk_card_count(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                   const alk_program* pred, const alk_ht* probe, int32_t probe_slot, int32_t key_slot,
                   int64_t key_min, int64_t key_max, uint64_t* h_counts, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!h_counts || ncols == 0 || ncols > kMaxCols) return ALK_ERR_ARG;
  if ((probe_slot >= 0) != (probe != nullptr) || (probe_slot >= 0 && (uint32_t)probe_slot >= ncols))
    return ALK_ERR_ARG;
  if (key_slot >= 0 && (uint32_t)key_slot >= ncols) return ALK_ERR_ARG;
  alk_program prog{};
  if (pred) prog = *pred;
  if (!prog_ok(prog, ncols, 0)) return ALK_ERR_ARG;
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, &prog, 1, hb, a, 0, &off_x);
  if (rc) return rc;
  a.probe_slot = probe_slot;
  if (probe) a.probe = probe->v;
  // distinct values are counted when the key range is known and at most 2^30 values
  uint64_t nbits = 0;
  if (key_slot >= 0 && key_max >= key_min) {
    const uint64_t span = (uint64_t)key_max - (uint64_t)key_min + 1;
    if (span != 0 && span <= (1ull << 30)) nbits = span;
  }
  const size_t off_cnt = (hb.size() + 255) & ~size_t(255);
  const size_t off_bits = off_cnt + ((24 * (size_t)nseg + 255) & ~size_t(255));
  const size_t words = (nbits + 31) / 32;
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, off_bits + words * 4 + 16, s));
  CK(cudaMemcpyAsync(db, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(db + off_cnt, 0, 24 * (size_t)nseg, s));
  std::vector<uint32_t> seg_tile(nseg + 1);
  std::memcpy(seg_tile.data(), hb.data() + (uintptr_t)a.seg_tile, 4 * (nseg + 1));  // offsets before patch()
  patch(a, db);
  for (uint32_t g = 0; g < nseg; g++) {
    const uint32_t tiles = seg_tile[g + 1] - seg_tile[g];
    if (!seg_mode[g] || tiles == 0) continue;
    if (nbits) CK(cudaMemsetAsync(db + off_bits, 0, words * 4, s));
    k_card_count<<<std::min<uint32_t>(tiles, (uint32_t)sms() * 4), kT, 0, s>>>(
        a, g, nbits ? key_slot : -1, key_min, nbits, (uint32_t*)(db + off_bits),
        (unsigned long long*)(db + off_cnt) + 3 * g);
    alk::g_kernel_launches++;
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(h_counts, db + off_cnt, 24 * (size_t)nseg, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  if (!nbits)
    for (uint32_t g = 0; g < nseg; g++) h_counts[3 * g + 2] = ~0ull;
  return ALK_OK;
}

}  // extern "C"
