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

using namespace alkd;

namespace {
constexpr int kT = 256;
constexpr int kItems = 8;
constexpr int kTile = kT * kItems;
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
};

__device__ __forceinline__ bool ht_member(const HtView& h, int64_t k) {
  const uint64_t o = (uint64_t)k - (uint64_t)h.kmin;
  if (o >= h.nbits) return false;
  return (__ldg(h.bits + (o >> 5)) >> (o & 31)) & 1u;
}

__device__ __forceinline__ int64_t ht_probe(const HtView& h, int64_t k) {
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

// A row that survived a stage's scan: its position and its probe key. The scan kernels
// stream the columns every row needs and append survivors here; the hit kernel then
// does the per-row random work (hash probe, payload and aggregate-input loads, atomics)
// for all survivors in parallel, away from the scan's tile pipeline.
struct Hit {
  uint64_t pos;  // segment << 32 | row within the segment
  int64_t key;   // probe key (0 when the stage probes nothing)
};

struct StageArgs {
  const alk_colseg* cols;  // [ncols][nseg]
  uint32_t ncols, nseg;
  const uint8_t* seg_mode;
  const uint32_t* tile_seg;
  const uint32_t* tile_row0;
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
  Hit* hits;
  uint64_t hit_cap;
  unsigned long long* hit_count;
  int* err;
};

// Appends the thread's live items (rows base + k * kT of segment seg) to the hit list with
// one atomic per warp. Called by all 32 lanes; entries beyond hit_cap are counted but not
// written (the hit kernel then refuses the whole list).
__device__ __forceinline__ void emit_hits(const StageArgs& a, uint32_t live, uint32_t seg, uint64_t base,
                                          const int64_t (&key)[kItems]) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = __popc(live);
  uint32_t incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0) return;
  unsigned long long b = 0;
  if (lane == 31) b = atomicAdd(a.hit_count, (unsigned long long)total);
  b = __shfl_sync(0xffffffffu, b, 31);
  uint64_t p = b + incl - n;
#pragma unroll
  for (int k = 0; k < kItems; k++) {
    if (!((live >> k) & 1)) continue;
    if (p < a.hit_cap) a.hits[p] = Hit{(uint64_t)seg << 32 | (base + (uint64_t)k * kT), key[k]};
    p++;
  }
}

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
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    __syncthreads();
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
    const bool all = a.seg_mode[seg] == 1 || s_n == 0;
    const uint64_t base = (uint64_t)row0 + threadIdx.x;
    uint32_t live = 0;
    int64_t key[kItems];
#pragma unroll 1
    for (int k = 0; k < kItems; k++) {
      key[k] = 0;
      if (k * kT + threadIdx.x >= rows) continue;
      const uint64_t row = base + (uint64_t)k * kT;
      rows_seen++;
      auto col = [&](uint32_t slot) -> int64_t {
        const alk_colseg& d = s_desc[slot];
        return load_for(d.data, d.bits, d.lower, row);
      };
      if (!all && vm_eval<kT>(s_ins, s_n, s_res, s_consts, s_regs + threadIdx.x, col) == 0) continue;
      if (a.probe_slot >= 0) {
        key[k] = col((uint32_t)a.probe_slot);
        if (a.probe.bits && !ht_member(a.probe, key[k])) continue;
      }
      live |= 1u << k;
    }
    emit_hits(a, live, seg, base, key);
  }
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
}

// Per-survivor work of a stage, one thread per hit: the hash probe (for the payload
// position, or for membership when the probed table has no key bitmap), then either the
// build-side insert with its payload or the aggregate updates. A list that overflowed
// its capacity is refused as a whole (nothing is applied), so a rerun with a larger list
// starts from unchanged tables and accumulators.
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
  unsigned long long inserted = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const Hit h = a.hits[i];
    const uint32_t seg = (uint32_t)(h.pos >> 32);
    const uint64_t row = h.pos & 0xffffffffull;
    int64_t j = -1;
    if (a.probe_slot >= 0 && (a.need_slot || !a.probe.bits)) {
      j = ht_probe(a.probe, h.key);
      if (j < 0) continue;
    }
    auto col = [&](uint32_t slot) -> int64_t {
      if (slot >= 32) return __ldg(a.probe.payload + (uint64_t)(slot - 32) * a.probe.slot_cap + j);
      const alk_colseg* d = a.cols + (uint64_t)slot * a.nseg + seg;
      const void* data = (const void*)__ldg((const unsigned long long*)&d->data);
      return load_for(data, __ldg(&d->bits), (int64_t)__ldg((const long long*)&d->lower), row);
    };
    if (kBuild) {
      const int64_t sl = ht_insert(a.build, col((uint32_t)a.build_slot));
      if (sl < 0) continue;
      inserted++;
      for (uint32_t p = 0; p < a.build.npay; p++)
        a.build.payload[(uint64_t)p * a.build.slot_cap + sl] = col((uint32_t)a.pay_src[p]);
    } else {
      for (uint32_t g = 0; g < a.nagg; g++) {
        unsigned long long* dst = (unsigned long long*)(a.acc + (uint64_t)g * a.acc_stride + j);
        const uint8_t kind = a.agg_kind[g];
        if (kind == ALK_AGG_COUNT) {
          atomicAdd(dst, 1ull);
          continue;
        }
        const int64_t v =
            vm_eval<kT>(s_ins[1 + g], s_n[1 + g], s_res[1 + g], s_consts[1 + g], s_regs + threadIdx.x, col);
        if (kind == ALK_AGG_SUM) atomicAdd(dst, (unsigned long long)v);
        else if (kind == ALK_AGG_MIN) atomicMin((long long*)dst, (long long)v);
        else atomicMax((long long*)dst, (long long)v);
      }
      if (a.cnt) atomicAdd(a.cnt + j, 1ull);
    }
  }
  if (kBuild) {
    for (int o = 16; o; o >>= 1) inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
    if ((threadIdx.x & 31) == 0 && inserted) atomicAdd(a.build.nslots, inserted);
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
__global__ void __launch_bounds__(kT) k_topk_local16(const int64_t* rank, const unsigned long long* live, uint64_t n,
                                                     uint32_t k, int64_t* out) {
  __shared__ int64_t s_v[kT * kTopK];
  int64_t t[kTopK];
#pragma unroll
  for (int i = 0; i < kTopK; i++) t[i] = INT64_MIN;
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    if (!live[i]) continue;
    const int64_t v = rank[i];
    if (v <= t[kTopK - 1]) continue;
#pragma unroll
    for (int q = kTopK - 1; q > 0; q--) {  // insert into the descending list, dropping the smallest
      const int64_t up = t[q - 1];
      t[q] = v > up ? up : (v > t[q] ? v : t[q]);
    }
    t[0] = v > t[0] ? v : t[0];
  }
#pragma unroll
  for (int i = 0; i < kTopK; i++) s_v[threadIdx.x * kTopK + i] = t[i];
  __syncthreads();
  // bitonic sort of kT * kTopK values, descending
  constexpr int N = kT * kTopK;
  for (int size = 2; size <= N; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < N / 2; i += kT) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool desc = (lo & size) == 0;
        const int64_t a = s_v[lo], b = s_v[hi];
        if (desc ? a < b : a > b) {
          s_v[lo] = b;
          s_v[hi] = a;
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x < k) out[(uint64_t)blockIdx.x * k + threadIdx.x] = s_v[threadIdx.x];
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
constexpr int kMaxConj = 4;
struct Conj {
  int64_t mul, k;
  uint32_t slot, op;
};
struct FastArgs {
  StageArgs a;
  Conj conj[kMaxConj];
  uint32_t nconj;
};

__device__ __forceinline__ bool cmp_apply(uint32_t op, int64_t a, int64_t b) {
  switch (op) {
    case ALK_OP_LT: return a < b;
    case ALK_OP_GT: return a > b;
    case ALK_OP_LE: return a <= b;
    case ALK_OP_GE: return a >= b;
    case ALK_OP_EQ: return a == b;
    default: return a != b;
  }
}

// Values of one column for the thread's items (rows base + k * kT), live items only.
__device__ __forceinline__ void load_batch(const alk_colseg& d, uint64_t base, uint32_t live, int64_t (&v)[kItems]) {
  const uint64_t lo = (uint64_t)d.lower;
  switch (d.bits) {
    case 8: {
      const uint8_t* p = (const uint8_t*)d.data + base;
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if ((live >> k) & 1) v[k] = (int64_t)((uint64_t)__ldg(p + k * kT) + lo);
    } break;
    case 16: {
      const uint16_t* p = (const uint16_t*)d.data + base;
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if ((live >> k) & 1) v[k] = (int64_t)((uint64_t)__ldg(p + k * kT) + lo);
    } break;
    case 32: {
      const uint32_t* p = (const uint32_t*)d.data + base;
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if ((live >> k) & 1) v[k] = (int64_t)((uint64_t)__ldg(p + k * kT) + lo);
    } break;
    default: {
      const unsigned long long* p = (const unsigned long long*)d.data + base;
#pragma unroll
      for (int k = 0; k < kItems; k++)
        if ((live >> k) & 1) v[k] = (int64_t)((uint64_t)__ldg(p + k * kT) + lo);
    } break;
  }
}

__global__ void __launch_bounds__(kT) k_stage_fast(const __grid_constant__ FastArgs f) {
  const StageArgs& a = f.a;
  __shared__ alk_colseg s_desc[kMaxCols];
  unsigned long long rows_seen = 0;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    __syncthreads();
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
    const uint64_t base = (uint64_t)row0 + threadIdx.x;
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (k * kT + threadIdx.x < rows) live |= 1u << k;
    rows_seen += __popc(live);
    if (a.seg_mode[seg] != 1) {
      for (uint32_t c = 0; c < f.nconj; c++) {
        const Conj cj = f.conj[c];
        int64_t v[kItems];
        load_batch(s_desc[cj.slot], base, live, v);
#pragma unroll
        for (int k = 0; k < kItems; k++)
          if (((live >> k) & 1) && !cmp_apply(cj.op, wrap_mul(v[k], cj.mul), cj.k)) live &= ~(1u << k);
      }
    }
    int64_t key[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) key[k] = 0;
    if (live && a.probe_slot >= 0) {
      load_batch(s_desc[a.probe_slot], base, live, key);
      if (a.probe.bits) {
#pragma unroll
        for (int k = 0; k < kItems; k++)
          if (((live >> k) & 1) && !ht_member(a.probe, key[k])) live &= ~(1u << k);
      }
    }
    emit_hits(a, live, seg, base, key);
  }
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
}

// ---------------------------------------------------------------- TMA-staged stage
// The same stage with the columns every row needs (conjunct columns and the probe key)
// brought into shared memory by bulk asynchronous copies (cp.async.bulk, completion on an
// mbarrier), two tiles in flight per block: the copy engine keeps HBM busy while the
// block evaluates the previous tile. Columns read only for matching rows (payload,
// aggregate inputs) are read from global memory.
constexpr int kStaged = 6;          // staged columns at most
constexpr uint32_t kWaitLimit = 1u << 22;

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

struct TmaArgs {
  FastArgs f;
  uint32_t nstaged;
  uint32_t staged_slot[kStaged];  // scan slot of each staged column
  uint32_t stage_bytes;           // shared bytes of one stage (all staged columns, 2048 rows)
};

__global__ void __launch_bounds__(kT) k_stage_tma(const __grid_constant__ TmaArgs t) {
  const FastArgs& f = t.f;
  const StageArgs& a = f.a;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ alk_colseg s_desc[2][kMaxCols];
  __shared__ uint32_t s_off[2][kStaged];  // byte offset of each staged column in a stage buffer
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_abort;
  // probe key and conjunct columns -> staged index
  int probe_st = -1;
  int conj_st[kMaxConj];
  for (uint32_t c = 0; c < kMaxConj; c++) conj_st[c] = -1;
  for (uint32_t i = 0; i < t.nstaged; i++) {
    if (a.probe_slot >= 0 && t.staged_slot[i] == (uint32_t)a.probe_slot) probe_st = (int)i;
    for (uint32_t c = 0; c < f.nconj; c++)
      if (t.staged_slot[i] == f.conj[c].slot) conj_st[c] = (int)i;
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // issue the copies of this block's local tile number `it` into stage it & 1 (thread 0)
  auto issue = [&](uint32_t it) {
    const uint32_t tile = blockIdx.x + it * gridDim.x;
    if (tile >= a.ntiles) return;
    const uint32_t st = it & 1;
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    for (uint32_t c = 0; c < a.ncols; c++) s_desc[st][c] = a.cols[c * a.nseg + seg];
    const uint32_t rows = min((uint32_t)kTile, s_desc[st][0].rows - row0);
    uint32_t off = 0, total = 0;
    for (uint32_t i = 0; i < t.nstaged; i++) {
      const alk_colseg& d = s_desc[st][t.staged_slot[i]];
      const uint32_t w = d.bits / 8;
      const uint32_t bytes = (rows * w + 15) & ~15u;
      s_off[st][i] = off;
      off += (kTile * w + 127) & ~127u;
      total += bytes;
    }
    unsigned char* buf = s_dyn + st * t.stage_bytes;
    mbar_expect_tx(&s_bar[st], total);
    for (uint32_t i = 0; i < t.nstaged; i++) {
      const alk_colseg& d = s_desc[st][t.staged_slot[i]];
      const uint32_t w = d.bits / 8;
      const uint32_t bytes = (rows * w + 15) & ~15u;
      bulk_g2s(buf + s_off[st][i], (const unsigned char*)d.data + (uint64_t)row0 * w, bytes, &s_bar[st]);
    }
  };
  if (threadIdx.x == 0) {
    issue(0);
    issue(1);
  }
  __syncthreads();
  unsigned long long rows_seen = 0;
  uint32_t abort_it = 0;
  for (uint32_t it = 0;; it++) {
    const uint32_t tile = blockIdx.x + it * gridDim.x;
    if (tile >= a.ntiles) break;
    const uint32_t st = it & 1;
    // wait for this stage's copies (bounded)
    if (threadIdx.x == 0) {
      uint32_t spins = 0;
      while (!mbar_try_wait(&s_bar[st], (it >> 1) & 1)) {
        if (++spins > kWaitLimit) {
          atomicExch(a.err, ALK_ERR_TIMEOUT);
          s_abort = 1;
          break;
        }
        __nanosleep(32);
      }
    }
    __syncthreads();
    if (s_abort) {
      abort_it = it;
      break;
    }
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    const uint32_t rows = min((uint32_t)kTile, s_desc[st][0].rows - row0);
    const unsigned char* buf = s_dyn + st * t.stage_bytes;
    auto staged = [&](int i, uint32_t r) -> int64_t {
      const alk_colseg& d = s_desc[st][t.staged_slot[i]];
      const unsigned char* p = buf + s_off[st][i];
      uint64_t x;
      switch (d.bits) {
        case 8: x = p[r]; break;
        case 16: x = ((const uint16_t*)p)[r]; break;
        case 32: x = ((const uint32_t*)p)[r]; break;
        default: x = ((const unsigned long long*)p)[r]; break;
      }
      return (int64_t)(x + (uint64_t)d.lower);
    };
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (k * kT + threadIdx.x < rows) live |= 1u << k;
    rows_seen += __popc(live);
    if (a.seg_mode[seg] != 1) {
      for (uint32_t c = 0; c < f.nconj; c++) {
        const Conj cj = f.conj[c];
#pragma unroll
        for (int k = 0; k < kItems; k++)
          if (((live >> k) & 1) &&
              !cmp_apply(cj.op, wrap_mul(staged(conj_st[c], k * kT + threadIdx.x), cj.mul), cj.k))
            live &= ~(1u << k);
      }
    }
    int64_t key[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) key[k] = 0;
    if (live && probe_st >= 0) {
#pragma unroll
      for (int k = 0; k < kItems; k++) {
        if (!((live >> k) & 1)) continue;
        key[k] = staged(probe_st, k * kT + threadIdx.x);
        if (a.probe.bits && !ht_member(a.probe, key[k])) live &= ~(1u << k);
      }
    }
    emit_hits(a, live, seg, (uint64_t)row0 + threadIdx.x, key);
    // every thread is done with this stage: refill it with the tile two ahead
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(it + 2);
    }
  }
  // an aborted block waits (bounded) for the copies still in flight (local tiles abort_it
  // and abort_it + 1) before it exits
  if (s_abort && threadIdx.x == 0) {
    for (uint32_t it = abort_it; it < abort_it + 2; it++) {
      if (blockIdx.x + it * gridDim.x >= a.ntiles) break;
      for (uint32_t spins = 0; spins < kWaitLimit && !mbar_try_wait(&s_bar[it & 1], (it >> 1) & 1); spins++)
        __nanosleep(32);
    }
  }
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
}

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

// Static shared memory of k_stage_tma (descriptors, barriers) next to the two dynamic
// stage buffers; the SM offers 227 KB per block.
constexpr size_t kTmaStaticSmem = 2 * 1024;
constexpr size_t kSmemPerBlock = 227 * 1024;

// Launch a stage as two kernels on one stream: the scan (the TMA-staged kernel when the
// predicate is a conjunction and the staged columns fit in shared memory, else the
// conjunctive kernel with direct loads, else the register-machine kernel), then the hit
// kernel over its survivors. cols is the host descriptor array [ncols][nseg].
template <bool kBuild>
cudaError_t launch_stage(const StageArgs& a, const alk_program& pred, const alk_colseg* cols,
                         const uint8_t* seg_mode, cudaStream_t s, alk_event_timer* timer) {
  if (!a.ntiles) return cudaSuccess;
  FastArgs fa;
  fa.a = a;
  const bool conj = as_conjuncts(pred, fa.conj, &fa.nconj);
  TmaArgs t{};
  bool tma = false;
  if (conj) {
    t.f = fa;
    std::vector<uint32_t> st;
    auto add = [&](uint32_t sl) {
      if (std::find(st.begin(), st.end(), sl) == st.end()) st.push_back(sl);
    };
    for (uint32_t c = 0; c < fa.nconj; c++) add(fa.conj[c].slot);
    if (a.probe_slot >= 0) add((uint32_t)a.probe_slot);
    uint32_t bytes = 0;
    for (uint32_t sl : st) {
      uint32_t w = 1;
      for (uint32_t g = 0; g < a.nseg; g++)
        if (seg_mode[g]) w = std::max<uint32_t>(w, cols[sl * a.nseg + g].bits / 8);
      bytes += (kTile * w + 127) & ~127u;
    }
    if (!st.empty() && st.size() <= (size_t)kStaged && kTmaStaticSmem + 2 * (size_t)bytes <= kSmemPerBlock) {
      t.nstaged = (uint32_t)st.size();
      for (size_t i = 0; i < st.size(); i++) t.staged_slot[i] = st[i];
      t.stage_bytes = bytes;
      tma = true;
    }
  }
  int occ = 0;
  if (tma) {
    cudaFuncSetAttribute(k_stage_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * t.stage_bytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_tma, kT, 2 * t.stage_bytes);
  } else if (conj) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_fast, kT, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_scan, kT, 0);
  }
  const int grid = std::min<int>((int)a.ntiles, sms() * std::max(occ, 1));
  int occ_hits = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_hits, k_stage_hits<kBuild>, kT, 0);
  if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev0, s);
  if (tma) k_stage_tma<<<grid, kT, 2 * t.stage_bytes, s>>>(t);
  else if (conj) k_stage_fast<<<grid, kT, 0, s>>>(fa);
  else k_stage_scan<<<grid, kT, 0, s>>>(a);
  k_stage_hits<kBuild><<<sms() * std::max(occ_hits, 1), kT, 0, s>>>(a);
  if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev1, s);
  alk::g_kernel_launches += 2;
  return cudaGetLastError();
}

bool prog_ok(const alk_program& p, uint32_t ncols, uint32_t npay) {
  if (p.n_instr > ALK_MAX_INSTR || p.result >= ALK_MAX_REGS) return false;
  for (uint32_t i = 0; i < p.n_instr; i++) {
    const alk_instr& in = p.ins[i];
    if (in.dst >= ALK_MAX_REGS || in.op < ALK_OP_ADD || in.op > ALK_OP_MOV) return false;
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
  // exact key bitmap when the key range is at most 2^29 values (64 MB)
  uint64_t nbits = 0;
  if (key_max >= key_min) {
    uint64_t span = (uint64_t)key_max - (uint64_t)key_min + 1;
    if (span != 0 && span <= (1ull << 29)) nbits = span;
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

const int64_t* alk_ht_payload(const alk_ht* h, uint32_t p) {
  if (!h || p >= h->v.npay) return nullptr;
  return h->v.payload + (uint64_t)p * h->v.slot_cap;
}

static int stage_common(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                        const alk_program* progs, uint32_t nprogs, std::vector<uint8_t>& hb, StageArgs& a,
                        size_t extra_bytes, size_t* off_extra) {
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
  a.ntiles = (uint32_t)tseg.size();
  size_t off_cols = 0;
  size_t off_mode = off_cols + sizeof(alk_colseg) * ncols * nseg;
  size_t off_tseg = (off_mode + nseg + 15) & ~size_t(15);
  size_t off_trow = off_tseg + 4 * tseg.size();
  size_t off_prog = (off_trow + 4 * trow.size() + 15) & ~size_t(15);
  size_t off_x = (off_prog + sizeof(alk_program) * nprogs + 15) & ~size_t(15);
  hb.assign(off_x + extra_bytes + 16, 0);
  std::memcpy(&hb[off_cols], cols, sizeof(alk_colseg) * ncols * nseg);
  std::memcpy(&hb[off_mode], seg_mode, nseg);
  if (!tseg.empty()) {
    std::memcpy(&hb[off_tseg], tseg.data(), 4 * tseg.size());
    std::memcpy(&hb[off_trow], trow.data(), 4 * trow.size());
  }
  std::memcpy(&hb[off_prog], progs, sizeof(alk_program) * nprogs);
  a.ncols = ncols;
  a.nseg = nseg;
  a.nprogs = nprogs;
  *off_extra = off_x;
  // device offsets are patched by the caller once the buffer exists
  a.cols = (const alk_colseg*)(uintptr_t)off_cols;
  a.seg_mode = (const uint8_t*)(uintptr_t)off_mode;
  a.tile_seg = (const uint32_t*)(uintptr_t)off_tseg;
  a.tile_row0 = (const uint32_t*)(uintptr_t)off_trow;
  a.progs = (const alk_program*)(uintptr_t)off_prog;
  return ALK_OK;
}

static void patch(StageArgs& a, uint8_t* db) {
  a.cols = (const alk_colseg*)(db + (uintptr_t)a.cols);
  a.seg_mode = db + (uintptr_t)a.seg_mode;
  a.tile_seg = (const uint32_t*)(db + (uintptr_t)a.tile_seg);
  a.tile_row0 = (const uint32_t*)(db + (uintptr_t)a.tile_row0);
  a.progs = (const alk_program*)(db + (uintptr_t)a.progs);
}

// Uploads a stage's arguments with its counters and hit list in one stream-ordered
// allocation, runs scan + hit kernels, reads the counters back (one synchronisation).
// hit_cap 0 (or above the rows scanned) means the rows scanned, which cannot overflow.
}  // extern "C"
template <bool kBuild>
static int run_stage(StageArgs& a, const alk_program& pred, const alk_colseg* cols, const uint8_t* seg_mode,
                     const std::vector<uint8_t>& hb, size_t off_x, uint64_t hit_cap, uint64_t* h_rows_in,
                     uint64_t* h_hits, cudaStream_t s, alk_event_timer* timer) {
  uint64_t upper = 0;
  for (uint32_t g = 0; g < a.nseg; g++)
    if (seg_mode[g]) upper += cols[g].rows;
  if (hit_cap == 0 || hit_cap > upper) hit_cap = upper;
  const size_t off_tail = (hb.size() + 15) & ~size_t(15);
  const size_t off_hits = off_tail + 32;
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, off_hits + std::max<uint64_t>(hit_cap, 1) * sizeof(Hit), s));
  CK(cudaMemcpyAsync(db, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  uint8_t* tail = db + off_tail;
  CK(cudaMemsetAsync(tail, 0, 32, s));
  patch(a, db);
  if (kBuild) a.pay_src = (const int32_t*)(db + off_x);
  else a.agg_kind = db + off_x;
  a.rows_in = (unsigned long long*)tail;
  a.hit_count = (unsigned long long*)(tail + 8);
  a.err = (int*)(tail + 16);
  a.hits = (Hit*)(db + off_hits);
  a.hit_cap = hit_cap;
  CK(launch_stage<kBuild>(a, pred, cols, seg_mode, s, timer));
  unsigned long long back[3] = {0, 0, 0};
  CK(cudaMemcpyAsync(back, tail, 24, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  if (timer && timer->on && a.ntiles) {
    float ms = 0;
    cudaEventElapsedTime(&ms, (cudaEvent_t)timer->ev0, (cudaEvent_t)timer->ev1);
    timer->ms += ms;
    timer->launches++;
  }
  if (h_rows_in) *h_rows_in = back[0];
  if (h_hits) *h_hits = back[1];
  return (int)(uint32_t)back[2];
}
extern "C" {

int alk_pipeline_build(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                       const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                       int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap, uint64_t* h_rows_in,
                       uint64_t* h_hits, alk_stream stream) {
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
  std::memcpy(&hb[off_x], pay_src, 4 * build->v.npay);
  a.probe_slot = probe_slot;
  if (probe) a.probe = probe->v;
  a.build_slot = build_slot;
  a.build = build->v;
  for (uint32_t p = 0; p < build->v.npay; p++)
    if (pay_src[p] >= 32) a.need_slot = 1;
  return run_stage<true>(a, prog, cols, seg_mode, hb, off_x, hit_cap, h_rows_in, h_hits, s, nullptr);
}

int alk_pipeline_probe_agg(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                           const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                           const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, int64_t* d_acc,
                           uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap, uint64_t* h_rows_in,
                           uint64_t* h_hits, alk_stream stream, alk_event_timer* timer) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!probe || probe_slot < 0 || (uint32_t)probe_slot >= ncols || ncols == 0 || ncols > kMaxCols || nagg > 7)
    return ALK_ERR_ARG;
  if (acc_stride < probe->v.slot_cap) return ALK_ERR_ARG;  // accumulators indexed by table position

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
  return run_stage<false>(a, progs[0], cols, seg_mode, hb, off_x, hit_cap, h_rows_in, h_hits, s, timer);
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
