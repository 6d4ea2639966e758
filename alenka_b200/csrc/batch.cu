// Batched filter + group-by: many queries of the single-table FILTER -> SELECT ... GROUP BY
// shape (the reference runs each as emit_filter + emit_select, operators.cu:2306 and
// :1801, one query at a time) in one persistent launch over a work list of (query,
// segment) items. Each block takes a contiguous range of the list's tiles, so it meets
// few query boundaries. One producer warp stages a tile's columns into shared memory with
// bulk copies; consumer warps evaluate the query's conjuncts on the stored values, form
// the group slot from small-domain key columns (dense: slot = sum (key - min) * stride)
// and fold each aggregate input, a product of two affine column terms, into accumulators
// private to each thread. A warp folds its lanes' accumulators into the query's global
// accumulators when it moves to another query and at the end.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"
#include "scan.cuh"

namespace {
constexpr int kGbCols = 8;
constexpr int kGbAggs = 8;
constexpr uint32_t kGbMaxStages = 4;

struct GbQuery {
  uint32_t ncols, nconj, nkeys, nagg;
  Conj conj[kMaxConj];  // slot: the query's column index
  int32_t key_col[2];
  int64_t key_min[2];
  uint64_t key_mul[2];
  uint64_t key_span[2];
  uint32_t nslots, nacc;  // nacc = nagg + 1: the row count is the last accumulator
  int32_t count_agg;      // an aggregate that is COUNT (it doubles as the row count), or -1
  uint32_t npriv;         // private words per slot: nagg with a COUNT aggregate, else nacc
  alk_gb_agg agg[kGbAggs];
  int64_t* acc;  // [nacc][nslots]
};
struct GbItem {
  uint32_t query, mode, rows, pad;
  alk_colseg col[kGbCols];
  ConjSeg cs[kMaxConj];
};
struct GbArgs {
  const GbItem* items;
  const uint32_t* item_tile;  // [nitems + 1]: item i owns tiles [item_tile[i], item_tile[i + 1])
  uint32_t nitems, ntiles;
  const GbQuery* queries;
  uint32_t nst, stage_bytes;  // stages in flight, bytes of one stage
  uint32_t cw;                // consumer warps; a tile is cw * 256 rows
  uint32_t max_acc;           // private accumulators per thread: (slots + 1) x (aggregates + 1)
  unsigned long long* item_rows;  // survivors per item
  int* err;
};

__device__ __forceinline__ uint32_t find_item(const uint32_t* item_tile, uint32_t n, uint32_t tile) {
  uint32_t lo = 0, hi = n;  // item_tile[lo] <= tile < item_tile[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(item_tile + mid) <= tile) lo = mid;
    else hi = mid;
  }
  return lo;
}

// A warp folds its lanes' private accumulators (slot-major, [acc][lane]) into the
// query's global accumulators and clears them.
__device__ void gb_flush(const GbQuery& q, int64_t* priv, uint32_t lane) {
  for (uint32_t j = 0; j < q.nslots * q.nacc; j++) {
    const uint32_t a = j % q.nacc, slot = j / q.nacc;
    const uint32_t kind = a < q.nagg ? q.agg[a].kind : (uint32_t)ALK_AGG_COUNT;
    // a query with a COUNT aggregate keeps no separate row count: it is that aggregate
    const uint32_t w = (a == q.nagg && q.count_agg >= 0) ? (uint32_t)q.count_agg : a;
    int64_t v = priv[(slot * q.npriv + w) * 32 + lane];  // gb_clear resets them for the next query
    for (int o = 16; o; o >>= 1) {
      const int64_t w = __shfl_xor_sync(0xffffffffu, v, o);
      v = kind == ALK_AGG_MIN ? min(v, w) : kind == ALK_AGG_MAX ? max(v, w) : (int64_t)((uint64_t)v + (uint64_t)w);
    }
    if (lane == 0) {
      int64_t* dst = q.acc + (size_t)a * q.nslots + slot;
      if (kind == ALK_AGG_MIN) {
        if (v != INT64_MAX) atomicMin((long long*)dst, (long long)v);
      } else if (kind == ALK_AGG_MAX) {
        if (v != INT64_MIN) atomicMax((long long*)dst, (long long)v);
      } else if (v) {
        atomicAdd((unsigned long long*)dst, (unsigned long long)v);
      }
    }
  }
}

__device__ __forceinline__ void gb_clear(const GbQuery& q, int64_t* priv, uint32_t lane) {
  for (uint32_t j = 0; j < q.nslots * q.npriv; j++) {
    const uint32_t a = j % q.npriv;
    const uint32_t kind = a < q.nagg ? q.agg[a].kind : (uint32_t)ALK_AGG_COUNT;
    priv[j * 32 + lane] = kind == ALK_AGG_MIN ? INT64_MAX : kind == ALK_AGG_MAX ? INT64_MIN : 0;
  }
}

__global__ void k_gb_tma(const __grid_constant__ GbArgs g) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ __align__(8) uint64_t s_full[kGbMaxStages], s_empty[kGbMaxStages];
  __shared__ uint32_t s_item[kGbMaxStages];           // item of the tile in each stage
  __shared__ uint32_t s_rows[kGbMaxStages];           // its rows
  __shared__ uint32_t s_coff[kGbMaxStages][kGbCols];  // its staged column offsets
  __shared__ int s_abort;
  const uint32_t nst = g.nst, cw = g.cw;
  const uint32_t tile_rows = cw * 32 * kItems;
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (uint32_t i = 0; i < nst; i++) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], cw);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int* abort_flag = &s_abort;
  // this block's contiguous range of the work list's tiles
  const uint32_t t0 = (uint32_t)((uint64_t)blockIdx.x * g.ntiles / gridDim.x);
  const uint32_t t1 = (uint32_t)((uint64_t)(blockIdx.x + 1) * g.ntiles / gridDim.x);

  if (warp == cw) {
    // ---- producer: one thread issues the bulk copies
    if (lane != 0) return;
    uint32_t issued = 0;
    // the block's tiles are contiguous: the item is found once and then advanced, with
    // its copy sources kept in registers; each stage carries the tile's item, rows and
    // column offsets for the consumers
    uint32_t i = t0 < t1 ? find_item(g.item_tile, g.nitems, t0) : 0;
    uint32_t first = 0, next = 0, irows = 0, ncols = 0;
    const unsigned char* src[kGbCols];
    uint32_t width[kGbCols];
    auto load_item = [&]() {
      first = __ldg(g.item_tile + i);
      next = __ldg(g.item_tile + i + 1);
      const GbItem& item = g.items[i];
      irows = item.rows;
      ncols = g.queries[item.query].ncols;
#pragma unroll
      for (int c = 0; c < kGbCols; c++) {
        src[c] = c < (int)ncols ? (const unsigned char*)item.col[c].data : nullptr;
        width[c] = c < (int)ncols ? item.col[c].bits / 8 : 0;
      }
    };
    if (t0 < t1) load_item();
    for (uint32_t it = 0; t0 + it < t1; it++) {
      if (*abort_flag) break;
      const uint32_t tile = t0 + it, st = it % nst;
      if (it >= nst && !mbar_wait(&s_empty[st], (it / nst - 1) & 1)) {
        atomicExch(g.err, ALK_ERR_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      while (tile >= next && i + 1 < g.nitems) {
        i++;
        load_item();
      }
      const uint32_t row0 = (tile - first) * tile_rows;
      const uint32_t rows = min(tile_rows, irows - row0);
      s_item[st] = i;
      s_rows[st] = rows;
      uint32_t total = 0;
#pragma unroll
      for (int c = 0; c < kGbCols; c++) {
        s_coff[st][c] = total;
        total += (rows * width[c] + 15) & ~15u;
      }
      unsigned char* buf = s_dyn + (size_t)st * g.stage_bytes;
      mbar_expect_tx(&s_full[st], total);
#pragma unroll
      for (int c = 0; c < kGbCols; c++) {
        if (c >= (int)ncols) break;
        const uint32_t n = (rows * width[c] + 15) & ~15u;
        bulk_g2s(buf + s_coff[st][c], src[c] + (uint64_t)row0 * width[c], n, &s_full[st]);
      }
      issued = it + 1;
    }
    for (uint32_t it = issued > nst ? issued - nst : 0; it < issued; it++)
      mbar_wait(&s_full[it % nst], (it / nst) & 1);
    return;
  }

  // ---- consumers: warp `warp` owns rows warp * 256 + k * 32 + lane of every tile
  int64_t* priv = (int64_t*)(s_dyn + (size_t)nst * g.stage_bytes) + (size_t)warp * g.max_acc * 32;
  // the warp's copies of its current query and item descriptors
  GbQuery& q = ((GbQuery*)(s_dyn + (size_t)nst * g.stage_bytes + (size_t)cw * g.max_acc * 32 * 8))[warp];
  GbItem& item = ((GbItem*)((unsigned char*)(&q - warp) + sizeof(GbQuery) * cw))[warp];
  uint32_t cur_q = 0xffffffffu, cur_item = 0xffffffffu;
  unsigned long long surv = 0;  // survivors of cur_item seen by this warp (warp-uniform)
  const uint32_t r0 = warp * (32 * kItems) + lane;
  for (uint32_t it = 0; t0 + it < t1; it++) {
    if (__any_sync(0xffffffffu, *abort_flag)) break;
    const uint32_t st = it % nst;
    if (!mbar_wait_warp(&s_full[st], (it / nst) & 1)) {
      if (lane == 0) {
        atomicExch(g.err, ALK_ERR_TIMEOUT);
        *abort_flag = 1;
      }
      break;
    }
    const uint32_t i = s_item[st];
    if (i != cur_item) {
      if (cur_item != 0xffffffffu && lane == 0 && surv) atomicAdd(g.item_rows + cur_item, surv);
      surv = 0;
      cur_item = i;
      __syncwarp();
      for (uint32_t w = lane; w < sizeof(GbItem) / 4; w += 32) ((uint32_t*)&item)[w] = ((const uint32_t*)(g.items + i))[w];
      __syncwarp();
      const uint32_t qi = item.query;
      if (qi != cur_q) {
        if (cur_q != 0xffffffffu) gb_flush(q, priv, lane);
        __syncwarp();
        for (uint32_t w = lane; w < sizeof(GbQuery) / 4; w += 32)
          ((uint32_t*)&q)[w] = ((const uint32_t*)(g.queries + qi))[w];
        __syncwarp();
        gb_clear(q, priv, lane);
        cur_q = qi;
      }
    }
    const uint32_t rows = s_rows[st];
    const unsigned char* buf = s_dyn + (size_t)st * g.stage_bytes;
    const uint32_t* coff = s_coff[st];  // staged column offsets of this tile
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
      if (r0 + k * 32 < rows) live |= 1u << k;
    if (item.mode != 1) {
      for (uint32_t c = 0; c < q.nconj && live; c++) {
        const uint32_t col = q.conj[c].slot;
        const alk_colseg& d = item.col[col];
        if (d.bits <= 32) {
          uint32_t x[kItems];
          load_raw32<32>(buf + coff[col], d.bits, r0, x);
          live = conj_filter32(q.conj[c], item.cs[c], d.lower, x, live);
        } else {
          uint64_t x[kItems];
          load_raw<false, 32>(buf + coff[col], d.bits, r0, live, x);
          live = conj_filter(q.conj[c], item.cs[c], d.lower, x, live);
        }
      }
    }
    surv += __reduce_add_sync(0xffffffffu, (unsigned)__popc(live));
    // fold the survivors a column at a time over the thread's 8 rows: the group slot in
    // 32-bit arithmetic (stored key + (segment base - key minimum), each below its span),
    // then every aggregate input into the slot's accumulators, private to the lane
    if (__any_sync(0xffffffffu, live)) {
      uint32_t slot[kItems];
#pragma unroll
      for (int k = 0; k < kItems; k++) slot[k] = 0;
      for (uint32_t j = 0; j < q.nkeys; j++) {
        const alk_colseg& d = item.col[q.key_col[j]];
        const uint32_t kd = (uint32_t)((uint64_t)d.lower - (uint64_t)q.key_min[j]);
        const uint32_t span = (uint32_t)q.key_span[j], mul = (uint32_t)q.key_mul[j];
        uint32_t x[kItems];
        if (d.bits > 32) {  // the low word suffices: the offset from the minimum is below the span
          uint64_t w[kItems];
          load_raw<false, 32>(buf + coff[q.key_col[j]], d.bits, r0, live, w);
#pragma unroll
          for (int k = 0; k < kItems; k++) x[k] = (uint32_t)w[k];
        } else {
          load_raw32<32>(buf + coff[q.key_col[j]], d.bits, r0, x);
        }
        uint32_t bad = 0;
#pragma unroll
        for (int k = 0; k < kItems; k++) {
          const uint32_t o = x[k] + kd;
          bad |= (o >= span ? 1u : 0u) << k;
          slot[k] += o * mul;
        }
        bad &= live;
        if (bad) {  // a key outside the zone maps' range: the plan is wrong
          atomicExch(g.err, ALK_ERR_ARG);
          live &= ~bad;
        }
      }
      const uint32_t nagg = q.nagg, stride = q.npriv * 32;
      int64_t* base = priv + lane;
      // rows that did not pass update the spare slot (index nslots): no branch per row
#pragma unroll
      for (int k = 0; k < kItems; k++) slot[k] = ((live >> k) & 1) ? slot[k] * stride : q.nslots * stride;
      for (uint32_t a = 0; a < nagg; a++) {
        const uint32_t kind = q.agg[a].kind;
        int64_t* pa = base + a * 32;
        if (kind == ALK_AGG_COUNT) {
#pragma unroll
          for (int k = 0; k < kItems; k++) pa[slot[k]] += 1;
          continue;
        }
        const int32_t ca = q.agg[a].a, cb = q.agg[a].b;
        const uint64_t am = (uint64_t)q.agg[a].am, ac = (uint64_t)q.agg[a].ac;
        const uint64_t la = (uint64_t)item.col[ca].lower;
        uint64_t v[kItems];
        load_raw<false, 32>(buf + coff[ca], item.col[ca].bits, r0, live, v);
        if (am == 1 && ac == 0) {
#pragma unroll
          for (int k = 0; k < kItems; k++) v[k] += la;
        } else {
#pragma unroll
          for (int k = 0; k < kItems; k++) v[k] = (v[k] + la) * am + ac;
        }
        if (cb >= 0) {
          const uint64_t bm = (uint64_t)q.agg[a].bm, bc = (uint64_t)q.agg[a].bc;
          const uint64_t lb = (uint64_t)item.col[cb].lower;
          uint64_t w[kItems];
          load_raw<false, 32>(buf + coff[cb], item.col[cb].bits, r0, live, w);
#pragma unroll
          for (int k = 0; k < kItems; k++) v[k] *= (w[k] + lb) * bm + bc;
        }
        if (kind == ALK_AGG_MIN) {
#pragma unroll
          for (int k = 0; k < kItems; k++) pa[slot[k]] = min(pa[slot[k]], (int64_t)v[k]);
        } else if (kind == ALK_AGG_MAX) {
#pragma unroll
          for (int k = 0; k < kItems; k++) pa[slot[k]] = max(pa[slot[k]], (int64_t)v[k]);
        } else {
#pragma unroll
          for (int k = 0; k < kItems; k++) pa[slot[k]] = (int64_t)((uint64_t)pa[slot[k]] + v[k]);
        }
      }
      if (q.count_agg < 0) {
        int64_t* pc = base + nagg * 32;
#pragma unroll
        for (int k = 0; k < kItems; k++) pc[slot[k]] += 1;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&s_empty[st]);
  }
  if (cur_q != 0xffffffffu) gb_flush(q, priv, lane);
  if (cur_item != 0xffffffffu && lane == 0 && surv) atomicAdd(g.item_rows + cur_item, surv);
}

// Every query's accumulators [nacc][nslots] at the identity of their aggregate: one
// launch for the batch, query blockIdx.y.
__global__ void k_gb_init(const GbQuery* queries) {
  const GbQuery& q = queries[blockIdx.y];
  const uint32_t n = q.nslots * q.nacc;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t a = i / q.nslots;
    const uint32_t k = a < q.nagg ? q.agg[a].kind : (uint32_t)ALK_AGG_COUNT;
    q.acc[i] = k == ALK_AGG_MIN ? INT64_MAX : k == ALK_AGG_MAX ? INT64_MIN : 0;
  }
}

int sms_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}
}  // namespace

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

extern "C" {

int alk_batch_groupby(const alk_gb_query* qs, uint32_t nq, const alk_gb_tuning* tune, alk_gb_tuning* used,
                      alk_event_timer* timer, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!qs || nq == 0) return ALK_ERR_ARG;
  std::vector<GbQuery> hq(nq);
  std::vector<GbItem> items;
  std::vector<uint32_t> item_tile;
  std::vector<std::pair<uint32_t, uint32_t>> item_src;  // (query, segment) of each item
  uint32_t max_acc = 1, max_stage = 16;
  const uint32_t cw = tune && tune->consumer_warps ? tune->consumer_warps : 8;
  if (cw != 4 && cw != 8) return ALK_ERR_ARG;
  const uint32_t tile_rows = cw * 32 * kItems;
  uint64_t ntiles = 0;
  for (uint32_t qi = 0; qi < nq; qi++) {
    const alk_gb_query& a = qs[qi];
    GbQuery& q = hq[qi];
    std::memset(&q, 0, sizeof(q));
    if (a.ncols == 0 || a.ncols > kGbCols || a.nkeys > 2 || a.nagg > kGbAggs || !a.cols || !a.d_acc) return ALK_ERR_ARG;
    q.ncols = a.ncols;
    q.nkeys = a.nkeys;
    q.nagg = a.nagg;
    uint64_t nslots = 1;
    for (int j = (int)a.nkeys - 1; j >= 0; j--) {
      if (a.key_col[j] < 0 || (uint32_t)a.key_col[j] >= a.ncols || a.key_max[j] < a.key_min[j]) return ALK_ERR_ARG;
      const uint64_t span = (uint64_t)a.key_max[j] - (uint64_t)a.key_min[j] + 1;
      if (span == 0 || span > 4096) return ALK_ERR_UNSUPPORTED;
      q.key_col[j] = a.key_col[j];
      q.key_min[j] = a.key_min[j];
      q.key_span[j] = span;
      q.key_mul[j] = nslots;
      nslots *= span;
    }
    q.nslots = (uint32_t)nslots;
    q.nacc = a.nagg + 1;
    q.count_agg = -1;
    for (uint32_t k = 0; k < a.nagg; k++)
      if (a.agg[k].kind == ALK_AGG_COUNT && q.count_agg < 0) q.count_agg = (int32_t)k;
    if (nslots * q.nacc > 64) return ALK_ERR_UNSUPPORTED;  // private accumulators per thread
    // one more slot per lane takes the updates of rows that did not pass, so that the
    // updates need no branch
    q.npriv = q.count_agg >= 0 ? a.nagg : q.nacc;
    max_acc = std::max<uint32_t>(max_acc, (uint32_t)((nslots + 1) * q.npriv));
    for (uint32_t k = 0; k < a.nagg; k++) {
      const alk_gb_agg& ag = a.agg[k];
      if (ag.kind > ALK_AGG_MAX) return ALK_ERR_ARG;
      if (ag.kind != ALK_AGG_COUNT && (ag.a < 0 || (uint32_t)ag.a >= a.ncols || ag.b >= (int32_t)a.ncols))
        return ALK_ERR_ARG;
      q.agg[k] = ag;
    }
    q.acc = a.d_acc;
    // the filter as conjuncts on the query's columns
    alk_program prog{};
    if (a.pred) prog = *a.pred;
    std::vector<alk::CardConj> cj;
    if (!alk::program_conjuncts(prog, cj) || cj.size() > (size_t)kMaxConj) return ALK_ERR_UNSUPPORTED;
    q.nconj = (uint32_t)cj.size();
    for (uint32_t c = 0; c < q.nconj; c++) {
      if (cj[c].slot >= a.ncols) return ALK_ERR_ARG;
      q.conj[c] = Conj{cj[c].mul, cj[c].k, cj[c].slot, cj[c].op};
    }
    // work items: the scanned segments
    for (uint32_t gi = 0; gi < a.nseg; gi++) {
      const uint8_t mode = a.seg_mode ? a.seg_mode[gi] : 2;
      if (mode == 0) continue;
      GbItem it;
      std::memset(&it, 0, sizeof(it));
      it.query = qi;
      it.mode = mode;
      it.rows = a.cols[gi].rows;
      uint32_t stage = 0;
      for (uint32_t c = 0; c < a.ncols; c++) {
        const alk_colseg& d = a.cols[(size_t)c * a.nseg + gi];
        if (d.rows != it.rows || !(d.bits == 8 || d.bits == 16 || d.bits == 32 || d.bits == 64)) return ALK_ERR_ARG;
        if (d.rows && (!d.data || ((uintptr_t)d.data & 15))) return ALK_ERR_ARG;  // bulk copies: 16-byte aligned
        it.col[c] = d;
        stage += (tile_rows * (d.bits / 8) + 15) & ~15u;
      }
      for (uint32_t c = 0; c < q.nconj; c++) it.cs[c] = conj_seg(q.conj[c], it.col[q.conj[c].slot]);
      if (it.rows == 0) continue;
      item_src.push_back({qi, gi});
      max_stage = std::max(max_stage, stage);
      item_tile.push_back((uint32_t)ntiles);
      ntiles += (it.rows + tile_rows - 1) / tile_rows;
      items.push_back(it);
    }
  }
  if (ntiles >= 0xffffffffull) return ALK_ERR_TOO_LARGE;
  item_tile.push_back((uint32_t)ntiles);
  const uint32_t nitems = (uint32_t)items.size();
  // device copies: queries, items, item tiles, item survivor counts, error flag
  const size_t o_q = 0;
  const size_t o_items = (o_q + sizeof(GbQuery) * nq + 255) & ~size_t(255);
  const size_t o_tile = (o_items + sizeof(GbItem) * nitems + 255) & ~size_t(255);
  const size_t o_rows = (o_tile + 4 * item_tile.size() + 255) & ~size_t(255);
  const size_t o_err = o_rows + 8 * (size_t)std::max<uint32_t>(nitems, 1);
  const size_t bytes = o_err + 16;
  std::vector<uint8_t> hb(o_rows, 0);
  std::memcpy(&hb[o_q], hq.data(), sizeof(GbQuery) * nq);
  if (nitems) std::memcpy(&hb[o_items], items.data(), sizeof(GbItem) * nitems);
  std::memcpy(&hb[o_tile], item_tile.data(), 4 * item_tile.size());
  uint8_t* db = nullptr;
  CK(cudaMallocAsync((void**)&db, bytes, s));
  cudaError_t ue;
  const void* src = alk::upload_source(hb.data(), hb.size(), s, &ue);
  CK(ue);
  CK(cudaMemcpyAsync(db, src, hb.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(db + o_rows, 0, bytes - o_rows, s));
  // accumulators: every query's [nacc][nslots] starts at the identity of its aggregate
  {
    uint32_t most = 1;
    for (uint32_t qi = 0; qi < nq; qi++) most = std::max(most, hq[qi].nslots * hq[qi].nacc);
    k_gb_init<<<dim3((most + 255) / 256, nq), 256, 0, s>>>((const GbQuery*)(db + o_q));
    alk::g_kernel_launches++;
    CK(cudaGetLastError());
  }
  GbArgs g{};
  g.items = (const GbItem*)(db + o_items);
  g.item_tile = (const uint32_t*)(db + o_tile);
  g.nitems = nitems;
  g.ntiles = (uint32_t)ntiles;
  g.queries = (const GbQuery*)(db + o_q);
  g.nst = tune && tune->stages ? std::min<uint32_t>(tune->stages, kGbMaxStages) : 3;
  g.cw = cw;
  g.stage_bytes = (max_stage + 127) & ~127u;
  g.max_acc = max_acc;
  g.item_rows = (unsigned long long*)(db + o_rows);
  g.err = (int*)(db + o_err);
  const size_t smem =
      (size_t)g.nst * g.stage_bytes + (size_t)cw * max_acc * 32 * 8 + (sizeof(GbQuery) + sizeof(GbItem)) * cw;
  int rc = ALK_OK;
  if (ntiles) {
    CK(cudaFuncSetAttribute(k_gb_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gb_tma, (int)(cw + 1) * 32, smem));
    if (occ < 1) {
      cudaFreeAsync(db, s);
      return ALK_ERR_UNSUPPORTED;
    }
    const uint32_t per_sm = tune && tune->blocks_per_sm ? std::min<uint32_t>(tune->blocks_per_sm, occ) : occ;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(ntiles, (uint64_t)sms_count() * per_sm);
    if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev0, s);
    k_gb_tma<<<grid, (cw + 1) * 32, smem, s>>>(g);
    if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev1, s);
    alk::g_kernel_launches++;
    CK(cudaGetLastError());
    if (used) {
      used->consumer_warps = cw;
      used->stages = g.nst;
      used->blocks_per_sm = per_sm;
    }
  }
  int herr = 0;
  std::vector<uint64_t> irows(nitems);
  CK(cudaMemcpyAsync(&herr, db + o_err, 4, cudaMemcpyDeviceToHost, s));
  if (nitems) CK(cudaMemcpyAsync(irows.data(), db + o_rows, 8 * (size_t)nitems, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  for (uint32_t qi = 0; qi < nq; qi++)
    if (qs[qi].h_seg_rows) std::fill(qs[qi].h_seg_rows, qs[qi].h_seg_rows + qs[qi].nseg, 0);
  for (uint32_t i = 0; i < nitems; i++)
    if (qs[item_src[i].first].h_seg_rows) qs[item_src[i].first].h_seg_rows[item_src[i].second] = irows[i];
  if (timer && timer->on && ntiles) {
    float ms = 0;
    cudaEventElapsedTime(&ms, (cudaEvent_t)timer->ev0, (cudaEvent_t)timer->ev1);
    timer->ms += ms;
    timer->launches++;
  }
  if (herr) rc = herr;
  return rc;
}

}  // extern "C"
