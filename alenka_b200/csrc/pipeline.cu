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

struct HtView {
  uint64_t cap;  // power of two
  uint32_t* state;
  int64_t* key;
  uint32_t* slot;
  int64_t* payload;  // [npay][slot_cap]
  uint64_t slot_cap;
  uint32_t npay;
  unsigned long long* nslots;
  int* flags;  // [0] duplicate key, [1] slot overflow, [2] timeout
};

__device__ __forceinline__ int64_t ht_probe(const HtView& h, int64_t k) {
  const uint64_t mask = h.cap - 1;
  uint64_t p = murmur_u64((uint64_t)k) & mask;
  for (uint64_t n = 0; n <= mask; n++) {
    const uint32_t s = __ldg(h.state + p);
    if (s == 0) return -1;
    if (__ldg(h.key + p) == k) return (int64_t)__ldg(h.slot + p);
    p = (p + 1) & mask;
  }
  return -1;
}

// Inserts a unique key; returns its payload slot or -1 (duplicate / overflow / timeout,
// recorded in flags).
__device__ __forceinline__ int64_t ht_insert(const HtView& h, int64_t k) {
  const uint64_t mask = h.cap - 1;
  uint64_t p = murmur_u64((uint64_t)k) & mask;
  uint32_t spins = 0;
  for (uint64_t n = 0; n <= mask;) {
    uint32_t s = *((volatile uint32_t*)h.state + p);
    if (s == 0) {
      if (atomicCAS(h.state + p, 0u, 1u) == 0u) {
        unsigned long long sl = atomicAdd(h.nslots, 1ull);
        if (sl >= h.slot_cap) {
          atomicExch(h.flags + 1, 1);
          h.key[p] = k;
          h.slot[p] = 0;
          __threadfence();
          atomicExch(h.state + p, 2u);
          return -1;
        }
        h.key[p] = k;
        h.slot[p] = (uint32_t)sl;
        __threadfence();
        atomicExch(h.state + p, 2u);
        return (int64_t)sl;
      }
      continue;
    }
    if (s == 1) {
      if (++spins > kSpinLimit) {
        atomicExch(h.flags + 2, 1);
        return -1;
      }
      continue;
    }
    __threadfence();
    if (__ldcg(h.key + p) == k) {
      atomicExch(h.flags, 1);  // duplicate build key: the fused plan does not apply
      return -1;
    }
    p = (p + 1) & mask;
    n++;
  }
  atomicExch(h.flags + 1, 1);
  return -1;
}

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
};

template <bool kBuild>
__global__ void __launch_bounds__(kT) k_stage(StageArgs a) {
  __shared__ alk_instr s_ins[8][ALK_MAX_INSTR];
  __shared__ int64_t s_consts[8][ALK_MAX_CONST];
  __shared__ uint32_t s_n[8], s_res[8];
  __shared__ int64_t s_regs[ALK_MAX_REGS * kT];
  __shared__ alk_colseg s_desc[kMaxCols];
  for (uint32_t p = 0; p < a.nprogs; p++) {
    for (uint32_t i = threadIdx.x; i < a.progs[p].n_instr; i += kT) s_ins[p][i] = a.progs[p].ins[i];
    for (uint32_t i = threadIdx.x; i < ALK_MAX_CONST; i += kT) s_consts[p][i] = a.progs[p].consts[i];
    if (threadIdx.x == 0) {
      s_n[p] = a.progs[p].n_instr;
      s_res[p] = a.progs[p].result;
    }
  }
  unsigned long long rows_seen = 0;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    __syncthreads();
    const uint32_t seg = a.tile_seg[tile];
    const uint32_t row0 = a.tile_row0[tile];
    if (threadIdx.x < a.ncols) s_desc[threadIdx.x] = a.cols[threadIdx.x * a.nseg + seg];
    __syncthreads();
    const uint32_t rows = min((uint32_t)kTile, s_desc[0].rows - row0);
    const bool all = a.seg_mode[seg] == 1 || s_n[0] == 0;
#pragma unroll 2
    for (int k = 0; k < kItems; k++) {
      const uint32_t r = k * kT + threadIdx.x;
      if (r >= rows) continue;
      const uint64_t row = (uint64_t)row0 + r;
      rows_seen++;
      int64_t j = -1;
      auto col = [&](uint32_t slot) -> int64_t {
        if (slot >= 32) return __ldg(a.probe.payload + (uint64_t)(slot - 32) * a.probe.slot_cap + j);
        const alk_colseg& d = s_desc[slot];
        return load_for(d.data, d.bits, d.lower, row);
      };
      if (!all && vm_eval<kT>(s_ins[0], s_n[0], s_res[0], s_consts[0], s_regs + threadIdx.x, col) == 0) continue;
      if (a.probe_slot >= 0) {
        j = ht_probe(a.probe, col((uint32_t)a.probe_slot));
        if (j < 0) continue;
      }
      if (kBuild) {
        const int64_t sl = ht_insert(a.build, col((uint32_t)a.build_slot));
        if (sl < 0) continue;
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
          const int64_t v = vm_eval<kT>(s_ins[1 + g], s_n[1 + g], s_res[1 + g], s_consts[1 + g],
                                        s_regs + threadIdx.x, col);
          if (kind == ALK_AGG_SUM) atomicAdd(dst, (unsigned long long)v);
          else if (kind == ALK_AGG_MIN) atomicMin((long long*)dst, (long long)v);
          else atomicMax((long long*)dst, (long long)v);
        }
        if (a.cnt) atomicAdd(a.cnt + j, 1ull);
      }
    }
  }
  for (int o = 16; o; o >>= 1) rows_seen += __shfl_xor_sync(0xffffffffu, rows_seen, o);
  if ((threadIdx.x & 31) == 0 && a.rows_in) atomicAdd(a.rows_in, rows_seen);
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

int grid_for(uint64_t n) {
  uint64_t b = (n + kT - 1) / kT;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sms() * 8));
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

int alk_ht_create(uint64_t max_keys, uint32_t npay, alk_ht** out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out || npay > 8 || max_keys >= 0xffffffffull) return ALK_ERR_ARG;
  auto* h = new alk_ht();
  uint64_t cap = 1024;
  while (cap < 2 * max_keys) cap <<= 1;
  uint64_t slot_cap = std::max<uint64_t>(max_keys, 1);
  size_t bytes = cap * (4 + 8 + 4) + slot_cap * 8 * npay + 64;
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
  h->v.state = (uint32_t*)p;
  p += cap * 4;
  h->v.slot = (uint32_t*)p;
  p += cap * 4;
  h->v.nslots = (unsigned long long*)p;
  h->v.flags = (int*)(p + 8);
  h->v.slot_cap = slot_cap;
  h->v.npay = npay;
  CK(cudaMemsetAsync(h->v.state, 0, cap * 4, s));
  CK(cudaMemsetAsync(p, 0, 64, s));
  *out = h;
  return ALK_OK;
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
  int f[3] = {0, 0, 0};
  CK(cudaMemcpyAsync(&n, h->v.nslots, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(f, h->v.flags, sizeof(f), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (nslots) *nslots = std::min<uint64_t>(n, h->v.slot_cap);
  if (flags) *flags = (f[0] ? 1 : 0) | (f[1] ? 2 : 0) | (f[2] ? 4 : 0);
  return ALK_OK;
}

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

int alk_pipeline_build(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                       const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                       int32_t build_slot, const int32_t* pay_src, uint64_t* h_rows_in, alk_stream stream) {
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
  if (!prog_ok(prog, ncols, npay_probe)) return ALK_ERR_ARG;
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, &prog, 1, hb, a, 4 * 8, &off_x);
  if (rc) return rc;
  std::memcpy(&hb[off_x], pay_src, 4 * build->v.npay);
  void* db = nullptr;
  CK(cudaMallocAsync(&db, hb.size() + 16, s));
  CK(cudaMemcpyAsync(db, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  unsigned long long* rows_in = (unsigned long long*)((uint8_t*)db + ((hb.size() + 7) & ~size_t(7)));
  CK(cudaMemsetAsync(rows_in, 0, 8, s));
  patch(a, (uint8_t*)db);
  a.pay_src = (const int32_t*)((uint8_t*)db + off_x);
  a.probe_slot = probe_slot;
  if (probe) a.probe = probe->v;
  a.build_slot = build_slot;
  a.build = build->v;
  a.rows_in = rows_in;
  if (a.ntiles) {
    int grid = std::min<int>((int)a.ntiles, sms() * 4);
    k_stage<true><<<grid, kT, 0, s>>>(a);
    alk::g_kernel_launches++;
  }
  CK(cudaGetLastError());
  unsigned long long rin = 0;
  CK(cudaMemcpyAsync(&rin, rows_in, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  if (h_rows_in) *h_rows_in = rin;
  return ALK_OK;
}

int alk_pipeline_probe_agg(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                           const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                           const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, int64_t* d_acc,
                           uint64_t acc_stride, uint64_t* d_cnt, uint64_t* h_rows_in, alk_stream stream,
                           alk_event_timer* timer) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!probe || probe_slot < 0 || (uint32_t)probe_slot >= ncols || ncols == 0 || ncols > kMaxCols || nagg > 7)
    return ALK_ERR_ARG;
  {
    // accumulators are indexed by the probed table's slots: one per inserted key
    unsigned long long ns = 0;
    CK(cudaMemcpyAsync(&ns, probe->v.nslots, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (acc_stride < std::min<uint64_t>(ns, probe->v.slot_cap)) return ALK_ERR_ARG;
  }
  std::vector<alk_program> progs(1 + nagg);
  std::memset(progs.data(), 0, sizeof(alk_program) * progs.size());
  if (pred) progs[0] = *pred;
  for (uint32_t g = 0; g < nagg; g++)
    if (agg_kind[g] != ALK_AGG_COUNT) progs[1 + g] = agg_progs[g];
  for (auto& p : progs)
    if (!prog_ok(p, ncols, probe->v.npay)) return ALK_ERR_ARG;
  StageArgs a{};
  std::vector<uint8_t> hb;
  size_t off_x;
  int rc = stage_common(cols, ncols, nseg, seg_mode, progs.data(), (uint32_t)progs.size(), hb, a, 16, &off_x);
  if (rc) return rc;
  std::memcpy(&hb[off_x], agg_kind, nagg);
  void* db = nullptr;
  CK(cudaMallocAsync(&db, hb.size() + 16, s));
  CK(cudaMemcpyAsync(db, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
  unsigned long long* rows_in = (unsigned long long*)((uint8_t*)db + ((hb.size() + 7) & ~size_t(7)));
  CK(cudaMemsetAsync(rows_in, 0, 8, s));
  patch(a, (uint8_t*)db);
  a.agg_kind = (const uint8_t*)db + off_x;
  a.probe_slot = probe_slot;
  a.probe = probe->v;
  a.build_slot = -1;
  a.nagg = nagg;
  a.acc = d_acc;
  a.acc_stride = acc_stride;
  a.cnt = (unsigned long long*)d_cnt;
  a.rows_in = rows_in;
  if (a.ntiles) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage<false>, kT, 0);
    int grid = std::min<int>((int)a.ntiles, sms() * std::max(occ, 1));
    if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev0, s);
    k_stage<false><<<grid, kT, 0, s>>>(a);
    if (timer && timer->on) cudaEventRecord((cudaEvent_t)timer->ev1, s);
    alk::g_kernel_launches++;
  }
  CK(cudaGetLastError());
  unsigned long long rin = 0;
  CK(cudaMemcpyAsync(&rin, rows_in, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  if (timer && timer->on && a.ntiles) {
    float ms = 0;
    cudaEventElapsedTime(&ms, (cudaEvent_t)timer->ev0, (cudaEvent_t)timer->ev1);
    timer->ms += ms;
    timer->launches++;
  }
  if (h_rows_in) *h_rows_in = rin;
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
  int blocks = (int)std::min<uint64_t>((n + 1023) / 1024, (uint64_t)sms() * 2);
  std::vector<int64_t> best((size_t)blocks * k);
  void* db = nullptr;
  CK(cudaMallocAsync(&db, best.size() * 8 + 16, s));
  k_topk_local<<<blocks, kT, 0, s>>>(d_rank, (const unsigned long long*)d_live, n, k, (int64_t*)db);
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
