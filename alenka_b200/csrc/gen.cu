// Device-side generator of the single-table lineitem shape, for workloads too large to
// write as files (the reference loads its tables from files; this stands in for them):
// every value is a function of (seed, column, row), so the segments can be generated in
// place in device memory, in two passes: the per-segment minimum and maximum of every
// column (the zone maps and frame-of-reference bases), then the stored values at the
// width the format's encoder picks for that range. Columns, in order: l_orderkey (4 rows
// per key), l_quantity U[1,50], l_extendedprice U[90000,10500000] (cents), l_discount
// U[0,10] (hundredths), l_shipdate uniform yyyymmdd over 1992-01-02..1998-12-01, and the
// dictionary codes of l_returnflag (3 values) and l_linestatus (2 values).
#include <algorithm>
#include <vector>

#include "internal.h"

namespace {
constexpr int kGenCols = 7;
constexpr int kT = 256;

__host__ __device__ inline uint64_t splitmix(uint64_t x) {
  uint64_t z = x + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// yyyymmdd of a day count since 1970-01-01 (proleptic Gregorian civil calendar)
__host__ __device__ inline int64_t civil(int64_t z) {
  z += 719468;
  const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  const int64_t doe = z - era * 146097;
  const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  int64_t y = yoe + era * 400;
  const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const int64_t mp = (5 * doy + 2) / 153;
  const int64_t d = doy - (153 * mp + 2) / 5 + 1;
  const int64_t m = mp + (mp < 10 ? 3 : -9);
  y += m <= 2;
  return y * 10000 + m * 100 + d;
}

constexpr int64_t kDay0 = 8036;   // 1992-01-02
constexpr int64_t kDay1 = 10561;  // 1998-12-01

__host__ __device__ inline int64_t gen_value(uint64_t seed, int col, uint64_t row) {
  const uint64_t h = splitmix(seed * 0x100000001b3ull + (uint64_t)col * 0x9e3779b97f4a7c15ull + row * 0xd1b54a32d192ed03ull);
  switch (col) {
    case 0: return 1 + (int64_t)(row / 4);
    case 1: return 1 + (int64_t)(h % 50);
    case 2: return 90000 + (int64_t)(h % (10500000 - 90000 + 1));
    case 3: return (int64_t)(h % 11);
    case 4: return civil(kDay0 + (int64_t)(h % (uint64_t)(kDay1 - kDay0 + 1)));
    case 5: return (int64_t)(h % 3);
    default: return (int64_t)(h % 2);
  }
}

struct GenSeg {
  uint64_t row0;  // first row of the segment within the table
  uint32_t rows, pad;
};

// per segment and column: [min, max] (initialised to [INT64_MAX, INT64_MIN])
__global__ void __launch_bounds__(kT) k_gen_minmax(uint64_t seed, const GenSeg* segs, long long* mm) {
  const GenSeg sg = segs[blockIdx.y];
  long long lo[kGenCols], hi[kGenCols];
#pragma unroll
  for (int c = 0; c < kGenCols; c++) {
    lo[c] = INT64_MAX;
    hi[c] = INT64_MIN;
  }
  for (uint32_t r = blockIdx.x * kT + threadIdx.x; r < sg.rows; r += gridDim.x * kT) {
#pragma unroll
    for (int c = 0; c < kGenCols; c++) {
      const long long v = gen_value(seed, c, sg.row0 + r);
      lo[c] = min(lo[c], v);
      hi[c] = max(hi[c], v);
    }
  }
#pragma unroll
  for (int c = 0; c < kGenCols; c++) {
    for (int o = 16; o; o >>= 1) {
      lo[c] = min(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = max(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(mm + ((size_t)blockIdx.y * kGenCols + c) * 2, lo[c]);
      atomicMax(mm + ((size_t)blockIdx.y * kGenCols + c) * 2 + 1, hi[c]);
    }
  }
}

__global__ void __launch_bounds__(kT) k_gen_write(uint64_t seed, const GenSeg* segs, const alk_colseg* cols,
                                                  uint32_t nseg) {
  const uint32_t g = blockIdx.y;
  const GenSeg sg = segs[g];
  for (uint32_t r = blockIdx.x * kT + threadIdx.x; r < sg.rows; r += gridDim.x * kT) {
#pragma unroll
    for (int c = 0; c < kGenCols; c++) {
      const alk_colseg& d = cols[(size_t)c * nseg + g];
      const uint64_t x = (uint64_t)gen_value(seed, c, sg.row0 + r) - (uint64_t)d.lower;
      switch (d.bits) {
        case 8: ((uint8_t*)d.data)[r] = (uint8_t)x; break;
        case 16: ((uint16_t*)d.data)[r] = (uint16_t)x; break;
        case 32: ((uint32_t*)d.data)[r] = (uint32_t)x; break;
        default: ((uint64_t*)d.data)[r] = x; break;
      }
    }
  }
}

void fill_segs(const uint32_t* seg_rows, uint32_t nseg, uint64_t row_base, std::vector<GenSeg>& out) {
  out.resize(nseg);
  uint64_t r = row_base;
  for (uint32_t g = 0; g < nseg; g++) {
    out[g] = GenSeg{r, seg_rows[g], 0};
    r += seg_rows[g];
  }
}
}  // namespace

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

extern "C" {

int alk_gen_flat_minmax(uint64_t seed, uint64_t row_base, const uint32_t* seg_rows, uint32_t nseg, int64_t* h_minmax,
                        alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!seg_rows || !h_minmax || nseg == 0 || nseg > 65535) return ALK_ERR_ARG;
  std::vector<GenSeg> segs;
  fill_segs(seg_rows, nseg, row_base, segs);
  std::vector<long long> init((size_t)nseg * kGenCols * 2);
  for (size_t i = 0; i < init.size(); i++) init[i] = (i & 1) ? INT64_MIN : INT64_MAX;
  uint8_t* db = nullptr;
  const size_t o_mm = ((sizeof(GenSeg) * nseg + 255) & ~size_t(255));
  CK(cudaMallocAsync((void**)&db, o_mm + init.size() * 8, s));
  CK(cudaMemcpyAsync(db, segs.data(), sizeof(GenSeg) * nseg, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(db + o_mm, init.data(), init.size() * 8, cudaMemcpyHostToDevice, s));
  uint32_t maxr = 0;
  for (uint32_t g = 0; g < nseg; g++) maxr = std::max(maxr, seg_rows[g]);
  dim3 grid(std::max<uint32_t>(1, std::min<uint32_t>((maxr + kT - 1) / kT, 512)), nseg);
  k_gen_minmax<<<grid, kT, 0, s>>>(seed, (const GenSeg*)db, (long long*)(db + o_mm));
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h_minmax, db + o_mm, init.size() * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_gen_flat_write(uint64_t seed, uint64_t row_base, const uint32_t* seg_rows, uint32_t nseg,
                       const alk_colseg* cols, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!seg_rows || !cols || nseg == 0 || nseg > 65535) return ALK_ERR_ARG;
  for (uint32_t i = 0; i < (uint32_t)kGenCols * nseg; i++) {
    const alk_colseg& d = cols[i];
    if (!(d.bits == 8 || d.bits == 16 || d.bits == 32 || d.bits == 64) || d.rows != seg_rows[i % nseg]) return ALK_ERR_ARG;
    if (d.rows && !d.data) return ALK_ERR_ARG;
  }
  std::vector<GenSeg> segs;
  fill_segs(seg_rows, nseg, row_base, segs);
  uint8_t* db = nullptr;
  const size_t o_cols = ((sizeof(GenSeg) * nseg + 255) & ~size_t(255));
  CK(cudaMallocAsync((void**)&db, o_cols + sizeof(alk_colseg) * kGenCols * nseg, s));
  CK(cudaMemcpyAsync(db, segs.data(), sizeof(GenSeg) * nseg, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(db + o_cols, cols, sizeof(alk_colseg) * kGenCols * nseg, cudaMemcpyHostToDevice, s));
  uint32_t maxr = 0;
  for (uint32_t g = 0; g < nseg; g++) maxr = std::max(maxr, seg_rows[g]);
  dim3 grid(std::max<uint32_t>(1, std::min<uint32_t>((maxr + kT - 1) / kT, 512)), nseg);
  k_gen_write<<<grid, kT, 0, s>>>(seed, (const GenSeg*)db, (const alk_colseg*)(db + o_cols), nseg);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  CK(cudaFreeAsync(db, s));
  CK(cudaStreamSynchronize(s));  // the caller's descriptor array may go away
  return ALK_OK;
}

int64_t alk_gen_flat_value(uint64_t seed, int col, uint64_t row) {
  return col < 0 || col >= kGenCols ? 0 : gen_value(seed, col, row);
}

}  // extern "C"
