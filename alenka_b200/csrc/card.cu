// Learned cardinality estimator: 16-bin column histograms per segment (features), and a
// small MLP (64 -> 128 -> 128 -> 3, ReLU) with BF16 weights and FP32 accumulation,
// trained on the GPU by these kernels (forward, backward, Adam). The network predicts
// per-segment log-selectivities that size the fused stages' tables and survivor lists
// on a query's first run; the exact counts the stages report remain the fallback and
// the measure of its error. No counterpart in the reference (it sizes from the free
// memory, cm.cu:3184).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"

using namespace alkd;

namespace {
constexpr int kT = 256;
constexpr int kIn = ALK_CARD_FEATURES, kHid = ALK_CARD_HIDDEN, kOut = ALK_CARD_OUTPUTS;
// parameter layout (fp32 master copy): W1 [kHid][kIn], b1, W2 [kHid][kHid], b2, W3 [kOut][kHid], b3
constexpr size_t kW1 = 0, kB1 = kW1 + (size_t)kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + (size_t)kHid * kHid,
                 kW3 = kB2 + kHid, kB3 = kW3 + (size_t)kOut * kHid, kParams = kB3 + kOut;

int grid_for(uint64_t n) { return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + kT - 1) / kT, 148 * 16)); }

// ---------------------------------------------------------------- histograms
__global__ void __launch_bounds__(kT) k_hist16(alk_colseg d, int64_t lo, uint64_t span, unsigned int* out) {
  __shared__ unsigned int s_h[16];
  if (threadIdx.x < 16) s_h[threadIdx.x] = 0;
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < d.rows; i += (uint64_t)gridDim.x * kT) {
    const int64_t v = load_for(d.data, d.bits, d.lower, i);
    const uint64_t o = (uint64_t)v - (uint64_t)lo;
    const uint32_t b = o >= span ? (v < lo ? 0u : 15u) : (uint32_t)((double)o / (double)span * 16.0);
    atomicAdd(&s_h[b > 15 ? 15 : b], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 16 && s_h[threadIdx.x]) atomicAdd(out + threadIdx.x, s_h[threadIdx.x]);
}

// ---------------------------------------------------------------- MLP kernels
// out[n][m] = act(b[m] + sum_k in[n][k] * W[m][k]), W in BF16, accumulation in FP32
__global__ void __launch_bounds__(kT) k_dense_fwd(const float* in, const __nv_bfloat16* W, const float* b,
                                                  float* out, uint64_t n, int K, int M, int relu) {
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n * M; t += (uint64_t)gridDim.x * kT) {
    const uint64_t r = t / M;
    const int m = (int)(t - r * M);
    const float* x = in + r * K;
    const __nv_bfloat16* w = W + (size_t)m * K;
    float acc = b[m];
    for (int k = 0; k < K; k++) acc = fmaf(x[k], __bfloat162float(w[k]), acc);
    out[t] = relu ? fmaxf(acc, 0.f) : acc;
  }
}
// dIn[n][k] = sum_m dZ[n][m] * W[m][k]
__global__ void __launch_bounds__(kT) k_dense_bwd_data(const float* dz, const __nv_bfloat16* W, float* din,
                                                       uint64_t n, int K, int M) {
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n * K; t += (uint64_t)gridDim.x * kT) {
    const uint64_t r = t / K;
    const int k = (int)(t - r * K);
    float acc = 0.f;
    for (int m = 0; m < M; m++) acc = fmaf(dz[r * M + m], __bfloat162float(W[(size_t)m * K + k]), acc);
    din[t] = acc;
  }
}
// dW[m][k] = sum_n dZ[n][m] * in[n][k]; db[m] = sum_n dZ[n][m]
__global__ void __launch_bounds__(kT) k_dense_bwd_weight(const float* dz, const float* in, float* dW, float* db,
                                                         uint64_t n, int K, int M) {
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < (uint64_t)M * (K + 1); t += (uint64_t)gridDim.x * kT) {
    const int m = (int)(t / (K + 1));
    const int k = (int)(t - (uint64_t)m * (K + 1));
    float acc = 0.f;
    if (k < K) {
      for (uint64_t r = 0; r < n; r++) acc = fmaf(dz[r * M + m], in[r * K + k], acc);
      dW[(size_t)m * K + k] = acc;
    } else {
      for (uint64_t r = 0; r < n; r++) acc += dz[r * M + m];
      db[m] = acc;
    }
  }
}
// dZ = dA where the ReLU output a is positive
__global__ void __launch_bounds__(kT) k_relu_bwd(float* d, const float* a, uint64_t n) {
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n; t += (uint64_t)gridDim.x * kT)
    if (!(a[t] > 0.f)) d[t] = 0.f;
}
// masked mean squared error: dY = 2 (y - t) mask / count, loss accumulated into *loss
__global__ void __launch_bounds__(kT) k_mse(const float* y, const float* tgt, const float* mask, float* dy,
                                            uint64_t n, float inv_count, float* loss) {
  float l = 0.f;
  for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n; t += (uint64_t)gridDim.x * kT) {
    const float e = (y[t] - tgt[t]) * mask[t];
    dy[t] = 2.f * e * inv_count;
    l += e * e;
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * inv_count);
}
// Adam on the FP32 master parameters; the BF16 weight copies follow
__global__ void __launch_bounds__(kT) k_adam(float* p, const float* g, float* m1, float* m2, __nv_bfloat16* wbf,
                                             uint64_t n, float lr, float b1, float b2, float c1, float c2,
                                             float eps) {
  for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
    const float gi = g[i];
    const float a = m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    const float v = m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    const float x = p[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
    wbf[i] = __float2bfloat16(x);
  }
}
}  // namespace

// Parameters on the device: FP32 master, Adam moments, gradients and BF16 copies (all
// kParams long; the BF16 copy of a bias is unused); a scratch of activations.
struct alk_mlp {
  float* master = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* grad = nullptr;
  __nv_bfloat16* wbf = nullptr;
  float* loss = nullptr;
  uint64_t step = 0;
};

#define CK(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return alk::cuda_fail(e_); \
  } while (0)

namespace {
int mlp_forward(alk_mlp* m, const float* x, uint64_t n, float* h1, float* h2, float* y, cudaStream_t s) {
  k_dense_fwd<<<grid_for(n * kHid), kT, 0, s>>>(x, m->wbf + kW1, m->master + kB1, h1, n, kIn, kHid, 1);
  k_dense_fwd<<<grid_for(n * kHid), kT, 0, s>>>(h1, m->wbf + kW2, m->master + kB2, h2, n, kHid, kHid, 1);
  k_dense_fwd<<<grid_for(n * kOut), kT, 0, s>>>(h2, m->wbf + kW3, m->master + kB3, y, n, kHid, kOut, 0);
  alk::g_kernel_launches += 3;
  CK(cudaGetLastError());
  return ALK_OK;
}
// gradients of the masked MSE over n samples into m->grad; *m->loss += loss
int mlp_backward(alk_mlp* m, const float* x, const float* t, const float* mask, uint64_t n, float inv_count,
                 float* buf, cudaStream_t s) {
  float* h1 = buf;
  float* h2 = h1 + n * kHid;
  float* y = h2 + n * kHid;
  float* dy = y + n * kOut;
  float* d2 = dy + n * kOut;
  float* d1 = d2 + n * kHid;
  int rc = mlp_forward(m, x, n, h1, h2, y, s);
  if (rc) return rc;
  k_mse<<<grid_for(n * kOut), kT, 0, s>>>(y, t, mask, dy, n * kOut, inv_count, m->loss);
  k_dense_bwd_weight<<<grid_for((uint64_t)kOut * (kHid + 1)), kT, 0, s>>>(dy, h2, m->grad + kW3, m->grad + kB3, n,
                                                                          kHid, kOut);
  k_dense_bwd_data<<<grid_for(n * kHid), kT, 0, s>>>(dy, m->wbf + kW3, d2, n, kHid, kOut);
  k_relu_bwd<<<grid_for(n * kHid), kT, 0, s>>>(d2, h2, n * kHid);
  k_dense_bwd_weight<<<grid_for((uint64_t)kHid * (kHid + 1)), kT, 0, s>>>(d2, h1, m->grad + kW2, m->grad + kB2, n,
                                                                          kHid, kHid);
  k_dense_bwd_data<<<grid_for(n * kHid), kT, 0, s>>>(d2, m->wbf + kW2, d1, n, kHid, kHid);
  k_relu_bwd<<<grid_for(n * kHid), kT, 0, s>>>(d1, h1, n * kHid);
  k_dense_bwd_weight<<<grid_for((uint64_t)kHid * (kIn + 1)), kT, 0, s>>>(d1, x, m->grad + kW1, m->grad + kB1, n,
                                                                         kIn, kHid);
  alk::g_kernel_launches += 8;
  CK(cudaGetLastError());
  return ALK_OK;
}
size_t mlp_scratch_floats(uint64_t n) { return n * (4 * (size_t)kHid + 2 * kOut); }
}  // namespace

extern "C" {

uint32_t alk_mlp_param_count(void) { return (uint32_t)kParams; }

int alk_mlp_create(uint64_t seed, alk_mlp** out, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!out) return ALK_ERR_ARG;
  // He-style uniform initialisation from a seeded splitmix64 stream; biases zero
  std::vector<float> p(kParams, 0.f);
  uint64_t st = seed;
  auto uni = [&]() {
    uint64_t z = (st += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (double)(z >> 11) / 9007199254740992.0 * 2.0 - 1.0;
  };
  auto fill = [&](size_t off, size_t cnt, int fan_in) {
    const double a = std::sqrt(6.0 / fan_in);
    for (size_t i = 0; i < cnt; i++) p[off + i] = (float)(a * uni());
  };
  fill(kW1, (size_t)kHid * kIn, kIn);
  fill(kW2, (size_t)kHid * kHid, kHid);
  fill(kW3, (size_t)kOut * kHid, kHid);
  std::vector<__nv_bfloat16> wb(kParams);
  for (size_t i = 0; i < kParams; i++) wb[i] = __float2bfloat16(p[i]);
  auto* m = new alk_mlp();
  cudaError_t e = cudaSuccess;
  void* base = nullptr;
  const size_t fbytes = kParams * 4;
  e = cudaMallocAsync(&base, 4 * fbytes + kParams * 2 + 64, s);
  if (e != cudaSuccess) {
    delete m;
    return alk::cuda_fail(e);
  }
  uint8_t* b = (uint8_t*)base;
  m->master = (float*)b;
  m->m1 = (float*)(b + fbytes);
  m->m2 = (float*)(b + 2 * fbytes);
  m->grad = (float*)(b + 3 * fbytes);
  m->loss = (float*)(b + 4 * fbytes);
  m->wbf = (__nv_bfloat16*)(b + 4 * fbytes + 64);
  CK(cudaMemcpyAsync(m->master, p.data(), fbytes, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(m->m1, 0, 3 * fbytes + 64, s));
  CK(cudaMemcpyAsync(m->wbf, wb.data(), kParams * 2, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // the host staging vectors go out of scope
  *out = m;
  return ALK_OK;
}

void alk_mlp_free(alk_mlp* m, alk_stream stream) {
  if (!m) return;
  if (m->master) cudaFreeAsync(m->master, (cudaStream_t)stream);
  delete m;
}

int alk_mlp_forward(alk_mlp* m, const float* d_x, uint64_t n, float* d_y, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!m || !d_x || !d_y) return ALK_ERR_ARG;
  if (n == 0) return ALK_OK;
  float* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, n * 2 * kHid * sizeof(float), s));
  int rc = mlp_forward(m, d_x, n, buf, buf + n * kHid, d_y, s);
  cudaFreeAsync(buf, s);
  return rc;
}

int alk_mlp_gradients(alk_mlp* m, const float* d_x, const float* d_t, const float* d_mask, uint64_t n,
                      float* d_grad, float* h_loss, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!m || !d_x || !d_t || !d_mask || n == 0) return ALK_ERR_ARG;
  float* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, mlp_scratch_floats(n) * sizeof(float), s));
  CK(cudaMemsetAsync(m->loss, 0, 4, s));
  int rc = mlp_backward(m, d_x, d_t, d_mask, n, 1.f / (float)n, buf, s);
  cudaFreeAsync(buf, s);
  if (rc) return rc;
  if (d_grad) CK(cudaMemcpyAsync(d_grad, m->grad, kParams * 4, cudaMemcpyDeviceToDevice, s));
  float l = 0;
  CK(cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (h_loss) *h_loss = l;
  return ALK_OK;
}

int alk_mlp_train(alk_mlp* m, const float* d_x, const float* d_t, const float* d_mask, uint64_t n, uint32_t epochs,
                  uint32_t batch, float lr, float* h_loss, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!m || !d_x || !d_t || !d_mask || n == 0 || batch == 0) return ALK_ERR_ARG;
  const uint64_t bsz = std::min<uint64_t>(batch, n);
  float* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, mlp_scratch_floats(bsz) * sizeof(float), s));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float last = 0;
  for (uint32_t ep = 0; ep < epochs; ep++) {
    CK(cudaMemsetAsync(m->loss, 0, 4, s));
    uint64_t nb = 0;
    for (uint64_t r0 = 0; r0 < n; r0 += bsz, nb++) {
      const uint64_t cnt = std::min<uint64_t>(bsz, n - r0);
      int rc = mlp_backward(m, d_x + r0 * kIn, d_t + r0 * kOut, d_mask + r0 * kOut, cnt, 1.f / (float)cnt, buf, s);
      if (rc) {
        cudaFreeAsync(buf, s);
        return rc;
      }
      m->step++;
      const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
      k_adam<<<grid_for(kParams), kT, 0, s>>>(m->master, m->grad, m->m1, m->m2, m->wbf, kParams, lr, b1, b2, c1, c2,
                                              eps);
      alk::g_kernel_launches++;
      CK(cudaGetLastError());
    }
    float l = 0;
    CK(cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    last = nb ? l / (float)nb : 0.f;
  }
  cudaFreeAsync(buf, s);
  if (h_loss) *h_loss = last;
  return ALK_OK;
}

int alk_mlp_set_params(alk_mlp* m, const float* h_master, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!m || !h_master) return ALK_ERR_ARG;
  std::vector<__nv_bfloat16> wb(kParams);
  for (size_t i = 0; i < kParams; i++) wb[i] = __float2bfloat16(h_master[i]);
  CK(cudaMemcpyAsync(m->master, h_master, kParams * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(m->wbf, wb.data(), kParams * 2, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_mlp_params(const alk_mlp* m, float* h_master, uint16_t* h_bf16, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!m) return ALK_ERR_ARG;
  if (h_master) CK(cudaMemcpyAsync(h_master, m->master, kParams * 4, cudaMemcpyDeviceToHost, s));
  if (h_bf16) CK(cudaMemcpyAsync(h_bf16, m->wbf, kParams * 2, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return ALK_OK;
}

int alk_card_hist16(const alk_colseg* seg, int64_t lo, int64_t hi, uint32_t* d_hist16, alk_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (!seg || !d_hist16 || hi < lo) return ALK_ERR_ARG;
  if (!(seg->bits == 8 || seg->bits == 16 || seg->bits == 32 || seg->bits == 64)) return ALK_ERR_ARG;
  CK(cudaMemsetAsync(d_hist16, 0, 64, s));
  if (seg->rows == 0) return ALK_OK;
  const uint64_t span = (uint64_t)hi - (uint64_t)lo + 1;  // 0 = the whole int64 range
  k_hist16<<<grid_for(seg->rows), kT, 0, s>>>(*seg, lo, span ? span : ~0ull, (unsigned int*)d_hist16);
  alk::g_kernel_launches++;
  CK(cudaGetLastError());
  return ALK_OK;
}

}  // extern "C"
