// Learned cost model: byte features of input regions and a small MLP
// regressor (two hidden ReLU layers of 64, one linear output) trained in FP32
// and run in FP32 or BF16. The kernels are plain SIMT: the model is tiny
// (about 22k parameters), so tensor cores would gain nothing.
//
// The reference has no cost model; it records the fetched worklist length per
// round (--motivate-worklist-length, code/src/ngap/kernel_ngap_OA.cu:366-369)
// and sizes its adaptive AAS interval from the longest table list
// (kernel_ngap_OA.cu:180-194). Here the engine's per-unit worklist traces are
// the training data, and the prediction (worklist entries per input byte)
// drives chunk lengths, queue capacity and serving admission.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "common.h"

namespace {

#define CM_TRY(expr)                                                                       \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess) {                                                               \
      ngap::set_error("CUDA error %s at %s:%d: %s", cudaGetErrorName(_e), __FILE__,        \
                      __LINE__, cudaGetErrorString(_e));                                   \
      return NGAP_E_CUDA;                                                                  \
    }                                                                                      \
  } while (0)

constexpr int kFeatThreads = 256;
constexpr int kFeatWarps = kFeatThreads / 32;
constexpr int kRows = 32;         // samples per CTA in the MLP kernels
constexpr int kMlpThreads = 256;
constexpr int kMaxIn = 512;       // largest input dimension
constexpr int kHidden = 64;       // hidden units per layer

// One CTA per region: 256-bin histogram of the whole region, and the Shannon
// entropy of each window of `window` bytes (one warp per window).
__global__ void __launch_bounds__(kFeatThreads) features_kernel(const uint8_t* __restrict__ data,
                                                                const uint64_t* __restrict__ offs,
                                                                const uint64_t* __restrict__ lens,
                                                                int n, int window,
                                                                float* __restrict__ out) {
  __shared__ unsigned hist[256];
  __shared__ unsigned whist[kFeatWarps][256];
  __shared__ float wsum[kFeatWarps], wmax[kFeatWarps];
  __shared__ unsigned wcnt[kFeatWarps];
  const int r = blockIdx.x;
  if (r >= n) return;  // whole blocks
  const uint8_t* p = data + offs[r];
  const uint64_t L = lens[r];
  for (int i = threadIdx.x; i < 256; i += kFeatThreads) hist[i] = 0u;
  __syncthreads();
  for (uint64_t i = threadIdx.x; i < L; i += kFeatThreads) atomicAdd(&hist[p[i]], 1u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t W = (uint64_t)window;
  const uint64_t nwin = L == 0 ? 0 : (L < W ? 1 : L / W);
  float s = 0.f, mx = 0.f;
  unsigned cnt = 0;
  for (uint64_t k = warp; k < nwin; k += kFeatWarps) {
    const uint64_t w0 = k * W;
    const uint64_t wl = L < W ? L : W;
    for (int b = lane; b < 256; b += 32) whist[warp][b] = 0u;
    __syncwarp();
    for (uint64_t i = lane; i < wl; i += 32) atomicAdd(&whist[warp][p[w0 + i]], 1u);
    __syncwarp();
    float h = 0.f;
    const float inv = 1.f / (float)wl;
    for (int b = lane; b < 256; b += 32) {
      const unsigned c = whist[warp][b];
      if (c) {
        const float q = (float)c * inv;
        h -= q * log2f(q);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    s += h;
    mx = fmaxf(mx, h);
    cnt++;
    __syncwarp();
  }
  if (lane == 0) {
    wsum[warp] = s;
    wmax[warp] = mx;
    wcnt[warp] = cnt;
  }
  __syncthreads();
  float* o = out + (size_t)r * NGAP_FEAT_BYTES;
  const float invL = L ? 1.f / (float)L : 0.f;
  for (int b = threadIdx.x; b < 256; b += kFeatThreads) o[b] = (float)hist[b] * invL;
  if (threadIdx.x == 0) {
    float S = 0.f, M = 0.f;
    unsigned C = 0;
    for (int k = 0; k < kFeatWarps; k++) {
      S += wsum[k];
      M = fmaxf(M, wmax[k]);
      C += wcnt[k];
    }
    o[256] = C ? S / (float)C / 8.f : 0.f;
    o[257] = M / 8.f;
  }
}

// Parameter layout (FP32, contiguous): W1[D][H], b1[H], W2[H][H], b2[H], w3[H], b3.
// Host rounding of an FP32 value to bfloat16 precision, round to nearest
// even (the upper 16 bits of the IEEE-754 single after adding half an ulp of
// bfloat16 plus the tie bit); NaN passes unchanged.
inline float bf16_round(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return v;
  u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

struct Layout {
  int D, H;
  size_t w1, b1, w2, b2, w3, b3, total;
  __host__ __device__ Layout(int d, int h) : D(d), H(h) {
    w1 = 0;
    b1 = w1 + (size_t)D * H;
    w2 = b1 + H;
    b2 = w2 + (size_t)H * H;
    w3 = b2 + H;
    b3 = w3 + H;
    total = b3 + 1;
  }
};

// Forward pass of kRows samples held in shared memory; T = float or bf16 weights.
// xs[kRows][D] (already rounded for BF16), h1/h2[kRows][H]; yo[kRows].
template <class T, bool ROUND>
__device__ void mlp_forward(const T* __restrict__ P, const Layout& L, const float* xs, float* h1,
                            float* h2, float* yo) {
  const int t = threadIdx.x;
  auto ld = [](const T* a, size_t i) -> float {
    if constexpr (sizeof(T) == 2) return __bfloat162float(a[i]);
    else return (float)a[i];
  };
  auto rnd = [](float v) -> float {
    if constexpr (ROUND) return __bfloat162float(__float2bfloat16(v));
    else return v;
  };
  // layer 1: thread t computes unit j = t % H for samples s = t / H + k * (256 / H)
  const int j = t % kHidden, s0 = t / kHidden, step = kMlpThreads / kHidden;
  for (int s = s0; s < kRows; s += step) {
    float acc = ld(P, L.b1 + j);
    for (int d = 0; d < L.D; d++) acc = fmaf(xs[s * L.D + d], ld(P, L.w1 + (size_t)d * kHidden + j), acc);
    h1[s * kHidden + j] = rnd(fmaxf(acc, 0.f));
  }
  __syncthreads();
  for (int s = s0; s < kRows; s += step) {
    float acc = ld(P, L.b2 + j);
    for (int i = 0; i < kHidden; i++)
      acc = fmaf(h1[s * kHidden + i], ld(P, L.w2 + (size_t)i * kHidden + j), acc);
    h2[s * kHidden + j] = rnd(fmaxf(acc, 0.f));
  }
  __syncthreads();
  // output: one warp per sample
  const int warp = t >> 5, lane = t & 31;
  for (int s = warp; s < kRows; s += kMlpThreads / 32) {
    float acc = 0.f;
    for (int i = lane; i < kHidden; i += 32) acc = fmaf(h2[s * kHidden + i], ld(P, L.w3 + i), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) yo[s] = acc + ld(P, L.b3);
  }
  __syncthreads();
}

// Gradient of the mean squared error over one mini-batch: CTA b takes
// samples idx[b * kRows ...] (fewer in the last CTA), adds its partial
// gradients to grad (zeroed by the caller) and its squared errors to *loss.
__global__ void __launch_bounds__(kMlpThreads) mlp_grad_kernel(const float* __restrict__ P,
                                                               int D, const float* __restrict__ X,
                                                               const float* __restrict__ Y,
                                                               const int* __restrict__ idx,
                                                               int nb, float inv_nb,
                                                               float* __restrict__ grad,
                                                               float* __restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  const Layout L(D, kHidden);
  float* xs = sm;                        // kRows * D
  float* h1 = xs + kRows * D;            // kRows * H
  float* h2 = h1 + kRows * kHidden;
  float* d2 = h2 + kRows * kHidden;
  float* d1 = d2 + kRows * kHidden;
  float* yo = d1 + kRows * kHidden;      // kRows
  float* dy = yo + kRows;                // kRows
  const int t = threadIdx.x;
  const int b0 = blockIdx.x * kRows;
  const int rows = min(kRows, nb - b0);
  for (int i = t; i < kRows * D; i += kMlpThreads) {
    const int s = i / D, d = i - s * D;
    xs[i] = s < rows ? X[(size_t)idx[b0 + s] * D + d] : 0.f;
  }
  __syncthreads();
  mlp_forward<float, false>(P, L, xs, h1, h2, yo);
  if (t < kRows) {
    float e = 0.f;
    if (t < rows) {
      e = yo[t] - Y[idx[b0 + t]];
      atomicAdd(loss, e * e);
    }
    dy[t] = 2.f * e * inv_nb;
  }
  __syncthreads();
  const int j = t % kHidden, s0 = t / kHidden, step = kMlpThreads / kHidden;
  // output layer
  if (t < kHidden) {
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g = fmaf(dy[s], h2[s * kHidden + t], g);
    atomicAdd(grad + L.w3 + t, g);
  }
  if (t == kHidden) {
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g += dy[s];
    atomicAdd(grad + L.b3, g);
  }
  for (int s = s0; s < kRows; s += step)
    d2[s * kHidden + j] = h2[s * kHidden + j] > 0.f ? dy[s] * P[L.w3 + j] : 0.f;
  __syncthreads();
  // layer 2: dW2[i][j] = sum_s h1[s][i] d2[s][j]
  for (int k = t; k < kHidden * kHidden; k += kMlpThreads) {
    const int i = k / kHidden, jj = k - i * kHidden;
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g = fmaf(h1[s * kHidden + i], d2[s * kHidden + jj], g);
    atomicAdd(grad + L.w2 + k, g);
  }
  if (t < kHidden) {
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g += d2[s * kHidden + t];
    atomicAdd(grad + L.b2 + t, g);
  }
  for (int s = s0; s < kRows; s += step) {
    float acc = 0.f;
    for (int jj = 0; jj < kHidden; jj++)
      acc = fmaf(d2[s * kHidden + jj], P[L.w2 + (size_t)j * kHidden + jj], acc);
    d1[s * kHidden + j] = h1[s * kHidden + j] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // layer 1: dW1[d][j] = sum_s xs[s][d] d1[s][j]
  for (int k = t; k < D * kHidden; k += kMlpThreads) {
    const int d = k / kHidden, jj = k - d * kHidden;
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g = fmaf(xs[s * D + d], d1[s * kHidden + jj], g);
    atomicAdd(grad + L.w1 + k, g);
  }
  if (t < kHidden) {
    float g = 0.f;
    for (int s = 0; s < kRows; s++) g += d1[s * kHidden + t];
    atomicAdd(grad + L.b1 + t, g);
  }
}

// Adam (Kingma and Ba, 2015) with bias correction; zeroes the gradient.
__global__ void adam_kernel(float* __restrict__ P, float* __restrict__ G, float* __restrict__ M,
                            float* __restrict__ V, size_t n, float lr, float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m * c1) / (sqrtf(v * c2) + eps);
    G[i] = 0.f;
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

// Inference: CTA b takes samples b * kRows ...; BF16 rounds inputs, weights
// and activations to bfloat16 and accumulates in FP32.
template <bool BF16>
__global__ void __launch_bounds__(kMlpThreads) mlp_infer_kernel(const void* __restrict__ Pv, int D,
                                                                const float* __restrict__ X,
                                                                int64_t n, float* __restrict__ Y) {
  extern __shared__ __align__(16) float sm[];
  const Layout L(D, kHidden);
  float* xs = sm;
  float* h1 = xs + kRows * D;
  float* h2 = h1 + kRows * kHidden;
  float* yo = h2 + kRows * kHidden;
  const int64_t b0 = (int64_t)blockIdx.x * kRows;
  const int64_t left = n - b0;
  const int rows = (int)(left < kRows ? left : kRows);
  for (int i = threadIdx.x; i < kRows * D; i += kMlpThreads) {
    const int s = i / D, d = i - s * D;
    const float v = s < rows ? X[(size_t)(b0 + s) * D + d] : 0.f;
    xs[i] = BF16 ? __bfloat162float(__float2bfloat16(v)) : v;
  }
  __syncthreads();
  if (BF16)
    mlp_forward<__nv_bfloat16, true>(static_cast<const __nv_bfloat16*>(Pv), L, xs, h1, h2, yo);
  else
    mlp_forward<float, false>(static_cast<const float*>(Pv), L, xs, h1, h2, yo);
  if (threadIdx.x < rows) Y[b0 + threadIdx.x] = yo[threadIdx.x];
}

size_t grad_smem(int D) { return sizeof(float) * ((size_t)kRows * D + 4 * kRows * kHidden + 2 * kRows); }
size_t infer_smem(int D) { return sizeof(float) * ((size_t)kRows * D + 2 * kRows * kHidden + kRows); }

}  // namespace

struct ngap_mlp {
  int device = 0, D = 0;
  Layout L{1, kHidden};
  uint64_t seed = 0;
  std::mt19937_64 rng;
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr, *loss = nullptr;
  __nv_bfloat16* Pb = nullptr;
  bool pb_stale = true;          // Pb needs converting from P
  // host copy of P for ngap_mlp_predict_host, and its bfloat16-rounded copy
  std::vector<float> hP, hPb;
  bool host_stale = true;
  int64_t steps = 0;
  // inference buffers (grow only) and the model's own stream, so that
  // predictions neither allocate nor order against other streams once warm
  float *ix = nullptr, *iy = nullptr;
  int64_t icap = 0;
  cudaStream_t st = nullptr;
  ~ngap_mlp() {
    cudaFree(P);
    cudaFree(G);
    cudaFree(M);
    cudaFree(V);
    cudaFree(loss);
    cudaFree(Pb);
    cudaFree(ix);
    cudaFree(iy);
    if (st) cudaStreamDestroy(st);
  }
};

extern "C" {

int ngap_features(const uint8_t* data, uint64_t bytes, int on_device, const uint64_t* offsets,
                  const uint64_t* lengths, int n, int window, float* out, void* stream) {
  if (n < 0 || (n > 0 && (!data || !offsets || !lengths || !out)) || window < 1) {
    ngap::set_error("ngap_features: bad argument");
    return NGAP_E_INVALID;
  }
  for (int i = 0; i < n; i++)
    if (offsets[i] > bytes || lengths[i] > bytes - offsets[i]) {  // no wrap-around
      ngap::set_error("ngap_features: region %d is out of range", i);
      return NGAP_E_INVALID;
    }
  if (n == 0) return NGAP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint8_t* d_data = nullptr;
  uint64_t *d_off = nullptr, *d_len = nullptr;
  float* d_out = nullptr;
  auto cleanup = [&]() {
    if (!on_device) cudaFree(d_data);
    cudaFree(d_off);
    cudaFree(d_len);
    cudaFree(d_out);
  };
  cudaError_t ce = cudaSuccess;
  if (on_device) {
    d_data = const_cast<uint8_t*>(data);
  } else {
    ce = cudaMalloc(&d_data, std::max<uint64_t>(bytes, 1));
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_data, data, bytes, cudaMemcpyHostToDevice, st);
  }
  if (ce == cudaSuccess) ce = cudaMalloc(&d_off, n * sizeof(uint64_t));
  if (ce == cudaSuccess) ce = cudaMalloc(&d_len, n * sizeof(uint64_t));
  if (ce == cudaSuccess) ce = cudaMalloc(&d_out, (size_t)n * NGAP_FEAT_BYTES * sizeof(float));
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(d_off, offsets, n * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(d_len, lengths, n * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) {
    features_kernel<<<n, kFeatThreads, 0, st>>>(d_data, d_off, d_len, n, window, d_out);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(out, d_out, (size_t)n * NGAP_FEAT_BYTES * sizeof(float),
                         cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  cleanup();
  if (ce != cudaSuccess) {
    ngap::set_error("ngap_features: %s", cudaGetErrorString(ce));
    return NGAP_E_CUDA;
  }
  return NGAP_OK;
}

int ngap_mlp_create(int device, int in_dim, int hidden, uint64_t seed, ngap_mlp** out) {
  if (!out || in_dim < 1 || in_dim > kMaxIn || hidden != kHidden) {
    ngap::set_error("ngap_mlp_create: in_dim must be 1..%d and hidden %d", kMaxIn, kHidden);
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  CM_TRY(cudaSetDevice(device));
  std::unique_ptr<ngap_mlp> m(new ngap_mlp());
  m->device = device;
  m->D = in_dim;
  m->L = Layout(in_dim, kHidden);
  m->seed = seed;
  m->rng.seed(seed);
  const size_t n = m->L.total;
  CM_TRY(cudaMalloc(&m->P, n * sizeof(float)));
  CM_TRY(cudaMalloc(&m->G, n * sizeof(float)));
  CM_TRY(cudaMalloc(&m->M, n * sizeof(float)));
  CM_TRY(cudaMalloc(&m->V, n * sizeof(float)));
  CM_TRY(cudaMalloc(&m->loss, sizeof(float)));
  CM_TRY(cudaMalloc(&m->Pb, n * sizeof(__nv_bfloat16)));
  CM_TRY(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
  CM_TRY(cudaMemset(m->G, 0, n * sizeof(float)));
  CM_TRY(cudaMemset(m->M, 0, n * sizeof(float)));
  CM_TRY(cudaMemset(m->V, 0, n * sizeof(float)));
  // He initialisation of the weights, zero biases
  std::vector<float> h(n, 0.f);
  std::normal_distribution<float> nd(0.f, 1.f);
  const Layout& L = m->L;
  for (size_t i = 0; i < (size_t)in_dim * kHidden; i++) h[L.w1 + i] = nd(m->rng) * sqrtf(2.f / in_dim);
  for (size_t i = 0; i < (size_t)kHidden * kHidden; i++) h[L.w2 + i] = nd(m->rng) * sqrtf(2.f / kHidden);
  for (size_t i = 0; i < (size_t)kHidden; i++) h[L.w3 + i] = nd(m->rng) * sqrtf(1.f / kHidden);
  CM_TRY(cudaMemcpy(m->P, h.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  CM_TRY(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)grad_smem(kMaxIn)));
  CM_TRY(cudaFuncSetAttribute(mlp_infer_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)infer_smem(kMaxIn)));
  CM_TRY(cudaFuncSetAttribute(mlp_infer_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)infer_smem(kMaxIn)));
  *out = m.release();
  return NGAP_OK;
}

void ngap_mlp_destroy(ngap_mlp* m) { delete m; }

int ngap_mlp_train(ngap_mlp* m, const float* x, const float* y, int64_t n, int epochs, int batch,
                   float lr, float* loss) {
  if (!m || !x || !y || n < 1 || epochs < 1 || batch < 1 || n > (int64_t)1 << 30) {
    ngap::set_error("ngap_mlp_train: bad argument");
    return NGAP_E_INVALID;
  }
  CM_TRY(cudaSetDevice(m->device));
  float *dx = nullptr, *dy = nullptr;
  int* didx = nullptr;
  auto cleanup = [&]() {
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(didx);
  };
  cudaError_t ce = cudaMalloc(&dx, (size_t)n * m->D * sizeof(float));
  if (ce == cudaSuccess) ce = cudaMalloc(&dy, (size_t)n * sizeof(float));
  if (ce == cudaSuccess) ce = cudaMalloc(&didx, (size_t)n * sizeof(int));
  if (ce == cudaSuccess)
    ce = cudaMemcpy(dx, x, (size_t)n * m->D * sizeof(float), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(dy, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  std::vector<int> idx(n);
  for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
  float last = 0.f;
  const size_t smem = grad_smem(m->D);
  for (int ep = 0; ep < epochs && ce == cudaSuccess; ep++) {
    std::shuffle(idx.begin(), idx.end(), m->rng);
    ce = cudaMemcpy(didx, idx.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(m->loss, 0, sizeof(float));
    for (int64_t b = 0; b < n && ce == cudaSuccess; b += batch) {
      const int nb = (int)std::min<int64_t>(batch, n - b);
      mlp_grad_kernel<<<(nb + kRows - 1) / kRows, kMlpThreads, smem>>>(
          m->P, m->D, dx, dy, didx + b, nb, 1.f / nb, m->G, m->loss);
      m->steps++;
      const float c1 = 1.f / (1.f - powf(0.9f, (float)m->steps));
      const float c2 = 1.f / (1.f - powf(0.999f, (float)m->steps));
      adam_kernel<<<64, 256>>>(m->P, m->G, m->M, m->V, m->L.total, lr, c1, c2);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(&last, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
  }
  cleanup();
  if (ce != cudaSuccess) {
    ngap::set_error("ngap_mlp_train: %s", cudaGetErrorString(ce));
    return NGAP_E_CUDA;
  }
  m->pb_stale = m->host_stale = true;
  if (loss) *loss = last / (float)n;
  return NGAP_OK;
}

int ngap_mlp_gradient(ngap_mlp* m, const float* x, const float* y, int64_t n, float* grad,
                      float* loss) {
  if (!m || !x || !y || !grad || n < 1 || n > (int64_t)1 << 30) {
    ngap::set_error("ngap_mlp_gradient: bad argument");
    return NGAP_E_INVALID;
  }
  CM_TRY(cudaSetDevice(m->device));
  float *dx = nullptr, *dy = nullptr;
  int* didx = nullptr;
  auto cleanup = [&]() {
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(didx);
  };
  std::vector<int> idx(n);
  for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
  cudaError_t ce = cudaMalloc(&dx, (size_t)n * m->D * sizeof(float));
  if (ce == cudaSuccess) ce = cudaMalloc(&dy, (size_t)n * sizeof(float));
  if (ce == cudaSuccess) ce = cudaMalloc(&didx, (size_t)n * sizeof(int));
  if (ce == cudaSuccess)
    ce = cudaMemcpy(dx, x, (size_t)n * m->D * sizeof(float), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(dy, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess)
    ce = cudaMemcpy(didx, idx.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemset(m->loss, 0, sizeof(float));
  if (ce == cudaSuccess) ce = cudaMemset(m->G, 0, m->L.total * sizeof(float));
  if (ce == cudaSuccess) {
    mlp_grad_kernel<<<(unsigned)((n + kRows - 1) / kRows), kMlpThreads, grad_smem(m->D)>>>(
        m->P, m->D, dx, dy, didx, (int)n, 1.f / (float)n, m->G, m->loss);
    ce = cudaGetLastError();
  }
  float l = 0.f;
  if (ce == cudaSuccess) ce = cudaMemcpy(grad, m->G, m->L.total * sizeof(float), cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess) ce = cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess) ce = cudaMemset(m->G, 0, m->L.total * sizeof(float));
  cleanup();
  if (ce != cudaSuccess) {
    ngap::set_error("ngap_mlp_gradient: %s", cudaGetErrorString(ce));
    return NGAP_E_CUDA;
  }
  if (loss) *loss = l / (float)n;
  return NGAP_OK;
}

int ngap_mlp_predict(ngap_mlp* m, const float* x, int64_t n, int bf16, float* y) {
  if (!m || !x || !y || n < 0) {
    ngap::set_error("ngap_mlp_predict: bad argument");
    return NGAP_E_INVALID;
  }
  if (n == 0) return NGAP_OK;
  CM_TRY(cudaSetDevice(m->device));
  if (n > m->icap) {
    const int64_t cap = std::max<int64_t>(n, 1024);
    cudaFree(m->ix);
    cudaFree(m->iy);
    m->ix = m->iy = nullptr;
    m->icap = 0;
    CM_TRY(cudaMalloc(&m->ix, (size_t)cap * m->D * sizeof(float)));
    CM_TRY(cudaMalloc(&m->iy, (size_t)cap * sizeof(float)));
    m->icap = cap;
  }
  cudaStream_t st = m->st;
  CM_TRY(cudaMemcpyAsync(m->ix, x, (size_t)n * m->D * sizeof(float), cudaMemcpyHostToDevice, st));
  const unsigned grid = (unsigned)((n + kRows - 1) / kRows);
  if (bf16) {
    if (m->pb_stale) {
      to_bf16_kernel<<<64, 256, 0, st>>>(m->P, m->Pb, m->L.total);
      m->pb_stale = false;
    }
    mlp_infer_kernel<true><<<grid, kMlpThreads, infer_smem(m->D), st>>>(m->Pb, m->D, m->ix, n, m->iy);
  } else {
    mlp_infer_kernel<false><<<grid, kMlpThreads, infer_smem(m->D), st>>>(m->P, m->D, m->ix, n, m->iy);
  }
  CM_TRY(cudaGetLastError());
  CM_TRY(cudaMemcpyAsync(y, m->iy, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CM_TRY(cudaStreamSynchronize(st));
  return NGAP_OK;
}

int ngap_mlp_get_params(const ngap_mlp* m, float* out, int64_t cap, int64_t* n) {
  if (!m || !n) {
    ngap::set_error("ngap_mlp_get_params: bad argument");
    return NGAP_E_INVALID;
  }
  *n = (int64_t)m->L.total;
  if (!out) return NGAP_OK;
  if (cap < *n) {
    ngap::set_error("ngap_mlp_get_params: %lld parameters, room for %lld", (long long)*n,
                    (long long)cap);
    return NGAP_E_INVALID;
  }
  CM_TRY(cudaSetDevice(m->device));
  CM_TRY(cudaMemcpy(out, m->P, m->L.total * sizeof(float), cudaMemcpyDeviceToHost));
  return NGAP_OK;
}

int ngap_mlp_set_params(ngap_mlp* m, const float* in, int64_t n) {
  if (!m || !in || n != (int64_t)m->L.total) {
    ngap::set_error("ngap_mlp_set_params: expected %lld parameters",
                    m ? (long long)m->L.total : 0ll);
    return NGAP_E_INVALID;
  }
  CM_TRY(cudaSetDevice(m->device));
  CM_TRY(cudaMemcpy(m->P, in, m->L.total * sizeof(float), cudaMemcpyHostToDevice));
  m->pb_stale = m->host_stale = true;
  return NGAP_OK;
}

int ngap_mlp_predict_host(ngap_mlp* m, const float* x, int64_t n, int bf16, float* y) {
  if (!m || (n > 0 && (!x || !y)) || n < 0) {
    ngap::set_error("ngap_mlp_predict_host: bad argument");
    return NGAP_E_INVALID;
  }
  if (n == 0) return NGAP_OK;
  if (m->host_stale) {  // the parameters changed (training, set_params): fetch them once
    CM_TRY(cudaSetDevice(m->device));
    m->hP.resize(m->L.total);
    CM_TRY(cudaMemcpy(m->hP.data(), m->P, m->L.total * sizeof(float), cudaMemcpyDeviceToHost));
    m->hPb.resize(m->L.total);
    for (size_t i = 0; i < m->L.total; i++) m->hPb[i] = bf16_round(m->hP[i]);
    m->host_stale = false;
  }
  const Layout& L = m->L;
  const float* P = bf16 ? m->hPb.data() : m->hP.data();
  auto rnd = [bf16](float v) { return bf16 ? bf16_round(v) : v; };
  std::vector<float> xs(L.D);
  float h1[kHidden], h2[kHidden];
  for (int64_t s = 0; s < n; s++) {
    for (int d = 0; d < L.D; d++) xs[d] = rnd(x[(size_t)s * L.D + d]);
    // the kernel's accumulation order per unit (bias, then inputs ascending),
    // with products rounded apart: a fused multiply-add without hardware
    // support is a library call per term, tens of microseconds per row
    for (int j = 0; j < kHidden; j++) h1[j] = P[L.b1 + j];
    for (int d = 0; d < L.D; d++) {
      const float xv = xs[d];
      const float* wr = P + L.w1 + (size_t)d * kHidden;
      for (int j = 0; j < kHidden; j++) h1[j] += xv * wr[j];
    }
    for (int j = 0; j < kHidden; j++) h1[j] = rnd(std::max(h1[j], 0.f));
    for (int j = 0; j < kHidden; j++) h2[j] = P[L.b2 + j];
    for (int i = 0; i < kHidden; i++) {
      const float hv = h1[i];
      const float* wr = P + L.w2 + (size_t)i * kHidden;
      for (int j = 0; j < kHidden; j++) h2[j] += hv * wr[j];
    }
    for (int j = 0; j < kHidden; j++) h2[j] = rnd(std::max(h2[j], 0.f));
    float acc = 0.f;
    for (int i = 0; i < kHidden; i++) acc += h2[i] * P[L.w3 + i];
    y[s] = acc + P[L.b3];
  }
  return NGAP_OK;
}

}  // extern "C"
