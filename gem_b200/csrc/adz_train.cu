// Training of the learned starting guess (adz_guess.cu): forward and backward
// passes of the 82 -> 128 -> 128 -> 3 GELU network in FP32, mean squared
// error on the departure displacement, Adam.  Hand-written: one tiled SIMT
// GEMM with selectable strides (so X.W^T, dY^T.A and dY.W need no transposed
// copies) and fused epilogues (bias + GELU, GELU', split-K accumulation),
// a column-sum for the bias gradients and an elementwise Adam step.  The
// arithmetic is restated in oracle/guess_oracle.py (forward, backward,
// adam_step), against which the gradients are checked.
//
// Parameter vector (FP32): W1 (128x82, row = output), b1, W2 (128x128), b2,
// W3 (3x128), b3; gradients and Adam moments share the layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>

#include "../../include/adz_b200.h"
#include "adz_internal.h"

namespace {

constexpr int F = ADZC_GUESS_NFEAT, H = ADZC_GUESS_HIDDEN, O = ADZC_GUESS_NOUT;
constexpr int oW1 = 0, oB1 = oW1 + H * F, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H, oB3 = oW3 + O * H;
constexpr int kNParam = oB3 + O;
static_assert(kNParam == ADZC_MLP_NPARAM, "parameter count");

__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

enum Epi { kStore = 0, kBias = 1, kBiasGelu = 2, kDGelu = 3, kAtomic = 4 };

constexpr int BM = 64, BN = 64, BK = 16;

// C[M x N] (ldc) <- epilogue(op(A) . op(B)), A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn]; blockIdx.z takes K in chunks of kchunk
template <int EPI>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, int kchunk, const float* __restrict__ A,
                                              long long sam, long long sak, const float* __restrict__ B,
                                              long long sbk, long long sbn, float* __restrict__ C, int ldc,
                                              const float* __restrict__ bias, float* __restrict__ Hout,
                                              const float* __restrict__ Hin) {
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = tid + q * 256;  // 0..1023 over a 64 x 16 tile
      {
        const int mm = e % BM, kk = e / BM;
        const int m = m0 + mm, k = k0 + kk;
        As[kk][mm] = (m < M && k < ke) ? A[m * sam + k * sak] : 0.0f;
      }
      {
        const int nn = e % BN, kk = e / BN;
        const int n = n0 + nn, k = k0 + kk;
        Bs[kk][nn] = (n < N && k < ke) ? B[k * sbk + n * sbn] : 0.0f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        a[q] = As[kk][ty * 4 + q];
        b[q] = Bs[kk][tx * 4 + q];
      }
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int m = m0 + ty * 4 + r;
    if (m >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int n = n0 + tx * 4 + c;
      if (n >= N) continue;
      const long long o = (long long)m * ldc + n;
      const float v = acc[r][c];
      if (EPI == kStore) C[o] = v;
      if (EPI == kBias) C[o] = v + bias[n];
      if (EPI == kBiasGelu) {
        const float h = v + bias[n];
        Hout[o] = h;
        C[o] = gelu(h);
      }
      if (EPI == kDGelu) C[o] = v * gelu_grad(Hin[o]);
      if (EPI == kAtomic) atomicAdd(C + o, v);
    }
  }
}

// out[n] += sum over rows of D[m*N + n]
__global__ void __launch_bounds__(256) k_colsum(const float* __restrict__ D, int M, int N, float* __restrict__ out) {
  __shared__ float red[8][33];
  const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
  const int n = blockIdx.x * 32 + cx;
  float s = 0.0f;
  if (n < N)
    for (int m = blockIdx.y * 256 + ry; m < min(M, (int)(blockIdx.y + 1) * 256); m += 8) s += D[(long long)m * N + n];
  red[ry][cx] = s;
  __syncthreads();
  if (ry == 0 && n < N) {
    float t = 0.0f;
    for (int q = 0; q < 8; q++) t += red[q][cx];
    atomicAdd(out + n, t);
  }
}

// dY = 2 (Y - T) / B; loss += sum (Y - T)^2 / B
__global__ void __launch_bounds__(256) k_loss(const float* __restrict__ Y, const float* __restrict__ T, int n,
                                              float inv_b, float* __restrict__ dY, float* __restrict__ loss) {
  float s = 0.0f;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const float d = Y[e] - T[e];
    dY[e] = 2.0f * inv_b * d;
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_b);
}

__global__ void __launch_bounds__(256) k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                              const float* __restrict__ g, int n, float lr, float b1, float b2,
                                              float c1, float c2, float eps) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gi = g[e];
  const float mi = b1 * m[e] + (1.0f - b1) * gi;
  const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
  m[e] = mi;
  v[e] = vi;
  p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

template <int EPI>
cudaError_t gemm(cudaStream_t s, int M, int N, int K, int kchunk, const float* A, long long sam, long long sak,
                 const float* B, long long sbk, long long sbn, float* C, int ldc, const float* bias = nullptr,
                 float* Hout = nullptr, const float* Hin = nullptr) {
  if (kchunk <= 0) kchunk = K;
  const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, (K + kchunk - 1) / kchunk);
  k_gemm<EPI><<<grid, 256, 0, s>>>(M, N, K, kchunk, A, sam, sak, B, sbk, sbn, C, ldc, bias, Hout, Hin);
  return cudaGetLastError();
}

}  // namespace

struct adzc_mlp {
  int max_batch = 0;
  long long step = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float *h1 = nullptr, *a1 = nullptr, *h2 = nullptr, *a2 = nullptr, *y = nullptr, *dy = nullptr;
  float *d2 = nullptr, *d1 = nullptr, *loss = nullptr;
};

extern "C" int adzc_mlp_destroy(adzc_mlp* t) {
  if (!t) return ADZC_OK;
  for (float* q : {t->p, t->g, t->m, t->v, t->h1, t->a1, t->h2, t->a2, t->y, t->dy, t->d2, t->d1, t->loss})
    cudaFree(q);
  delete t;
  return ADZC_OK;
}

extern "C" int adzc_mlp_create(const float* params, int max_batch, adzc_mlp** out) {
  if (!params || !out || max_batch < 1 || max_batch > (1 << 22)) return adz_internal_fail(ADZC_ERR_ARG);
  auto* t = new (std::nothrow) adzc_mlp();
  if (!t) return adz_internal_fail(ADZC_ERR_ALLOC);
  t->max_batch = max_batch;
  const size_t P = kNParam * sizeof(float), BH = (size_t)max_batch * H * sizeof(float);
  const size_t BO = (size_t)max_batch * O * sizeof(float);
  bool ok = cudaMalloc(&t->p, P) == cudaSuccess && cudaMalloc(&t->g, P) == cudaSuccess &&
            cudaMalloc(&t->m, P) == cudaSuccess && cudaMalloc(&t->v, P) == cudaSuccess &&
            cudaMalloc(&t->h1, BH) == cudaSuccess && cudaMalloc(&t->a1, BH) == cudaSuccess &&
            cudaMalloc(&t->h2, BH) == cudaSuccess && cudaMalloc(&t->a2, BH) == cudaSuccess &&
            cudaMalloc(&t->d2, BH) == cudaSuccess && cudaMalloc(&t->d1, BH) == cudaSuccess &&
            cudaMalloc(&t->y, BO) == cudaSuccess && cudaMalloc(&t->dy, BO) == cudaSuccess &&
            cudaMalloc(&t->loss, sizeof(float)) == cudaSuccess;
  if (!ok) {
    adzc_mlp_destroy(t);
    return adz_internal_fail(ADZC_ERR_ALLOC);
  }
  ok = cudaMemcpy(t->p, params, P, cudaMemcpyHostToDevice) == cudaSuccess && cudaMemset(t->m, 0, P) == cudaSuccess &&
       cudaMemset(t->v, 0, P) == cudaSuccess && cudaMemset(t->g, 0, P) == cudaSuccess &&
       cudaMemset(t->loss, 0, sizeof(float)) == cudaSuccess;
  if (!ok) {
    adzc_mlp_destroy(t);
    return adz_internal_fail(ADZC_ERR_CUDA);
  }
  *out = t;
  return ADZC_OK;
}

// forward pass of a batch into the trainer's activations; y (batch x 3) kept
static cudaError_t forward(adzc_mlp* t, const float* x, int b, cudaStream_t s) {
  const float* P = t->p;
  cudaError_t e;
  if ((e = gemm<kBiasGelu>(s, b, H, F, 0, x, F, 1, P + oW1, 1, F, t->a1, H, P + oB1, t->h1)) != cudaSuccess) return e;
  if ((e = gemm<kBiasGelu>(s, b, H, H, 0, t->a1, H, 1, P + oW2, 1, H, t->a2, H, P + oB2, t->h2)) != cudaSuccess)
    return e;
  return gemm<kBias>(s, b, O, H, 0, t->a2, H, 1, P + oW3, 1, H, t->y, O, P + oB3);
}

extern "C" int adzc_mlp_forward(adzc_mlp* t, const float* x, int batch, float* y, void* stream) {
  if (!t || !x || !y || batch < 1 || batch > t->max_batch) return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  if (forward(t, x, batch, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  if (cudaMemcpyAsync(y, t->y, (size_t)batch * O * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return adz_internal_fail(ADZC_ERR_CUDA);
  return ADZC_OK;
}

extern "C" int adzc_mlp_grad(adzc_mlp* t, const float* x, const float* target, int batch, void* stream) {
  if (!t || !x || !target || batch < 1 || batch > t->max_batch) return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  const int b = batch;
  const float* P = t->p;
  float* G = t->g;
  const int kc = 256;  // split-K chunk of the weight gradients (sum over the batch)
  bool ok = cudaMemsetAsync(G, 0, kNParam * sizeof(float), s) == cudaSuccess &&
            cudaMemsetAsync(t->loss, 0, sizeof(float), s) == cudaSuccess && forward(t, x, b, s) == cudaSuccess;
  if (ok) {
    const int n = b * O;
    k_loss<<<std::min(1024, (n + 255) / 256), 256, 0, s>>>(t->y, target, n, 1.0f / (float)b, t->dy, t->loss);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && gemm<kAtomic>(s, O, H, b, kc, t->dy, 1, O, t->a2, H, 1, G + oW3, H) == cudaSuccess;
  if (ok) {
    k_colsum<<<dim3(1, (b + 255) / 256), 256, 0, s>>>(t->dy, b, O, G + oB3);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && gemm<kDGelu>(s, b, H, O, 0, t->dy, O, 1, P + oW3, H, 1, t->d2, H, nullptr, nullptr, t->h2) == cudaSuccess;
  ok = ok && gemm<kAtomic>(s, H, H, b, kc, t->d2, 1, H, t->a1, H, 1, G + oW2, H) == cudaSuccess;
  if (ok) {
    k_colsum<<<dim3(H / 32, (b + 255) / 256), 256, 0, s>>>(t->d2, b, H, G + oB2);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && gemm<kDGelu>(s, b, H, H, 0, t->d2, H, 1, P + oW2, H, 1, t->d1, H, nullptr, nullptr, t->h1) == cudaSuccess;
  ok = ok && gemm<kAtomic>(s, H, F, b, kc, t->d1, 1, H, x, F, 1, G + oW1, F) == cudaSuccess;
  if (ok) {
    k_colsum<<<dim3(H / 32, (b + 255) / 256), 256, 0, s>>>(t->d1, b, H, G + oB1);
    ok = cudaGetLastError() == cudaSuccess;
  }
  return ok ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

extern "C" int adzc_mlp_adam(adzc_mlp* t, float lr, void* stream) {
  if (!t || !(lr > 0.0f)) return adz_internal_fail(ADZC_ERR_ARG);
  t->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 - std::pow(0.9, (double)t->step)), c2 = (float)(1.0 - std::pow(0.999, (double)t->step));
  k_adam<<<(kNParam + 255) / 256, 256, 0, (cudaStream_t)stream>>>(t->p, t->m, t->v, t->g, kNParam, lr, b1, b2, c1, c2,
                                                                  1e-8f);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

extern "C" int adzc_mlp_read(adzc_mlp* t, int what, float* host_out, void* stream) {
  if (!t || !host_out || what < 0 || what > 2) return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  const float* src = what == 0 ? t->p : what == 1 ? t->g : t->loss;
  const size_t n = what == 2 ? 1 : kNParam;
  if (cudaMemcpyAsync(host_out, src, n * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return adz_internal_fail(ADZC_ERR_CUDA);
  return ADZC_OK;
}
