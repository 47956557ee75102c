// Proposal network of the learned Wyckoff search: a 3-layer MLP
// (d_in -> width -> width -> d_out, ReLU), trained on the GPU by the
// kernels below on (state, move, fitness change) records the plain search
// writes, and used to pre-rank batched proposals.  The exact structure-factor
// fitness still decides every acceptance.
//
// Training keeps FP32 master weights with Adam; its products are one
// strided, tiled SIMT GEMM (64 x 64 tiles, 4 x 4 per thread) with a bias /
// ReLU / accumulate epilogue, so forward, backward (A^T B and A B^T) and the
// masked-MSE gradient share one kernel.  Inference -- tens of thousands of
// candidate rows per search generation -- runs the two hidden layers on the
// tensor cores: bf16 activations and weights, tcgen05.mma into a TMEM
// accumulator (one 128 x 256 tile per CTA, all K-blocks staged by TMA at
// once), bias and ReLU applied by the epilogue warps, bf16 out; the output
// layer (width -> d_out) is a warp-per-row dot product.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mlp_internal.h"
#include "p6_common.cuh"
#include "tc_common.cuh"

namespace p6 {
namespace mlp {

constexpr int TM = 64, TN = 64, TK = 16;

// C[i][j] = act(sum_k A(i,k) B(k,j) + bias[j]) (+ C[i][j] when accumulate)
// A(i,k) = A[i*sa0 + k*sa1], B(k,j) = B[k*sb0 + j*sb1], C row-major ldc.
template <typename BT>
__global__ void __launch_bounds__(256) gemm_kernel(const float *A, long sa0, long sa1, const BT *B, long sb0, long sb1,
                                                   float *C, int ldc, int M, int N, int K, const float *bias, int relu,
                                                   int accumulate) {
  __shared__ float As[TK][TM + 4], Bs[TK][TN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = threadIdx.x; e < TM * TK; e += 256) {
      const int r = e / TK, k = e % TK;
      const int gi = m0 + r, gk = k0 + k;
      As[k][r] = (gi < M && gk < K) ? A[gi * sa0 + gk * sa1] : 0.f;
    }
    for (int e = threadIdx.x; e < TN * TK; e += 256) {
      const int c = e % TN, k = e / TN;
      const int gj = n0 + c, gk = k0 + k;
      Bs[k][c] = (gj < N && gk < K) ? (float)B[gk * sb0 + gj * sb1] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TK; ++k) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[k][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gi = m0 + ty * 4 + i;
    if (gi >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gj = n0 + tx * 4 + j;
      if (gj >= N) continue;
      float v = acc[i][j] + (bias ? bias[gj] : 0.f);
      if (relu) v = fmaxf(v, 0.f);
      float *c = C + (size_t)gi * ldc + gj;
      *c = accumulate ? *c + v : v;
    }
  }
}

// dY = 2 (Y - T) mask / n  (masked mean-squared error), loss partials per block.
__global__ void mse_grad_kernel(const float *Y, const float *T, const float *mask, int n, int d, float *dY,
                                float *lossOut) {
  __shared__ float part[256];
  float l = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * d; i += gridDim.x * blockDim.x) {
    const float m = mask ? mask[i] : 1.f;
    const float e = (Y[i] - T[i]) * m;
    dY[i] = 2.f * e / (float)n;
    l += e * e;
  }
  part[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(lossOut, part[0] / (float)n);
}

// dH *= (H > 0)
__global__ void relu_mask_kernel(float *dH, const float *H, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!(H[i] > 0.f)) dH[i] = 0.f;
}

// db[j] = sum_i dY[i][j]
__global__ void bias_grad_kernel(const float *dY, int n, int d, float *db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d) return;
  float s = 0.f;
  for (int i = 0; i < n; ++i) s += dY[(size_t)i * d + j];
  db[j] = s;
}

__global__ void adam_kernel(float *w, const float *g, float *m, float *v, size_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, __nv_bfloat16 *wh) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wh) wh[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16_kernel(const float *w, __nv_bfloat16 *wh, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    wh[i] = __float2bfloat16_rn(w[i]);
}

// ---------------------------------------------------------------------------
// Inference on the tensor cores.
// ---------------------------------------------------------------------------
constexpr int LBM = 128, LBN = 256;                 // one tile: 128 rows x the full width
constexpr int L_A = LBM * 64 * 2, L_B = LBN * 64 * 2;  // bytes of one K-block of A and of B
constexpr uint32_t kLayerIdesc = tc::idesc_bf16(LBM, LBN);

// out[r][n] = act(sum_k A[r][k] W[k][n] + bias[n]) for one 128-row tile, with
// B = W^T (width x K, K-major) in bf16; KB K-blocks of 64, all loaded at once.
template <int KB>
__global__ void __launch_bounds__(128, 1) layer_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                                                          const __grid_constant__ CUtensorMap tmB, const float *bias,
                                                          __nv_bfloat16 *out, int M, int relu, int *errFlag) {
  using namespace p6::tc;
  extern __shared__ unsigned char smemRaw[];
  __shared__ __align__(8) uint64_t fullBar, accBar;
  __shared__ uint32_t tmemBase;
  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, m0 = blockIdx.x * LBM;
  if (threadIdx.x == 0) {
    mbar_init(&fullBar, 1);
    mbar_init(&accBar, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemBase)),
                 "r"((uint32_t)LBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmemBase;
  bool loaded = true;
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&fullBar, (uint32_t)KB * (L_A + L_B));
    for (int kb = 0; kb < KB; ++kb) {
      tma_load_2d(smem + kb * L_A, &tmA, kb * 64, m0, &fullBar);
      tma_load_2d(smem + KB * L_A + kb * L_B, &tmB, kb * 64, 0, &fullBar);
    }
    loaded = wait_phase(&fullBar, 0);
    if (!loaded) {
      raise_flag(errFlag, 21);
      wait_phase(&fullBar, 0);              // copies in flight land before the CTA moves on
    } else {
      fence_after_sync();
      const uint32_t base = smem_u32(smem);
      for (int kb = 0; kb < KB; ++kb)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint64_t a = smem_desc(base + kb * L_A + k * 32), b = smem_desc(base + KB * L_A + kb * L_B + k * 32);
          umma_bf16(tmem, a, b, kLayerIdesc, (kb > 0 || k > 0) ? 1u : 0u);
        }
      umma_commit(&accBar);
    }
    if (!loaded) mbar_arrive(&accBar);
  }
  const bool ok = __all_sync(0xffffffffu, wait_phase(&accBar, 0));
  if (!ok && lane == 0) raise_flag(errFlag, 22);
  fence_after_sync();
  const int row = m0 + warp * 32 + lane;
  for (int c = 0; c < LBN; c += 64) {
    float v[64];
    tmem_ld64(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (row < M && ok) {
      __align__(16) __nv_bfloat16 h[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        float x = v[j] + bias[c + j];
        if (relu) x = fmaxf(x, 0.f);
        h[j] = __float2bfloat16_rn(x);
      }
      uint4 *dst = reinterpret_cast<uint4 *>(out + (size_t)row * LBN + c);
#pragma unroll
      for (int q = 0; q < 8; ++q) dst[q] = reinterpret_cast<const uint4 *>(h)[q];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)LBN) : "memory");
  }
}

// y[r][o] = sum_k H[r][k] W3[k][o] + b3[o]: one warp per row.
__global__ void out_layer_kernel(const __nv_bfloat16 *H, int rows, int width, const float *W3, const float *b3,
                                 int dOut, float *Y) {
  const int warpsPerBlock = blockDim.x >> 5;
  const int r = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= rows) return;
  for (int o = 0; o < dOut; ++o) {
    float acc = 0.f;
    for (int k = lane; k < width; k += 32) acc = fmaf(__bfloat162float(H[(size_t)r * width + k]), W3[k * dOut + o], acc);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
    if (lane == 0) Y[(size_t)r * dOut + o] = acc + b3[o];
  }
}

__global__ void rows_to_bf16_kernel(const float *X, size_t n, __nv_bfloat16 *Xh) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    Xh[i] = __float2bfloat16_rn(X[i]);
}

// Wt[n][k] = bf16(W[k][n]): the K-major operand copy of a K x N weight matrix.
__global__ void transpose_bf16_kernel(const float *W, int K, int N, __nv_bfloat16 *Wt) {
  const size_t total = (size_t)K * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(i / K), k = (int)(i % K);
    Wt[i] = __float2bfloat16_rn(W[(size_t)k * N + n]);
  }
}

template <typename BT>
void gemm(cudaStream_t st, const float *A, long sa0, long sa1, const BT *B, long sb0, long sb1, float *C, int ldc,
          int M, int N, int K, const float *bias, bool relu, bool accumulate) {
  const dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  gemm_kernel<BT><<<grid, 256, 0, st>>>(A, sa0, sa1, B, sb0, sb1, C, ldc, M, N, K, bias, relu ? 1 : 0,
                                        accumulate ? 1 : 0);
}

}  // namespace mlp
}  // namespace p6

using namespace p6;
using namespace p6::mlp;

// Parameter block layout (flat, FP32): W1 (dIn x W), b1 (W), W2 (W x W), b2 (W), W3 (W x dOut), b3 (dOut).
struct p6_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  int dIn = 0, width = 0, dOut = 0;
  size_t nParams = 0;
  size_t off[6] = {};
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // master weights, gradients, Adam moments
  __nv_bfloat16 *wh = nullptr;                                    // inference copy
  __nv_bfloat16 *w1t = nullptr, *w2t = nullptr;                   // K-major copies for the tensor-core layers
  bool tc = false;                                                // width 256 and d_in a multiple of 64
  int tcCap = 0;
  __nv_bfloat16 *Xh = nullptr, *H1h = nullptr, *H2h = nullptr;
  int *dErr = nullptr;
  long long step = 0;
  // scratch for a batch of cap rows
  int cap = 0;
  float *X = nullptr, *T = nullptr, *Mk = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr, *dY = nullptr,
        *dH1 = nullptr, *dH2 = nullptr, *loss = nullptr;
};

static void mlp_free(p6_mlp *n) {
  if (!n) return;
  cudaSetDevice(n->device);
  if (n->stream) cudaStreamSynchronize(n->stream);
  for (void *p : {(void *)n->w1t, (void *)n->w2t, (void *)n->Xh, (void *)n->H1h, (void *)n->H2h, (void *)n->dErr})
    if (p) cudaFree(p);
  for (void *p : {(void *)n->w, (void *)n->g, (void *)n->m, (void *)n->v, (void *)n->wh, (void *)n->X, (void *)n->T,
                  (void *)n->Mk, (void *)n->H1, (void *)n->H2, (void *)n->Y, (void *)n->dY, (void *)n->dH1,
                  (void *)n->dH2, (void *)n->loss})
    if (p) cudaFree(p);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
}

// K-major bf16 copies of W1 and W2 for the tensor-core layers.
static p6_status mlp_refresh_tc(p6_mlp *n) {
  if (!n->tc) return P6_OK;
  transpose_bf16_kernel<<<256, 256, 0, n->stream>>>(n->w + n->off[0], n->dIn, n->width, n->w1t);
  transpose_bf16_kernel<<<256, 256, 0, n->stream>>>(n->w + n->off[2], n->width, n->width, n->w2t);
  P6_CUDA(cudaGetLastError());
  return P6_OK;
}

static p6_status mlp_ensure_tc(p6_mlp *n, int rows) {
  if (rows <= n->tcCap) return P6_OK;
  for (__nv_bfloat16 **p : {&n->Xh, &n->H1h, &n->H2h}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  n->tcCap = 0;
  const size_t r = ((size_t)rows + LBM - 1) / LBM * LBM;
  P6_CUDA(cudaMalloc(&n->Xh, r * n->dIn * sizeof(__nv_bfloat16)));
  P6_CUDA(cudaMalloc(&n->H1h, r * LBN * sizeof(__nv_bfloat16)));
  P6_CUDA(cudaMalloc(&n->H2h, r * LBN * sizeof(__nv_bfloat16)));
  n->tcCap = rows;
  return P6_OK;
}

template <int KB>
static cudaError_t layer_launch(const CUtensorMap &a, const CUtensorMap &b, const float *bias, __nv_bfloat16 *out,
                                int rows, int *err, cudaStream_t st) {
  // at least 100 KB of shared memory: at most two CTAs (2 x 256 TMEM columns) per SM
  const int smem = std::max(KB * (L_A + L_B) + 1024, 100 * 1024);
  cudaError_t e = cudaFuncSetAttribute(layer_tc_kernel<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  layer_tc_kernel<KB><<<(rows + LBM - 1) / LBM, 128, smem, st>>>(a, b, bias, out, rows, 1, err);
  return cudaGetLastError();
}

static p6_status mlp_ensure(p6_mlp *n, int rows) {
  if (rows <= n->cap) return P6_OK;
  for (float **p : {&n->X, &n->T, &n->Mk, &n->H1, &n->H2, &n->Y, &n->dY, &n->dH1, &n->dH2}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  n->cap = 0;
  const size_t r = rows;
  P6_CUDA(cudaMalloc(&n->X, r * n->dIn * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->T, r * n->dOut * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->Mk, r * n->dOut * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->H1, r * n->width * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->H2, r * n->width * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->Y, r * n->dOut * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->dY, r * n->dOut * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->dH1, r * n->width * sizeof(float)));
  P6_CUDA(cudaMalloc(&n->dH2, r * n->width * sizeof(float)));
  n->cap = rows;
  return P6_OK;
}

namespace p6 {
namespace mlp {
// Forward pass of `rows` inputs at dX (device) into dY (device); bf16 weights
// when `inference`, else the FP32 master weights with the activations kept.
p6_status forward_device(p6_mlp *n, const float *dX, int rows, float *dY, bool inference, float *H1, float *H2,
                         cudaStream_t st) {
  const int W = n->width;
  if (inference) {
    const __nv_bfloat16 *w = n->wh;
    gemm(st, dX, n->dIn, 1, w + n->off[0], W, 1, H1, W, rows, W, n->dIn, n->w + n->off[1], true, false);
    gemm(st, H1, W, 1, w + n->off[2], W, 1, H2, W, rows, W, W, n->w + n->off[3], true, false);
    gemm(st, H2, W, 1, w + n->off[4], n->dOut, 1, dY, n->dOut, rows, n->dOut, W, n->w + n->off[5], false, false);
  } else {
    const float *w = n->w;
    gemm(st, dX, n->dIn, 1, w + n->off[0], W, 1, H1, W, rows, W, n->dIn, w + n->off[1], true, false);
    gemm(st, H1, W, 1, w + n->off[2], W, 1, H2, W, rows, W, W, w + n->off[3], true, false);
    gemm(st, H2, W, 1, w + n->off[4], n->dOut, 1, dY, n->dOut, rows, n->dOut, W, w + n->off[5], false, false);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? P6_OK : cuda_error(e, "mlp forward");
}

p6_status predict_device(p6_mlp *n, const float *dX, int rows, float *dY, cudaStream_t st) {
  if (!n->tc) {
    p6_status s = mlp_ensure(n, rows);
    if (s != P6_OK) return s;
    return forward_device(n, dX, rows, dY, true, n->H1, n->H2, st);
  }
  p6_status s = mlp_ensure_tc(n, rows);
  if (s != P6_OK) return s;
  rows_to_bf16_kernel<<<592, 256, 0, st>>>(dX, (size_t)rows * n->dIn, n->Xh);
  CUtensorMap a1, b1, a2, b2;
  if ((s = tc::make_map(&a1, n->Xh, rows, n->dIn, LBM)) != P6_OK || (s = tc::make_map(&b1, n->w1t, LBN, n->dIn, LBN)) != P6_OK ||
      (s = tc::make_map(&a2, n->H1h, rows, LBN, LBM)) != P6_OK || (s = tc::make_map(&b2, n->w2t, LBN, LBN, LBN)) != P6_OK)
    return s;
  cudaError_t e;
  switch (n->dIn / 64) {
    case 1: e = layer_launch<1>(a1, b1, n->w + n->off[1], n->H1h, rows, n->dErr, st); break;
    case 2: e = layer_launch<2>(a1, b1, n->w + n->off[1], n->H1h, rows, n->dErr, st); break;
    case 3: e = layer_launch<3>(a1, b1, n->w + n->off[1], n->H1h, rows, n->dErr, st); break;
    default: e = layer_launch<4>(a1, b1, n->w + n->off[1], n->H1h, rows, n->dErr, st); break;
  }
  if (e == cudaSuccess) e = layer_launch<4>(a2, b2, n->w + n->off[3], n->H2h, rows, n->dErr, st);
  if (e != cudaSuccess) return cuda_error(e, "mlp tensor-core layers");
  out_layer_kernel<<<(rows + 7) / 8, 256, 0, st>>>(n->H2h, rows, LBN, n->w + n->off[4], n->w + n->off[5], n->dOut, dY);
  e = cudaGetLastError();
  return e == cudaSuccess ? P6_OK : cuda_error(e, "mlp output layer");
}

int input_dim(const p6_mlp *n) { return n->dIn; }
int output_dim(const p6_mlp *n) { return n->dOut; }
}  // namespace mlp
}  // namespace p6

// Gradients of the masked MSE over rows already in n->X, n->T, n->Mk; loss added to n->loss.
static p6_status mlp_backward(p6_mlp *n, int rows) {
  const int W = n->width;
  cudaStream_t st = n->stream;
  p6_status s = forward_device(n, n->X, rows, n->Y, false, n->H1, n->H2, st);
  if (s != P6_OK) return s;
  mse_grad_kernel<<<64, 256, 0, st>>>(n->Y, n->T, n->Mk, rows, n->dOut, n->dY, n->loss);
  float *g = n->g;
  const float *w = n->w;
  // layer 3: dW3 = H2^T dY, db3, dH2 = dY W3^T * (H2 > 0)
  gemm<float>(st, n->H2, 1, W, n->dY, n->dOut, 1, g + n->off[4], n->dOut, W, n->dOut, rows, nullptr, false, false);
  bias_grad_kernel<<<(n->dOut + 127) / 128, 128, 0, st>>>(n->dY, rows, n->dOut, g + n->off[5]);
  gemm<float>(st, n->dY, n->dOut, 1, w + n->off[4], 1, n->dOut, n->dH2, W, rows, W, n->dOut, nullptr, false, false);
  relu_mask_kernel<<<296, 256, 0, st>>>(n->dH2, n->H2, (size_t)rows * W);
  // layer 2
  gemm<float>(st, n->H1, 1, W, n->dH2, W, 1, g + n->off[2], W, W, W, rows, nullptr, false, false);
  bias_grad_kernel<<<(W + 127) / 128, 128, 0, st>>>(n->dH2, rows, W, g + n->off[3]);
  gemm<float>(st, n->dH2, W, 1, w + n->off[2], 1, W, n->dH1, W, rows, W, W, nullptr, false, false);
  relu_mask_kernel<<<296, 256, 0, st>>>(n->dH1, n->H1, (size_t)rows * W);
  // layer 1
  gemm<float>(st, n->X, 1, n->dIn, n->dH1, W, 1, g + n->off[0], W, n->dIn, W, rows, nullptr, false, false);
  bias_grad_kernel<<<(W + 127) / 128, 128, 0, st>>>(n->dH1, rows, W, g + n->off[1]);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? P6_OK : cuda_error(e, "mlp backward");
}

static p6_status mlp_upload_rows(p6_mlp *n, const float *X, const float *T, const float *mask, int rows) {
  P6_CUDA(cudaMemcpyAsync(n->X, X, (size_t)rows * n->dIn * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  if (T) P6_CUDA(cudaMemcpyAsync(n->T, T, (size_t)rows * n->dOut * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  if (mask)
    P6_CUDA(cudaMemcpyAsync(n->Mk, mask, (size_t)rows * n->dOut * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  else {
    std::vector<float> ones((size_t)rows * n->dOut, 1.f);
    P6_CUDA(cudaMemcpyAsync(n->Mk, ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    P6_CUDA(cudaStreamSynchronize(n->stream));
  }
  return P6_OK;
}

extern "C" {

p6_status p6_mlp_create(int d_in, int width, int d_out, uint32_t seed, int device, p6_mlp **out) {
  clear_error();
  if (!out || d_in <= 0 || width <= 0 || d_out <= 0) return set_error(P6_ERR_INVALID_ARG, "bad network shape");
  *out = nullptr;
  p6_mlp *n = new p6_mlp();
  n->device = device;
  n->dIn = d_in;
  n->width = width;
  n->dOut = d_out;
  const size_t sizes[6] = {(size_t)d_in * width, (size_t)width, (size_t)width * width, (size_t)width,
                           (size_t)width * d_out, (size_t)d_out};
  size_t o = 0;
  for (int i = 0; i < 6; ++i) {
    n->off[i] = o;
    o += sizes[i];
  }
  n->nParams = o;
  // He-uniform initial weights, zero biases, from a seeded host generator
  std::vector<float> h(o, 0.f);
  std::mt19937 rng(seed);
  const int fanIn[3] = {d_in, width, width};
  for (int L = 0; L < 3; ++L) {
    std::uniform_real_distribution<float> u(-std::sqrt(6.f / fanIn[L]), std::sqrt(6.f / fanIn[L]));
    for (size_t i = 0; i < sizes[2 * L]; ++i) h[n->off[2 * L] + i] = u(rng);
  }
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&n->w, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->g, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->m, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->v, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->wh, o * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMalloc(&n->loss, sizeof(float));
  n->tc = width == LBN && d_in % 64 == 0 && d_in <= 256;
  if (e == cudaSuccess && n->tc) e = cudaMalloc(&n->w1t, (size_t)d_in * width * sizeof(__nv_bfloat16));
  if (e == cudaSuccess && n->tc) e = cudaMalloc(&n->w2t, (size_t)width * width * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMalloc(&n->dErr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(n->dErr, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(n->w, h.data(), o * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(n->m, 0, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(n->v, 0, o * sizeof(float));
  if (e == cudaSuccess) {
    to_bf16_kernel<<<256, 256, 0, n->stream>>>(n->w, n->wh, o);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && mlp_refresh_tc(n) != P6_OK) e = cudaErrorUnknown;
  if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
  if (e != cudaSuccess) {
    mlp_free(n);
    return cuda_error(e, "mlp create");
  }
  *out = n;
  return P6_OK;
}

p6_status p6_mlp_destroy(p6_mlp *n) {
  clear_error();
  if (!n) return set_error(P6_ERR_INVALID_ARG, "null network");
  mlp_free(n);
  return P6_OK;
}

p6_status p6_mlp_params(p6_mlp *n, float *get, const float *set, long long *count) {
  clear_error();
  if (!n) return set_error(P6_ERR_INVALID_ARG, "null network");
  P6_CUDA(cudaSetDevice(n->device));
  if (count) *count = (long long)n->nParams;
  if (set) {
    P6_CUDA(cudaMemcpy(n->w, set, n->nParams * sizeof(float), cudaMemcpyHostToDevice));
    to_bf16_kernel<<<256, 256, 0, n->stream>>>(n->w, n->wh, n->nParams);
    P6_CUDA(cudaGetLastError());
    p6_status s = mlp_refresh_tc(n);
    if (s != P6_OK) return s;
    P6_CUDA(cudaStreamSynchronize(n->stream));
  }
  if (get) P6_CUDA(cudaMemcpy(get, n->w, n->nParams * sizeof(float), cudaMemcpyDeviceToHost));
  return P6_OK;
}

p6_status p6_mlp_gradients(p6_mlp *n, const float *X, const float *T, const float *mask, int rows, float *grad,
                           float *loss) {
  clear_error();
  if (!n || !X || !T || rows <= 0 || !grad) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(n->device));
  p6_status s = mlp_ensure(n, rows);
  if (s != P6_OK) return s;
  if ((s = mlp_upload_rows(n, X, T, mask, rows)) != P6_OK) return s;
  P6_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), n->stream));
  if ((s = mlp_backward(n, rows)) != P6_OK) return s;
  P6_CUDA(cudaMemcpyAsync(grad, n->g, n->nParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  if (loss) P6_CUDA(cudaMemcpyAsync(loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  P6_CUDA(cudaStreamSynchronize(n->stream));
  return P6_OK;
}

p6_status p6_mlp_train(p6_mlp *n, const float *X, const float *T, const float *mask, int rows, int epochs, int batch,
                       float lr, uint32_t seed, float *epoch_loss) {
  clear_error();
  if (!n || !X || !T || rows <= 0 || epochs <= 0 || batch <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(n->device));
  batch = std::min(batch, rows);
  p6_status s = mlp_ensure(n, batch);
  if (s != P6_OK) return s;
  std::vector<int> perm(rows);
  for (int i = 0; i < rows; ++i) perm[i] = i;
  std::mt19937 rng(seed);
  std::vector<float> bx((size_t)batch * n->dIn), bt((size_t)batch * n->dOut), bm((size_t)batch * n->dOut);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    P6_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), n->stream));
    int nb = 0;
    for (int b0 = 0; b0 + batch <= rows; b0 += batch, ++nb) {
      for (int i = 0; i < batch; ++i) {
        const int r = perm[b0 + i];
        std::memcpy(&bx[(size_t)i * n->dIn], X + (size_t)r * n->dIn, n->dIn * sizeof(float));
        std::memcpy(&bt[(size_t)i * n->dOut], T + (size_t)r * n->dOut, n->dOut * sizeof(float));
        if (mask) std::memcpy(&bm[(size_t)i * n->dOut], mask + (size_t)r * n->dOut, n->dOut * sizeof(float));
        else std::fill(bm.begin() + (size_t)i * n->dOut, bm.begin() + (size_t)(i + 1) * n->dOut, 1.f);
      }
      if ((s = mlp_upload_rows(n, bx.data(), bt.data(), bm.data(), batch)) != P6_OK) return s;
      if ((s = mlp_backward(n, batch)) != P6_OK) return s;
      ++n->step;
      const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
      adam_kernel<<<592, 256, 0, n->stream>>>(n->w, n->g, n->m, n->v, n->nParams, lr, b1, b2, eps, c1, c2, n->wh);
      P6_CUDA(cudaGetLastError());
      P6_CUDA(cudaStreamSynchronize(n->stream));   // the host batch buffers are reused
    }
    if (epoch_loss) {
      float l = 0.f;
      P6_CUDA(cudaMemcpy(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost));
      epoch_loss[ep] = nb ? l / nb : 0.f;
    }
  }
  s = mlp_refresh_tc(n);
  if (s != P6_OK) return s;
  P6_CUDA(cudaStreamSynchronize(n->stream));
  return P6_OK;
}

p6_status p6_mlp_predict(p6_mlp *n, const float *X, int rows, float *Y) {
  clear_error();
  if (!n || !X || !Y || rows <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(n->device));
  p6_status s = mlp_ensure(n, rows);
  if (s != P6_OK) return s;
  if ((s = mlp_upload_rows(n, X, nullptr, nullptr, rows)) != P6_OK) return s;
  if ((s = predict_device(n, n->X, rows, n->Y, n->stream)) != P6_OK) return s;
  P6_CUDA(cudaMemcpyAsync(Y, n->Y, (size_t)rows * n->dOut * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  int flag = 0;
  P6_CUDA(cudaMemcpyAsync(&flag, n->dErr, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
  P6_CUDA(cudaStreamSynchronize(n->stream));
  if (flag) {
    cudaMemset(n->dErr, 0, sizeof(int));
    return set_error(P6_ERR_TIMEOUT, "a tensor-core layer wait did not complete in time");
  }
  return P6_OK;
}

}  // extern "C"
