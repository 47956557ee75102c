// Profile contraction Y = I . P with the cell and profile fixed.
//
// When a Wyckoff search holds the cell and the profile fixed, the calculated
// pattern of every replica is the product of its reflection intensities I
// (replicas x reflections) and one banded profile matrix P (reflections x
// points): column j of P is nonzero only for the reflections whose window
// covers point j, and with the reflections sorted by 2-theta the nonzero
// rows of a run of columns form one contiguous range.
//
// The split-BF16 path runs on the 5th-generation tensor cores:
//  * I = I_hi + I_lo and P = P_hi + P_lo with bf16 parts (I_hi = bf16(I),
//    I_lo = bf16(I - I_hi)); Y = I_hi P_hi + I_hi P_lo + I_lo P_hi with FP32
//    accumulation (the dropped I_lo P_lo term is ~2^-16 relative);
//  * 128 x 256 output tiles, handed round-robin to one persistent CTA per
//    SM; a tile's K loop covers only the K-blocks (64 reflections) its band
//    touches;
//  * warp 0 issues TMA loads (128B-swizzled, K-major tiles of the four bf16
//    operands) into a two-stage shared-memory ring; warp 1 issues
//    tcgen05.mma (M 128, N 256, K 16) into one of two TMEM accumulators
//    (alternating per tile, so one tile's epilogue overlaps the next tile's
//    MMAs) and commits each stage back to the producer; warps 2-17 (four
//    per TMEM lane quarter, 64 of the tile's columns each) read the
//    accumulator with tcgen05.ld and reduce the weighted residual against
//    the observed pattern (terms in FP32, sums in FP64, the only FP64 on
//    this path), optionally storing Y;
//  * per-tile chi^2 partials are summed per replica in a fixed order.
// The three-part split (P6_CT_SPLIT3_BF16) goes one part further: I = I_h
// + I_m + I_l exactly for FP32 inputs (I_h = bf16(I), I_m = bf16(I - I_h),
// I_l = bf16(I - I_h - I_m)), likewise P, and Y = I_h P_h + I_h P_m + I_m P_h
// + I_h P_l + I_l P_h + I_m P_m: every operand exact to 2^-27 and every
// product down to 2^-24 kept, so the tensor core's FP32 accumulation is the
// limit (measured: chi^2 within 3.7e-6 of FP64, against 1.2e-5 for the
// two-part split and 3.4e-7 for the FP32 CUDA-core product).  The same
// pipeline runs it as two virtual K-blocks per K-block, each staging four
// operand tiles and issuing its share of the six products (v0: h,m x h,m,
// four products; v1: h.l + l.h), so each distinct operand tile but the high
// parts is staged once per K-block.
// A plain FP32 CUDA-core kernel over the same bands is the comparison
// method.  Every device wait is bounded; a wait that runs out records an
// error the host reports as P6_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "p6_common.cuh"
#include "tc_common.cuh"
#include "ct_internal.h"

namespace p6 {
namespace ct {

using namespace p6::tc;

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 2;
constexpr int A_TILE = BM * BK * 2;                       // 16 KB per bf16 operand tile
constexpr int B_TILE = BN * BK * 2;                       // 32 KB
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;      // 96 KB: A_hi, A_lo, B_hi, B_lo
constexpr int kEpiWarps = 16;                             // four per TMEM lane quarter
constexpr int kEpiSpan = BN / (kEpiWarps / 4);              // columns per epilogue warp (64)
constexpr int kThreads = 64 + 32 * kEpiWarps;               // warp 0 TMA, warp 1 MMA, warps 2-17 epilogue
constexpr int EPI_W_BYTES = 2 * kEpiWarps * kEpiSpan * 16;  // fitted epilogue: {w y, w} of each warp's columns, two tiles
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_W_BYTES + 1024;   // + alignment slack (1024-B swizzle atoms)
constexpr uint32_t TMEM_COLS = 2 * BN;                    // two accumulator buffers

// SIMT comparison kernel tiles
constexpr int FM = 128, FN = 128, FK = 16;

constexpr uint32_t kIdesc = idesc_bf16(BM, BN);

enum CtError : int { CT_OK = 0, CT_WAIT_FULL = 11, CT_WAIT_EMPTY = 12, CT_WAIT_ACC = 13, CT_WAIT_DRAIN = 14 };

struct Params {
  int M, N, Kp, nTilesN, nTilesM;
  int virt;               // virtual K-blocks per K-block: 1 (two-part split) or 2 (three-part split)
  const int2 *kRange;     // per BN tile: K-blocks [x, y)
  const float *yobs, *w;  // N
  const double *wy, *w64; // N: w y_obs and w in FP64 (fitted-scale sums)
  float *Y;               // optional, M x ldY
  int ldY;
  double *chiPart;        // M x nTilesN x (epilogue warps per lane quarter), two per slot when fitted
  int *errFlag;
};

// FITTED: instead of sum w (y - y_calc)^2 the epilogue forms, per replica,
// a = sum w y y_calc and b = sum w y_calc^2 (FP64 products and sums), from
// which chi^2 at the best scale s = a / b is sum w y^2 - a^2 / b.
template <bool FITTED>
__global__ void __launch_bounds__(kThreads, 1)
    contract_tc_kernel(const __grid_constant__ CUtensorMap tmAhi, const __grid_constant__ CUtensorMap tmAlo,
                       const __grid_constant__ CUtensorMap tmBhi, const __grid_constant__ CUtensorMap tmBlo,
                       const __grid_constant__ CUtensorMap tmAlo2, const __grid_constant__ CUtensorMap tmBlo2,
                       const Params P) {
  extern __shared__ unsigned char smemRaw[];
  __shared__ __align__(8) uint64_t fullBar[STAGES], emptyBar[STAGES], accFull[2], accEmpty[2];
  __shared__ uint32_t tmemBase;
  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nTiles = P.nTilesN * P.nTilesM;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&fullBar[s], 1);
      mbar_init(&emptyBar[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&accFull[a], 1);
      mbar_init(&accEmpty[a], kEpiWarps);   // one arrival per epilogue warp
    }
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemBase)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmemBase;

  // Tiles t = blockIdx.x, + gridDim.x, ...: column tile t % nTilesN of row tile
  // t / nTilesN, so the CTAs at work share the rows of I in L2.
  if (warp == 0) {
    if (lane == 0) {
      // producer: TMA loads of the four operand tiles of each K-block
      int it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < nTiles && ok; t += gridDim.x) {
        const int nt = t % P.nTilesN, mt = t / P.nTilesN;
        const int2 kr = P.kRange[nt];
        for (int vi = kr.x * P.virt; vi < kr.y * P.virt; ++vi, ++it) {
          const int s = it % STAGES;
          if (it >= STAGES && !wait_phase(&emptyBar[s], ((it / STAGES) - 1) & 1)) {
            raise_flag(P.errFlag, CT_WAIT_EMPTY);
            ok = false;
            break;
          }
          unsigned char *st = smem + s * STAGE_BYTES;
          mbar_arrive_expect_tx(&fullBar[s], STAGE_BYTES);
          const int kx = (vi / P.virt) * BK, v = vi % P.virt;
          // the stage's operand slots A1, A2, B1, B2 for this virtual K-block
          const CUtensorMap *a1 = &tmAhi, *a2 = v == 1 ? &tmAlo2 : &tmAlo;
          const CUtensorMap *b1 = v == 1 ? &tmBlo2 : &tmBhi, *b2 = v == 1 ? &tmBhi : &tmBlo;
          tma_load_2d(st, a1, kx, mt * BM, &fullBar[s]);
          tma_load_2d(st + A_TILE, a2, kx, mt * BM, &fullBar[s]);
          tma_load_2d(st + 2 * A_TILE, b1, kx, nt * BN, &fullBar[s]);
          tma_load_2d(st + 2 * A_TILE + B_TILE, b2, kx, nt * BN, &fullBar[s]);
        }
      }
      // every copy issued has landed before the CTA may exit
      for (int i = max(0, it - STAGES); i < it; ++i)
        if (!wait_phase(&fullBar[i % STAGES], (i / STAGES) & 1)) raise_flag(P.errFlag, CT_WAIT_DRAIN);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer: three bf16 products per K step, accumulators alternating
      // between two TMEM buffers so the epilogue of one tile overlaps the next
      int it = 0, j = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < nTiles && ok; t += gridDim.x, ++j) {
        const int nt = t % P.nTilesN, acc = j & 1;
        const int2 kr = P.kRange[nt];
        if (j >= 2 && !wait_phase(&accEmpty[acc], ((j >> 1) - 1) & 1)) {
          raise_flag(P.errFlag, CT_WAIT_ACC);
          break;
        }
        fence_after_sync();
        const uint32_t d = tmem + (uint32_t)(acc * BN);
        int done = 0;
        for (int vi = kr.x * P.virt; vi < kr.y * P.virt; ++vi, ++it) {
          const int s = it % STAGES;
          if (!wait_phase(&fullBar[s], (it / STAGES) & 1)) {
            raise_flag(P.errFlag, CT_WAIT_FULL);
            ok = false;
            break;
          }
          fence_after_sync();
          const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
          // products of the slots: bit 0 A1.B1, bit 1 A1.B2, bit 2 A2.B1, bit 3 A2.B2
          const int v = vi % P.virt;
          const int mask = P.virt == 1 ? 0x7 : (v == 0 ? 0xF : 0x9);
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
            const uint32_t off = k * 32;   // 16 bf16 along K inside the 128-byte swizzle row
            const uint64_t a1 = smem_desc(base + off), a2 = smem_desc(base + A_TILE + off);
            const uint64_t b1 = smem_desc(base + 2 * A_TILE + off), b2 = smem_desc(base + 2 * A_TILE + B_TILE + off);
            umma_bf16(d, a1, b1, kIdesc, (done > 0 || k > 0) ? 1u : 0u);
            if (mask & 2) umma_bf16(d, a1, b2, kIdesc, 1u);
            if (mask & 4) umma_bf16(d, a2, b1, kIdesc, 1u);
            if (mask & 8) umma_bf16(d, a2, b2, kIdesc, 1u);
          }
          umma_commit(&emptyBar[s]);
          ++done;
        }
        if (done > 0)
          umma_commit(&accFull[acc]);   // arrives once every MMA of the tile has completed
        else
          mbar_arrive(&accFull[acc]);   // empty band (or a failed wait): nothing in flight
      }
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (one replica row per
    // thread) and columns kEpiSpan * part .. + kEpiSpan of the tile; the terms
    // w (y - y_calc)^2 are formed in FP32 and summed in FP64
    const int q = warp & 3, part = (warp - 2) >> 2, cBeg = part * kEpiSpan;
    const int slots = kEpiWarps / 4;
    // fitted: this warp's weights for a tile's columns, copied into shared
    // memory one tile ahead (cp.async into two buffers) and read back as
    // broadcasts, so their trip from L2 overlaps the tile before
    double2 *wbase = reinterpret_cast<double2 *>(smem + STAGES * STAGE_BYTES) + (size_t)(warp - 2) * kEpiSpan;
    auto prefetch = [&](int tile, double2 *dst) {
      const int col0 = (tile % P.nTilesN) * BN + cBeg;
      for (int c = lane; c < kEpiSpan; c += 32) {
        const int col = col0 + c;
        if (col < P.N) {
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(&dst[c].x)), "l"(P.wy + col)
                       : "memory");
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(&dst[c].y)), "l"(P.w64 + col)
                       : "memory");
        } else {
          dst[c] = make_double2(0.0, 0.0);
        }
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (FITTED && blockIdx.x < nTiles) prefetch(blockIdx.x, wbase);
    int j = 0;
    for (int t = blockIdx.x; t < nTiles; t += gridDim.x, ++j) {
      const int nt = t % P.nTilesN, mt = t / P.nTilesN, acc = j & 1;
      const int2 kr = P.kRange[nt];
      const int row = q * 32 + lane, grow = mt * BM + row;
      double2 *wbuf = wbase + (size_t)(j & 1) * kEpiWarps * kEpiSpan;
      if (FITTED) {
        // the next tile's weights go into the other buffer (its last reader,
        // the tile before this one, finished at its closing __syncwarp)
        if (t + (int)gridDim.x < nTiles) {
          prefetch(t + gridDim.x, wbase + (size_t)((j + 1) & 1) * kEpiWarps * kEpiSpan);
          asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
          asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncwarp();
      }
      const bool ok = __all_sync(0xffffffffu, wait_phase(&accFull[acc], (j >> 1) & 1));
      if (!ok) {
        if (lane == 0) raise_flag(P.errFlag, CT_WAIT_ACC);
        break;
      }
      fence_after_sync();
      float v[kEpiSpan];
      if (kr.y > kr.x) {
        tmem_ld64(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + cBeg), v);
      } else {
#pragma unroll
        for (int jj = 0; jj < kEpiSpan; ++jj) v[jj] = 0.f;
      }
      double chi0 = 0.0, chi1 = 0.0;
      if (FITTED && grow < P.M) {
        const int col0 = nt * BN + cBeg;
        double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
        // columns past the active points carry zero weights
#pragma unroll
        for (int g = 0; g < kEpiSpan / 2; ++g) {
          const double2 q0 = wbuf[2 * g], q1 = wbuf[2 * g + 1];
          const double y0 = (double)v[2 * g], y1 = (double)v[2 * g + 1];
          a0 = fma(q0.x, y0, a0);
          a1 = fma(q1.x, y1, a1);
          b0 = fma(q0.y * y0, y0, b0);
          b1 = fma(q1.y * y1, y1, b1);
        }
        double *dst = P.chiPart + (((size_t)grow * P.nTilesN + nt) * slots + part) * 2;
        dst[0] = a0 + a1;
        dst[1] = b0 + b1;
        if (P.Y) {
#pragma unroll
          for (int jj = 0; jj < kEpiSpan; ++jj)
            if (col0 + jj < P.N) P.Y[(size_t)grow * P.ldY + col0 + jj] = v[jj];
        }
      } else if (grow < P.M) {
        const int col0 = nt * BN + cBeg;
        if (col0 + kEpiSpan <= P.N) {
          // whole span inside the pattern: vector loads of the observed counts and weights
          const float4 *yo4 = reinterpret_cast<const float4 *>(P.yobs + col0);
          const float4 *w4 = reinterpret_cast<const float4 *>(P.w + col0);
#pragma unroll
          for (int g = 0; g < kEpiSpan / 4; ++g) {
            const float4 yo = __ldg(yo4 + g), ww = __ldg(w4 + g);
            const float d0 = yo.x - v[4 * g], d1 = yo.y - v[4 * g + 1], d2 = yo.z - v[4 * g + 2], d3 = yo.w - v[4 * g + 3];
            chi0 += (double)(ww.x * d0 * d0) + (double)(ww.y * d1 * d1);
            chi1 += (double)(ww.z * d2 * d2) + (double)(ww.w * d3 * d3);
          }
          if (P.Y && (P.ldY & 3) == 0) {
            float4 *dst = reinterpret_cast<float4 *>(P.Y + (size_t)grow * P.ldY + col0);
#pragma unroll
            for (int g = 0; g < kEpiSpan / 4; ++g)
              dst[g] = make_float4(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
          } else if (P.Y) {
#pragma unroll
            for (int jj = 0; jj < kEpiSpan; ++jj) P.Y[(size_t)grow * P.ldY + col0 + jj] = v[jj];
          }
        } else {
#pragma unroll
          for (int jj = 0; jj < kEpiSpan; ++jj) {
            const int col = col0 + jj;
            if (col < P.N) {
              if (P.Y) P.Y[(size_t)grow * P.ldY + col] = v[jj];
              const float dd = __ldg(P.yobs + col) - v[jj];
              chi0 += (double)(__ldg(P.w + col) * dd * dd);
            }
          }
        }
        P.chiPart[((size_t)grow * P.nTilesN + nt) * slots + part] = chi0 + chi1;
      }
      // the accumulator buffer is free for the tile after next
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accEmpty[acc]);
    }
    if (FITTED) asm volatile("cp.async.wait_group 0;" ::: "memory");   // no copy outlives the loop
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// Split of an FP32 matrix (rows x cols, leading dimension ld) into bf16 hi/lo
// parts (rows x Kp, zero padded to Kp columns, Kp a multiple of 4): four
// columns per thread, 16-byte loads where the row stride allows, 8-byte stores.
__device__ __forceinline__ void split4(const float x[4], __nv_bfloat16 *hi, __nv_bfloat16 *lo, __nv_bfloat16 *lo2,
                                       size_t at) {
  __align__(8) __nv_bfloat16 h[4], l[4], l2[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    h[i] = __float2bfloat16_rn(x[i]);
    const float r = x[i] - __bfloat162float(h[i]);   // exact in FP32
    l[i] = __float2bfloat16_rn(r);
    l2[i] = __float2bfloat16_rn(r - __bfloat162float(l[i]));
  }
  *reinterpret_cast<uint2 *>(hi + at) = *reinterpret_cast<const uint2 *>(h);
  *reinterpret_cast<uint2 *>(lo + at) = *reinterpret_cast<const uint2 *>(l);
  if (lo2) *reinterpret_cast<uint2 *>(lo2 + at) = *reinterpret_cast<const uint2 *>(l2);
}

__global__ void split_kernel(const float *src, int rows, int cols, int ld, int Kp, __nv_bfloat16 *hi,
                             __nv_bfloat16 *lo, __nv_bfloat16 *lo2) {
  const int q = Kp / 4;
  const size_t total = (size_t)rows * q;
  const bool vec = (ld & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / q;
    const int k = (int)(i - r * q) * 4;
    float x[4];
    if (vec && k + 3 < cols) {
      const float4 f = __ldg(reinterpret_cast<const float4 *>(src + r * ld + k));
      x[0] = f.x; x[1] = f.y; x[2] = f.z; x[3] = f.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = k + j < cols ? src[r * ld + k + j] : 0.f;
    }
    split4(x, hi, lo, lo2, r * Kp + k);
  }
}

// Plain FP32 comparison: 128 x 128 tile, 16 x 16 threads x (8 x 8) outputs, K steps of 16
// over the tile's band; FP64 chi^2 partials per 128-column tile.
// FITTED: the partials are a = sum w y y_calc and b = sum w y_calc^2 (two per
// tile), as in the tensor-core kernel.  ldY: row stride of the stored Y.
template <bool FITTED>
__global__ void __launch_bounds__(256) contract_fp32_kernel(const float *I, int ldI, const float *PT, int ldP,
                                                            const int2 *kRange128, int M, int N, int nTiles128,
                                                            const float *yobs, const float *w, const double *wy,
                                                            const double *w64, float *Y, int ldY,
                                                            double *chiPart) {
  __shared__ float As[FK][FM + 4], Bs[FK][FN + 4];
  __shared__ double rowChi[FM][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int nt = blockIdx.x, mt = blockIdx.y;
  const int2 kr = kRange128[nt];
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  for (int k0 = kr.x; k0 < kr.y; k0 += FK) {
    for (int e = threadIdx.x; e < FM * FK; e += 256) {
      const int r = e / FK, k = e % FK;
      const int gm = mt * FM + r, gn = nt * FN + r, gk = k0 + k;
      As[k][r] = (gm < M && gk < kr.y) ? I[(size_t)gm * ldI + gk] : 0.f;
      Bs[k][r] = (gn < N && gk < kr.y) ? PT[(size_t)gn * ldP + gk] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < FK; ++k) {
      float a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[k][ty * 8 + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[k][tx * 8 + j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double cb[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = mt * FM + ty * 8 + i;
    double c = 0.0, b = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = nt * FN + tx * 8 + j;
      if (gm < M && gn < N) {
        if (Y) Y[(size_t)gm * ldY + gn] = acc[i][j];
        const double y = (double)acc[i][j];
        if (FITTED) {
          c = fma(wy[gn], y, c);
          b = fma(w64[gn] * y, y, b);
        } else {
          const double d = (double)yobs[gn] - y;
          c += (double)w[gn] * d * d;
        }
      }
    }
    rowChi[ty * 8 + i][tx] = c;
    cb[i] = b;
  }
  __syncthreads();
  if (threadIdx.x < FM) {
    const int gm = mt * FM + threadIdx.x;
    double c = 0.0;
    for (int t = 0; t < 16; ++t) c += rowChi[threadIdx.x][t];
    if (gm < M) chiPart[((size_t)gm * nTiles128 + nt) * (FITTED ? 2 : 1)] = c;
  }
  if (FITTED) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; ++i) rowChi[ty * 8 + i][tx] = cb[i];
    __syncthreads();
    if (threadIdx.x < FM) {
      const int gm = mt * FM + threadIdx.x;
      double b = 0.0;
      for (int t = 0; t < 16; ++t) b += rowChi[threadIdx.x][t];
      if (gm < M) chiPart[((size_t)gm * nTiles128 + nt) * 2 + 1] = b;
    }
  }
}

// chi2[r] = sum of the row's tile partials: one warp per row, lane l
// summing partials l, l + 32, ... in order, then a fixed butterfly across
// the lanes (the same order every call: bit-reproducible).
__global__ void chi_reduce_kernel(const double *part, int M, int nTiles, double *chi2) {
  const int r = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (r >= M) return;
  const double *row = part + (size_t)r * nTiles;
  double s = 0.0;
  for (int t = lane; t < nTiles; t += 32) s += row[t];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) chi2[r] = s;
}

// Fitted scale: a and b summed in tile order; chi^2 at s = a / b is
// syy - a s (syy = sum w y^2 over the active points); s = 0 and chi^2 = syy
// when no positive scale lowers it.
__global__ void chi_reduce_fitted_kernel(const double *part, int M, int nTiles, double syy, double *chi2,
                                         double *scale) {
  const int r = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (r >= M) return;
  const double2 *row = reinterpret_cast<const double2 *>(part) + (size_t)r * nTiles;
  double a = 0.0, b = 0.0;
  for (int t = lane; t < nTiles; t += 32) {
    const double2 v = row[t];
    a += v.x;
    b += v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane != 0) return;
  double s = 0.0, c = syy;
  if (a > 0.0 && b > 0.0) {
    s = a / b;
    c = fmax(syy - a * s, 0.0);
  }
  chi2[r] = c;
  if (scale) scale[r] = s;
}

}  // namespace ct
}  // namespace p6

// ===========================================================================
// Host side.
// ===========================================================================
using namespace p6;
using namespace p6::ct;
using namespace p6::tc;

namespace {
// K-ranges of each column tile of width `tile`: the smallest and largest
// reflection with a nonzero profile value in the tile, rounded out to `align`.
std::vector<int2> bands(const float *PT, int N, int K, int tile, int align, int Kp) {
  const int nt = (N + tile - 1) / tile;
  std::vector<int2> out(nt);
  for (int t = 0; t < nt; ++t) {
    int lo = K, hi = -1;
    for (int j = t * tile; j < std::min(N, (t + 1) * tile); ++j) {
      const float *row = PT + (size_t)j * K;
      int a = 0;
      while (a < K && row[a] == 0.f) ++a;
      if (a == K) continue;
      int b = K - 1;
      while (b > a && row[b] == 0.f) --b;
      lo = std::min(lo, a);
      hi = std::max(hi, b);
    }
    if (hi < lo) {
      out[t] = make_int2(0, 0);
    } else {
      const int kLo = lo / align * align, kHi = std::min(Kp, (hi + 1 + align - 1) / align * align);
      out[t] = make_int2(kLo, kHi);
    }
  }
  return out;
}
}  // namespace

struct p6_ct_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int K = 0, Kp = 0, N = 0, Np = 0, maxM = 0, M = 0;
  int nTilesN = 0, nTiles128 = 0;
  float *dPT = nullptr;                 // N x K (FP32, the comparison path)
  __nv_bfloat16 *dBhi = nullptr, *dBlo = nullptr, *dAhi = nullptr, *dAlo = nullptr;
  __nv_bfloat16 *dBlo2 = nullptr, *dAlo2 = nullptr;   // third parts of the three-part split
  float *dI = nullptr;                  // maxM x K (FP32 intensities)
  float *dY = nullptr;                  // maxM x N, allocated on first request
  float *dYobs = nullptr, *dW = nullptr;
  double *dPart = nullptr, *dChi = nullptr;
  double *dWy = nullptr, *dW64 = nullptr, *dScale = nullptr;   // fitted-scale mode
  std::vector<double> syyPrefix;        // sum of w y^2 over the first j points, j = 0..N
  int fitted = 0;
  int2 *dRange = nullptr, *dRange128 = nullptr, *dRangeDense = nullptr;
  int *dErr = nullptr;
  long long bandBlocks = 0, bandCols128 = 0;   // sum of K-blocks over BN tiles; sum of K over 128-col tiles
  CUtensorMap mapAhi, mapAlo, mapBhi, mapBlo, mapAlo2, mapBlo2;
  long long launches = 0;
  int numSMs = 148;
};

static void ct_free(p6_ct_session *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void *p : {(void *)s->dPT, (void *)s->dBhi, (void *)s->dBlo, (void *)s->dAhi, (void *)s->dAlo, (void *)s->dI,
                  (void *)s->dBlo2, (void *)s->dAlo2,
                  (void *)s->dY, (void *)s->dYobs, (void *)s->dW, (void *)s->dPart, (void *)s->dChi,
                  (void *)s->dWy, (void *)s->dW64, (void *)s->dScale, (void *)s->dRangeDense,
                  (void *)s->dRange, (void *)s->dRange128, (void *)s->dErr})
    if (p) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static p6_status ct_check_flag(p6_ct_session *s) {
  int flag = 0;
  P6_CUDA(cudaMemcpyAsync(&flag, s->dErr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  if (flag) {
    cudaMemsetAsync(s->dErr, 0, sizeof(int), s->stream);
    return set_error(P6_ERR_TIMEOUT, "a tensor-core pipeline wait did not complete in time (code " +
                                         std::to_string(flag) + ")");
  }
  return P6_OK;
}

// Y = I . P for the first M rows of I (M x K, FP32, row-major) on `st`, over
// the first nAct points: with `fitted`, chi^2 at each replica's best scale
// (and the scale), else the plain weighted chi^2; Y kept when given.
static p6_status ct_enqueue(p6_ct_session *s, cudaStream_t st, const float *I, int M, int method, bool fitted,
                            int nAct, float *Y, bool reduce = true, int *partsOut = nullptr) {
  if (M <= 0 || M > s->maxM) return set_error(P6_ERR_CAPACITY, "replica count outside the session's capacity");
  nAct = std::max(1, std::min(nAct, s->N));
  const int slots = kEpiWarps / 4;
  int nParts;
  if (method == P6_CT_SPLIT_BF16 || method == P6_CT_SPLIT3_BF16) {
    const bool three = method == P6_CT_SPLIT3_BF16;
    split_kernel<<<2368, 256, 0, st>>>(I, M, s->K, s->K, s->Kp, s->dAhi, s->dAlo, three ? s->dAlo2 : nullptr);
    P6_CUDA(cudaGetLastError());
    Params P;
    P.M = M; P.N = nAct; P.Kp = s->Kp; P.nTilesN = (nAct + BN - 1) / BN; P.nTilesM = (M + BM - 1) / BM;
    P.virt = three ? 2 : 1;
    P.kRange = s->dRange; P.yobs = s->dYobs; P.w = s->dW; P.wy = s->dWy; P.w64 = s->dW64;
    P.Y = Y; P.ldY = s->N; P.chiPart = s->dPart; P.errFlag = s->dErr;
    // persistent: one CTA per SM, tiles handed out round-robin
    const int grid = std::min(P.nTilesN * P.nTilesM, s->numSMs);
    if (fitted)
      contract_tc_kernel<true><<<grid, kThreads, SMEM_BYTES, st>>>(s->mapAhi, s->mapAlo, s->mapBhi, s->mapBlo,
                                                                    s->mapAlo2, s->mapBlo2, P);
    else
      contract_tc_kernel<false><<<grid, kThreads, SMEM_BYTES, st>>>(s->mapAhi, s->mapAlo, s->mapBhi, s->mapBlo,
                                                                     s->mapAlo2, s->mapBlo2, P);
    P6_CUDA(cudaGetLastError());
    nParts = P.nTilesN * slots;   // per replica: tiles x epilogue slots, in order
    s->launches += 2;
  } else {
    const int nT = (nAct + FN - 1) / FN;
    const dim3 grid(nT, (M + FM - 1) / FM);
    const int2 *range = method == P6_CT_FP32_DENSE ? s->dRangeDense : s->dRange128;
    if (fitted)
      contract_fp32_kernel<true><<<grid, 256, 0, st>>>(I, s->K, s->dPT, s->K, range, M, nAct, nT, s->dYobs, s->dW,
                                                        s->dWy, s->dW64, Y, s->N, s->dPart);
    else
      contract_fp32_kernel<false><<<grid, 256, 0, st>>>(I, s->K, s->dPT, s->K, range, M, nAct, nT, s->dYobs, s->dW,
                                                         s->dWy, s->dW64, Y, s->N, s->dPart);
    P6_CUDA(cudaGetLastError());
    nParts = nT;
    s->launches += 1;
  }
  if (partsOut) *partsOut = nParts;
  if (!reduce) return P6_OK;
  // one warp per replica row, eight rows per block
  if (fitted)
    chi_reduce_fitted_kernel<<<(M + 7) / 8, 256, 0, st>>>(s->dPart, M, nParts, s->syyPrefix[nAct], s->dChi,
                                                           s->dScale);
  else
    chi_reduce_kernel<<<(M + 7) / 8, 256, 0, st>>>(s->dPart, M, nParts, s->dChi);
  P6_CUDA(cudaGetLastError());
  s->launches += 1;
  return P6_OK;
}

namespace p6 {
namespace ct {
// The link a fixed-profile search uses (ct_internal.h).
ProfileLink link(p6_ct_session *s) {
  ProfileLink L;
  L.intensities = s->dI;
  L.chi2 = s->dChi;
  L.n_refl = s->K;
  L.n_points = s->N;
  L.max_replicas = s->maxM;
  L.device = s->device;
  return L;
}
p6_status enqueue_fitted(p6_ct_session *s, cudaStream_t stream, int n_replicas, int method, int n_active_points) {
  return ct_enqueue(s, stream, s->dI, n_replicas, method, true, n_active_points, nullptr);
}
p6_status enqueue_fitted_partials(p6_ct_session *s, cudaStream_t stream, int n_replicas, int method,
                                  int n_active_points, const double2 **part, int *n_parts) {
  *part = reinterpret_cast<const double2 *>(s->dPart);
  return ct_enqueue(s, stream, s->dI, n_replicas, method, true, n_active_points, nullptr, false, n_parts);
}
double syy(p6_ct_session *s, int n_active_points) {
  return s->syyPrefix[std::max(0, std::min(n_active_points, s->N))];
}
p6_status check(p6_ct_session *s) { return ct_check_flag(s); }
}  // namespace ct
}  // namespace p6

extern "C" {

p6_status p6_ct_create(const p6_ct_problem *pr, int device, p6_ct_session **out) {
  clear_error();
  if (!pr || !out) return set_error(P6_ERR_INVALID_ARG, "null problem or output pointer");
  *out = nullptr;
  if (pr->n_refl <= 0 || pr->n_points <= 0 || pr->max_replicas <= 0 || !pr->profile_t || !pr->yobs || !pr->w)
    return set_error(P6_ERR_INVALID_ARG, "empty problem");
  p6_ct_session *s = new p6_ct_session();
  s->device = device;
  s->K = pr->n_refl;
  s->Kp = (pr->n_refl + BK - 1) / BK * BK;
  s->N = pr->n_points;
  s->Np = (pr->n_points + BN - 1) / BN * BN;
  s->maxM = pr->max_replicas;
  s->nTilesN = s->Np / BN;
  s->nTiles128 = (s->N + FN - 1) / FN;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { ct_free(s); return cuda_error(e, "cudaSetDevice"); }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { ct_free(s); return cuda_error(e, "cudaStreamCreate"); }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  const std::vector<int2> rBN = bands(pr->profile_t, s->N, s->K, BN, BK, s->Kp);
  const std::vector<int2> r128 = bands(pr->profile_t, s->N, s->K, FN, 1, s->K);
  std::vector<int2> kb(rBN.size());
  for (size_t t = 0; t < rBN.size(); ++t) {
    kb[t] = make_int2(rBN[t].x / BK, rBN[t].y / BK);
    s->bandBlocks += kb[t].y - kb[t].x;
  }
  for (const int2 &r : r128) s->bandCols128 += r.y - r.x;
  const size_t K = s->K, Kp = s->Kp, N = s->N, Np = s->Np, M = s->maxM;
  p6_status st = P6_OK;
#define CT_ALLOC(ptr, bytes)                                   \
  do {                                                         \
    e = cudaMalloc((void **)&(ptr), (bytes));                  \
    if (e != cudaSuccess) { ct_free(s); return cuda_error(e, "cudaMalloc"); } \
  } while (0)
  CT_ALLOC(s->dPT, N * K * sizeof(float));
  CT_ALLOC(s->dBhi, Np * Kp * 2);
  CT_ALLOC(s->dBlo, Np * Kp * 2);
  CT_ALLOC(s->dAhi, M * Kp * 2);
  CT_ALLOC(s->dAlo, M * Kp * 2);
  CT_ALLOC(s->dBlo2, Np * Kp * 2);
  CT_ALLOC(s->dAlo2, M * Kp * 2);
  CT_ALLOC(s->dI, M * K * sizeof(float));
  CT_ALLOC(s->dYobs, N * sizeof(float));
  CT_ALLOC(s->dW, N * sizeof(float));
  CT_ALLOC(s->dPart, 2 * M * std::max((size_t)s->nTilesN * (kEpiWarps / 4), (size_t)s->nTiles128) * sizeof(double));
  CT_ALLOC(s->dChi, M * sizeof(double));
  CT_ALLOC(s->dScale, M * sizeof(double));
  CT_ALLOC(s->dWy, N * sizeof(double));
  CT_ALLOC(s->dW64, N * sizeof(double));
  CT_ALLOC(s->dRange, kb.size() * sizeof(int2));
  CT_ALLOC(s->dRange128, r128.size() * sizeof(int2));
  CT_ALLOC(s->dRangeDense, r128.size() * sizeof(int2));
  CT_ALLOC(s->dErr, sizeof(int));
#undef CT_ALLOC
  cudaMemsetAsync(s->dErr, 0, sizeof(int), s->stream);
  cudaMemsetAsync(s->dBhi, 0, Np * Kp * 2, s->stream);
  cudaMemsetAsync(s->dBlo, 0, Np * Kp * 2, s->stream);
  cudaMemsetAsync(s->dBlo2, 0, Np * Kp * 2, s->stream);
  cudaMemcpyAsync(s->dPT, pr->profile_t, N * K * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->dYobs, pr->yobs, N * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->dW, pr->w, N * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->dRange, kb.data(), kb.size() * sizeof(int2), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->dRange128, r128.data(), r128.size() * sizeof(int2), cudaMemcpyHostToDevice, s->stream);
  // the dense comparison: every 128-point tile runs over all reflections
  const std::vector<int2> dense(r128.size(), make_int2(0, s->K));
  cudaMemcpyAsync(s->dRangeDense, dense.data(), dense.size() * sizeof(int2), cudaMemcpyHostToDevice, s->stream);
  // fitted-scale operands: w (points with w <= 0 excluded) and w y in FP64
  std::vector<double> w64(N), wy(N);
  s->syyPrefix.assign(N + 1, 0.0);
  for (size_t j = 0; j < N; ++j) {
    w64[j] = pr->w[j] > 0.f ? (double)pr->w[j] : 0.0;
    wy[j] = w64[j] * (double)pr->yobs[j];
    s->syyPrefix[j + 1] = s->syyPrefix[j] + wy[j] * (double)pr->yobs[j];
  }
  cudaMemcpyAsync(s->dW64, w64.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->dWy, wy.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->stream);
  split_kernel<<<2368, 256, 0, s->stream>>>(s->dPT, s->N, s->K, s->K, s->Kp, s->dBhi, s->dBlo, s->dBlo2);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) { ct_free(s); return cuda_error(e, "profile upload"); }
  if ((st = make_map(&s->mapAhi, s->dAhi, s->maxM, s->Kp, BM)) != P6_OK ||
      (st = make_map(&s->mapAlo, s->dAlo, s->maxM, s->Kp, BM)) != P6_OK ||
      (st = make_map(&s->mapBhi, s->dBhi, s->Np, s->Kp, BN)) != P6_OK ||
      (st = make_map(&s->mapBlo, s->dBlo, s->Np, s->Kp, BN)) != P6_OK ||
      (st = make_map(&s->mapAlo2, s->dAlo2, s->maxM, s->Kp, BM)) != P6_OK ||
      (st = make_map(&s->mapBlo2, s->dBlo2, s->Np, s->Kp, BN)) != P6_OK) {
    ct_free(s);
    return st;
  }
  cudaDeviceGetAttribute(&s->numSMs, cudaDevAttrMultiProcessorCount, device);
  e = cudaFuncSetAttribute(contract_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(contract_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e != cudaSuccess) { ct_free(s); return cuda_error(e, "cudaFuncSetAttribute"); }
  *out = s;
  return P6_OK;
}

p6_status p6_ct_destroy(p6_ct_session *s) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  ct_free(s);
  return P6_OK;
}

p6_status p6_ct_set_intensities(p6_ct_session *s, const float *intensities, int n_replicas) {
  clear_error();
  if (!s || !intensities || n_replicas <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  if (n_replicas > s->maxM) return set_error(P6_ERR_CAPACITY, "more replicas than the session was created for");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaMemcpyAsync(s->dI, intensities, (size_t)n_replicas * s->K * sizeof(float), cudaMemcpyHostToDevice,
                          s->stream));
  s->M = n_replicas;
  return P6_OK;
}

p6_status p6_ct_evaluate(p6_ct_session *s, int method, int store_pattern) {
  clear_error();
  if (!s || s->M <= 0) return set_error(P6_ERR_INVALID_ARG, "no intensities set");
  if (method < P6_CT_SPLIT_BF16 || method > P6_CT_FP32_DENSE) return set_error(P6_ERR_INVALID_ARG, "unknown method");
  P6_CUDA(cudaSetDevice(s->device));
  if (store_pattern && !s->dY) P6_CUDA(cudaMalloc(&s->dY, (size_t)s->maxM * s->N * sizeof(float)));
  P6_CUDA(cudaEventRecord(s->ev0, s->stream));
  const p6_status st = ct_enqueue(s, s->stream, s->dI, s->M, method, s->fitted != 0, s->N,
                                  store_pattern ? s->dY : nullptr);
  if (st != P6_OK) return st;
  P6_CUDA(cudaEventRecord(s->ev1, s->stream));
  return P6_OK;
}

p6_status p6_ct_set_fitted(p6_ct_session *s, int fitted) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  s->fitted = fitted ? 1 : 0;
  return P6_OK;
}

p6_status p6_ct_read_scale(p6_ct_session *s, double *scale) {
  clear_error();
  if (!s || !scale) return set_error(P6_ERR_INVALID_ARG, "null argument");
  if (!s->fitted) return set_error(P6_ERR_INVALID_ARG, "the session is not in fitted-scale mode");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaMemcpyAsync(scale, s->dScale, (size_t)s->M * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return ct_check_flag(s);
}

p6_status p6_ct_read(p6_ct_session *s, double *chi2, float *pattern) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (pattern && !s->dY) return set_error(P6_ERR_INVALID_ARG, "no pattern was stored");
  if (chi2) P6_CUDA(cudaMemcpyAsync(chi2, s->dChi, (size_t)s->M * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (pattern)
    P6_CUDA(cudaMemcpyAsync(pattern, s->dY, (size_t)s->M * s->N * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return ct_check_flag(s);
}

p6_status p6_ct_run_host(p6_ct_session *s, const float *intensities, int n_replicas, int method, double *chi2) {
  p6_status st = p6_ct_set_intensities(s, intensities, n_replicas);
  if (st != P6_OK) return st;
  st = p6_ct_evaluate(s, method, 0);
  if (st != P6_OK) return st;
  return p6_ct_read(s, chi2, nullptr);
}

p6_status p6_ct_synchronize(p6_ct_session *s) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return ct_check_flag(s);
}

p6_status p6_ct_last_ms(p6_ct_session *s, float *ms) {
  clear_error();
  if (!s || !ms) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaEventSynchronize(s->ev1));
  P6_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
  return P6_OK;
}

p6_status p6_ct_query(p6_ct_session *s, long long *band_kblocks, long long *band_cols128, int *n_tiles,
                      long long *launches) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (band_kblocks) *band_kblocks = s->bandBlocks;
  if (band_cols128) *band_cols128 = s->bandCols128;
  if (n_tiles) *n_tiles = s->nTilesN;
  if (launches) *launches = s->launches;
  return P6_OK;
}

}  // extern "C"
