// Dual-space charge flipping on a powder reflection model: the cycle of
// charge_flipping.wgsl:182-632, in the order js/charge_flipping_worker.js:
// 2353-2395 dispatches it, for any number of independent trials at once.
//
// One cycle is seven launches, captured once in a CUDA graph and replayed:
//   1-3  inverse 3-D FFT, one axis per launch, in place.  Each CTA loads a
//        tile of XT lines into shared memory (whole lines along x; XT
//        consecutive x of every line along y and z, so every global access is
//        a coalesced run), transforms every line (radix-2, decimation in time
//        from the bit-reversed load), and writes the tile back.  Launch 1
//        first copies its input to the best grid when the previous cycle
//        improved R; launch 3 scales by 1/n^3 and leaves the tile's sums of
//        Re rho and (Re rho)^2.
//   4-6  forward FFT; launch 4 reduces those sums to delta = delta_sigma *
//        sigma and flips on load (Re rho < delta -> -Re rho, Im rho = 0).
//   7    reciprocal step: a warp per 2-theta cluster computes the cluster's
//        R terms, the Le Bail repartition of its observed intensity, the
//        symmetrisation and the amplitude constraint (or quarter-turn) of each
//        orbit; other threads zero the absent reflections and F(000).  The
//        last CTA of a trial to finish (a ticket counter, no waiting) sums the
//        per-CTA R terms in a fixed order and writes R, the best R and the keep
//        flag.
// Trials are blockIdx.y of every launch; the model tables are shared.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <thread>
#include <vector>

#include "p6_common.cuh"

namespace p6 {
namespace cf {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kIdxMask = 0x7fffffffu, kConjBit = 0x80000000u;
constexpr int kMaxTrials = 4096;

enum Prologue { PRO_NONE = 0, PRO_KEEP = 1, PRO_FLIP = 2 };
enum Epilogue { EPI_NONE = 0, EPI_SCALE_MOMENTS = 1, EPI_SCALE = 2 };

struct Params {
  int n;
  int tiles;           // tiles per trial per pass (n^2 / XT)
  int nTrials;
  long long cells;     // n^3
  int nOrbits, nClusters, nAbsent;
  const uint32_t *orbitStart, *orbitCount, *orbitIdx, *clusterOrbitStart, *clusterNOrbits, *absentIdx;
  const float *phase, *clusterObs;
  const float *deltaSigma, *symLambda;
  const uint32_t *seed;
  const uint8_t *weak;     // nTrials x nOrbits, or null
  float2 *grid, *best;     // nTrials x cells each
  double2 *moments;        // nTrials x tiles
  double2 *rPartial;       // nTrials x (reciprocal CTAs)
  unsigned *ticket;        // nTrials
  float *bestR;            // nTrials
  int *pending;            // nTrials
  int *cycleCount;         // nTrials
  float *history;          // nTrials x historyCap
  int historyCap;
};

// Lines per tile: XT consecutive x for the y and z passes, so XT <= n; the
// tile holds at most 2048 complex values (16 KB of shared memory).
__host__ __device__ constexpr int tile_lines(int n) { return n < 2048 / n ? n : 2048 / n; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of two doubles in a fixed order (warp trees, then warps in
// order): the result, in every thread, is the same in every CTA for the
// same inputs.
__device__ __forceinline__ void block_sum2(double &a, double &b, double *red) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) {
    red[warp] = a;
    red[kWarps + warp] = b;
  }
  __syncthreads();
  a = 0;
  b = 0;
  for (int w = 0; w < kWarps; ++w) {
    a += red[w];
    b += red[kWarps + w];
  }
}

// Where a tile's lines lie: element e of line t is data[base + t*tS + e*eS].
template <int N>
__device__ __forceinline__ void tile_geometry(int axis, int tile, long long &base, int &tS, long long &eS) {
  constexpr int XT = tile_lines(N);
  if (axis == 0) {
    base = (long long)tile * XT * N;
    tS = N;
    eS = 1;
    return;
  }
  const int xb = tile % (N / XT), o = tile / (N / XT);
  tS = 1;
  if (axis == 1) {
    base = (long long)xb * XT + (long long)o * N * N;
    eS = N;
  } else {
    base = (long long)xb * XT + (long long)o * N;
    eS = (long long)N * N;
  }
}

// Bit reversal of i over log2(R) bits, at compile time.
template <int R>
__host__ __device__ constexpr int bitrev(int i) {
  int r = 0;
  for (int m = 1, k = R >> 1; m < R; m <<= 1, k >>= 1)
    if (i & m) r |= k;
  return r;
}

// In-register DFT of R points (R = 1, 2, 4, 8, 16): radix-2 decimation in
// time from the bit-reversed order, fully unrolled.  tw[m] = exp(-+2 pi i m /
// N); the DFT's own twiddle exp(-+2 pi i k / 2L) is tw[k (R / 2L) (N / R)].
template <int R, int N>
__device__ __forceinline__ void dft_regs(float2 (&a)[R], const float2 *tw) {
  float2 b[R];
#pragma unroll
  for (int i = 0; i < R; ++i) b[bitrev<R>(i)] = a[i];
#pragma unroll
  for (int L = 1; L < R; L <<= 1) {
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
      const int k = j & (L - 1), i0 = ((j - k) << 1) + k, i1 = i0 + L;
      const float2 w = tw[k * (R / (2 * L)) * (N / R)];
      const float2 c = make_float2(b[i1].x * w.x - b[i1].y * w.y, b[i1].x * w.y + b[i1].y * w.x);
      b[i1] = make_float2(b[i0].x - c.x, b[i0].y - c.y);
      b[i0] = make_float2(b[i0].x + c.x, b[i0].y + c.y);
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) a[i] = b[i];
}

// One axis of the 3-D transform for every tile of every trial (in place).
// Forward: F(h) = sum_x rho(x) exp(-2 pi i h x / n); inverse: the + sign, and
// the 1/n^3 of the whole inverse transform applied by EPI_SCALE*.
//
// Each line of n = R1 R2 points (R1 = 8) is a four-step transform: with
// x index R2 n1 + n2 and X index k1 + R1 k2,
//   X[k1 + R1 k2] = sum_n2 W_R2^(n2 k2) W_n^(n2 k1) sum_n1 x[R2 n1 + n2] W_R1^(n1 k1).
// Step 1 (a thread per line and n2) loads its R1 points straight from global
// memory, transforms them in registers and applies W_n^(n2 k1); one exchange
// through shared memory (rows padded against bank conflicts); step 2 (a
// thread per line and k1) transforms over n2 in registers and stores.  Every
// global access is a coalesced run: consecutive threads take consecutive
// points of a line along x, and consecutive x (lines) along y and z.
template <int N>
__global__ void __launch_bounds__(kThreads, 4) cf_fft_kernel(const Params P, float2 *data, int trialBase, int axis,
                                                             int inverse, int prologue, int epilogue) {
  constexpr int XT = tile_lines(N);
  constexpr int R1 = N < 8 ? N : 8, R2 = N / R1;
  constexpr int ROW = R1 + 1;          // exchange row of one n2, padded
  constexpr int LDMAX = R2 * ROW + 1;
  __shared__ float2 y[XT * LDMAX];
  // line stride of the exchange: along x consecutive lanes walk n2 (or k1)
  // within a line, and the unpadded stride R2 ROW keeps the lines a half-warp
  // touches on disjoint 8-byte banks; along y and z consecutive lanes walk the
  // lines, and R2 ROW + 1 does
  const int ld = axis == 0 ? LDMAX - 1 : LDMAX;
  __shared__ float2 tw[N];
  __shared__ double red[2 * kWarps];
  __shared__ float sDelta;
  __shared__ int sKeep;
  const int tid = threadIdx.x, tile = blockIdx.x, trial = trialBase + blockIdx.y;
  float2 *g = data + (long long)trial * P.cells;
  long long base, eS;
  int tS;
  tile_geometry<N>(axis, tile, base, tS, eS);
  for (int m = tid; m < N; m += kThreads) {
    float sn, cs;
    sincospif(2.0f * (float)m / (float)N, &sn, &cs);
    tw[m] = make_float2(cs, inverse ? sn : -sn);
  }
  if (prologue == PRO_FLIP) {
    double a = 0, b = 0;
    for (int i = tid; i < P.tiles; i += kThreads) {
      const double2 m = P.moments[(long long)trial * P.tiles + i];
      a += m.x;
      b += m.y;
    }
    block_sum2(a, b, red);
    if (tid == 0) {
      const double inv = 1.0 / (double)P.cells, mean = a * inv, var = fmax(0.0, b * inv - mean * mean);
      sDelta = (float)((double)P.deltaSigma[trial] * sqrt(var));
    }
  }
  if (tid == 0) {
    sKeep = prologue == PRO_KEEP ? P.pending[trial] : 0;
    if (prologue != PRO_FLIP) sDelta = 0.f;
  }
  __syncthreads();
  float2 *keep = sKeep ? P.best + (long long)trial * P.cells : nullptr;
  const float delta = sDelta;
  for (int vt = tid; vt < XT * R2; vt += kThreads) {
    const int t = axis == 0 ? vt / R2 : vt % XT, n2 = axis == 0 ? vt % R2 : vt / XT;
    const long long lineBase = base + (long long)t * tS;
    float2 a[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) a[n1] = g[lineBase + (long long)(R2 * n1 + n2) * eS];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      if (keep) keep[lineBase + (long long)(R2 * n1 + n2) * eS] = a[n1];
      if (prologue == PRO_FLIP) {
        float re = a[n1].x;
        if (re < delta) re = -re;
        a[n1] = make_float2(re, 0.f);
      }
    }
    dft_regs<R1, N>(a, tw);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      const float2 w = tw[(n2 * k1) & (N - 1)];
      y[t * ld + n2 * ROW + k1] = make_float2(a[k1].x * w.x - a[k1].y * w.y, a[k1].x * w.y + a[k1].y * w.x);
    }
  }
  __syncthreads();
  const float scale = epilogue != EPI_NONE ? 1.0f / (float)P.cells : 1.0f;
  double sa = 0, sb = 0;
  for (int vt = tid; vt < XT * R1; vt += kThreads) {
    const int t = axis == 0 ? vt / R1 : vt % XT, k1 = axis == 0 ? vt % R1 : vt / XT;
    const long long lineBase = base + (long long)t * tS;
    float2 a[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) a[n2] = y[t * ld + n2 * ROW + k1];
    dft_regs<R2, N>(a, tw);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      float2 x = a[k2];
      if (epilogue != EPI_NONE) {
        x.x *= scale;
        x.y *= scale;
      }
      g[lineBase + (long long)(k1 + R1 * k2) * eS] = x;
      sa += (double)x.x;
      sb += (double)x.x * (double)x.x;
    }
  }
  if (epilogue == EPI_SCALE_MOMENTS) {
    block_sum2(sa, sb, red);
    if (tid == 0) P.moments[(long long)trial * P.tiles + tile] = make_double2(sa, sb);
  }
}

// The common case of the reciprocal step: a cluster whose orbits are
// consecutive in the member table and hold at most 32 members together.  Each
// lane keeps one member's F in registers through the R terms, repartition,
// symmetrisation and constraint (per-orbit sums by shuffles), so the grid is
// read and written once.  Same arithmetic as the general path below.
__device__ __forceinline__ bool cluster_in_registers(const Params &P, float2 *g, int c, int o0, int no, double obs,
                                                     int lane, float lam, bool doSym, uint32_t seed,
                                                     const uint8_t *weak, double &dSum, double &tSum) {
  if (no > 32) return false;
  const int m0 = (int)P.orbitStart[o0];
  // lane j < no reads orbit o0 + j; the members must be consecutive and few
  int myStart = 0, myCnt = 0;
  if (lane < no) {
    myStart = (int)P.orbitStart[o0 + lane];
    myCnt = (int)P.orbitCount[o0 + lane];
  }
  int end = myStart + myCnt;
  const int prevEnd = __shfl_up_sync(0xffffffffu, end, 1);
  const bool chain = lane == 0 || lane >= no || myStart == prevEnd;
  if (!__all_sync(0xffffffffu, chain)) return false;
  const int total_m = __shfl_sync(0xffffffffu, end, no - 1) - m0;
  if (total_m > 32) return false;
  // this lane's member and its orbit (local index j)
  const bool live = lane < total_m;
  const int p = m0 + lane;
  int j = 0;
  for (int q = 1; q < no; ++q)
    if (p >= __shfl_sync(0xffffffffu, myStart, q)) j = q;
  const int cnt = __shfl_sync(0xffffffffu, myCnt, j);
  uint32_t word = 0, idx = 0;
  float2 f = make_float2(0.f, 0.f);
  float cr = 0.f, ci = 0.f;
  if (live) {
    word = P.orbitIdx[p];
    idx = word & kIdxMask;
    f = g[idx];
    cr = P.phase[2 * p];
    ci = P.phase[2 * p + 1];
  }
  const double f2 = live ? (double)f.x * f.x + (double)f.y * f.y : 0.0;
  const double total = warp_sum(f2);
  const double tObs = sqrt(fmax(0.0, obs));
  dSum += fabs(sqrt(fmax(0.0, total)) - tObs);
  tSum += tObs;
  // per-orbit |F|^2 and, for the symmetrisation, the reduced sums
  const float b0 = (word & kConjBit) ? -f.y : f.y;
  const float rr = live ? f.x * cr + b0 * ci : 0.f, ri = live ? b0 * cr - f.x * ci : 0.f;
  double so = 0;
  float sr = 0.f, si = 0.f;
  for (int q = 0; q < no; ++q) {
    const bool mine = live && j == q;
    const double sq = warp_sum(mine ? f2 : 0.0);
    if (j == q) so = sq;
    if (doSym) {
      const float a = warp_sumf(mine ? rr : 0.f), b = warp_sumf(mine ? ri : 0.f);
      if (j == q) {
        sr = a;
        si = b;
      }
    }
  }
  if (!live) return true;
  const double members = (double)total_m;
  const double target = total > 1e-20 ? so * (obs / total) : (members > 0 ? obs * cnt / members : 0.0);
  if (doSym && cnt >= 2) {
    const float inv = 1.0f / (float)cnt;
    sr *= inv;
    si *= inv;
    const float a = sr * cr - si * ci;
    float b = sr * ci + si * cr;
    if (word & kConjBit) b = -b;
    f = make_float2(f.x * (1.f - lam) + a * lam, f.y * (1.f - lam) + b * lam);
  }
  if (weak && weak[o0 + j]) {
    const uint32_t n = (uint32_t)P.n, h = idx % n, k = (idx / n) % n, l = idx / (n * n);
    const uint32_t mate = (n - h) % n + ((n - k) % n) * n + ((n - l) % n) * n * n;
    f = idx > mate ? make_float2(f.y, -f.x) : make_float2(-f.y, f.x);
  } else {
    const float amp = (float)sqrt(fmax(0.0, target) / (double)cnt);
    const float m = sqrtf(f.x * f.x + f.y * f.y);
    if (m > 1e-20f) {
      const float sc = amp / m;
      f = make_float2(f.x * sc, f.y * sc);
    } else {
      const uint4 r = philox4x32_10(make_uint4((uint32_t)p, 0x43465246u, 0u, 0u), make_uint2(seed, 0x52535452u));
      float sn, cs;
      sincospif(2.0f * u01(r.x), &sn, &cs);
      f = make_float2(amp * cs, amp * sn);
    }
  }
  g[idx] = f;
  return true;
}

// The reciprocal-space half of a cycle (charge_flipping.wgsl reduce_rfactor,
// repartition, symmetrize, constrain, zero_absent, zero_dc, finalize_rfactor,
// keep_best's comparison and commit_best).  The member sets of different
// clusters, the absent list and F(000) are disjoint, so one warp per cluster
// applies the reference's global kernel order exactly within its cluster.
__global__ void __launch_bounds__(kThreads) cf_reciprocal_kernel(const Params P, int trialBase) {
  __shared__ double red[2 * kWarps];
  __shared__ int sLast;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, trial = trialBase + blockIdx.y;
  float2 *g = P.grid + (long long)trial * P.cells;
  const float lamRaw = P.symLambda[trial];
  const float lam = fminf(fmaxf(lamRaw, 0.f), 1.f);
  const uint32_t seed = P.seed[trial];
  const uint8_t *weak = P.weak ? P.weak + (long long)trial * P.nOrbits : nullptr;
  const uint32_t n = (uint32_t)P.n;
  double dSum = 0, tSum = 0;
  for (int c = blockIdx.x * kWarps + warp; c < P.nClusters; c += gridDim.x * kWarps) {
    const int o0 = (int)P.clusterOrbitStart[c], no = (int)P.clusterNOrbits[c];
    const double obs = (double)P.clusterObs[c];
    if (cluster_in_registers(P, g, c, o0, no, obs, lane, lam, lamRaw > 0.f, seed, weak, dSum, tSum)) continue;
    double total = 0, members = 0;
    for (int o = o0; o < o0 + no; ++o) {
      const int st = (int)P.orbitStart[o], cnt = (int)P.orbitCount[o];
      members += cnt;
      for (int i = lane; i < cnt; i += 32) {
        const float2 f = g[P.orbitIdx[st + i] & kIdxMask];
        total += (double)f.x * f.x + (double)f.y * f.y;
      }
    }
    total = warp_sum(total);
    const double tObs = sqrt(fmax(0.0, obs));
    dSum += fabs(sqrt(fmax(0.0, total)) - tObs);
    tSum += tObs;
    for (int o = o0; o < o0 + no; ++o) {
      const int st = (int)P.orbitStart[o], cnt = (int)P.orbitCount[o];
      double so = 0;
      for (int i = lane; i < cnt; i += 32) {
        const float2 f = g[P.orbitIdx[st + i] & kIdxMask];
        so += (double)f.x * f.x + (double)f.y * f.y;
      }
      so = warp_sum(so);
      const double target = total > 1e-20 ? so * (obs / total) : (members > 0 ? obs * cnt / members : 0.0);
      if (lamRaw > 0.f && cnt >= 2) {
        float sr = 0.f, si = 0.f;
        for (int i = lane; i < cnt; i += 32) {
          const int p = st + i;
          const uint32_t word = P.orbitIdx[p];
          const float2 f = g[word & kIdxMask];
          const float b = (word & kConjBit) ? -f.y : f.y, cr = P.phase[2 * p], ci = P.phase[2 * p + 1];
          sr += f.x * cr + b * ci;
          si += b * cr - f.x * ci;
        }
        const float inv = 1.0f / (float)cnt;
        sr = warp_sumf(sr) * inv;
        si = warp_sumf(si) * inv;
        for (int i = lane; i < cnt; i += 32) {
          const int p = st + i;
          const uint32_t word = P.orbitIdx[p], idx = word & kIdxMask;
          const float cr = P.phase[2 * p], ci = P.phase[2 * p + 1];
          const float a = sr * cr - si * ci;
          float b = sr * ci + si * cr;
          if (word & kConjBit) b = -b;
          const float2 f = g[idx];
          g[idx] = make_float2(f.x * (1.f - lam) + a * lam, f.y * (1.f - lam) + b * lam);
        }
      }
      if (weak && weak[o]) {
        // a real density: each Friedel pair turns by opposite quarter-turns
        for (int i = lane; i < cnt; i += 32) {
          const uint32_t idx = P.orbitIdx[st + i] & kIdxMask;
          const float2 f = g[idx];
          const uint32_t h = idx % n, k = (idx / n) % n, l = idx / (n * n);
          const uint32_t mate = (n - h) % n + ((n - k) % n) * n + ((n - l) % n) * n * n;
          g[idx] = idx > mate ? make_float2(f.y, -f.x) : make_float2(-f.y, f.x);
        }
      } else {
        const float amp = (float)sqrt(fmax(0.0, target) / (double)cnt);
        for (int i = lane; i < cnt; i += 32) {
          const int p = st + i;
          const uint32_t idx = P.orbitIdx[p] & kIdxMask;
          const float2 f = g[idx];
          const float m = sqrtf(f.x * f.x + f.y * f.y);
          if (m > 1e-20f) {
            const float sc = amp / m;
            g[idx] = make_float2(f.x * sc, f.y * sc);
          } else {
            // a collapsed reflection restarts on a random phase (Philox draw per member and seed)
            const uint4 r = philox4x32_10(make_uint4((uint32_t)p, 0x43465246u, 0u, 0u), make_uint2(seed, 0x52535452u));
            float sn, cs;
            sincospif(2.0f * u01(r.x), &sn, &cs);
            g[idx] = make_float2(amp * cs, amp * sn);
          }
        }
      }
    }
  }
  for (long long i = (long long)blockIdx.x * kThreads + tid; i < P.nAbsent; i += (long long)gridDim.x * kThreads)
    g[P.absentIdx[i] & kIdxMask] = make_float2(0.f, 0.f);
  if (blockIdx.x == 0 && tid == 0) g[0] = make_float2(0.f, 0.f);
  // R terms: lane 0 of every warp holds its clusters' sums
  if (lane != 0) dSum = tSum = 0;
  block_sum2(dSum, tSum, red);
  if (tid == 0) {
    P.rPartial[(long long)trial * gridDim.x + blockIdx.x] = make_double2(dSum, tSum);
    __threadfence();
    const unsigned ticket = atomicAdd(&P.ticket[trial], 1u);
    sLast = ticket == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!sLast) return;
  // the last CTA of this trial: every partial is visible; sum them in a fixed order
  __threadfence();
  double a = 0, b = 0;
  for (unsigned i = tid; i < gridDim.x; i += kThreads) {
    const double2 v = __ldcg(&P.rPartial[(long long)trial * gridDim.x + i]);
    a += v.x;
    b += v.y;
  }
  block_sum2(a, b, red);
  if (tid == 0) {
    const float R = b > 0 ? (float)(a / b) : NAN;
    const int cyc = P.cycleCount[trial];
    if (cyc < P.historyCap) P.history[(long long)trial * P.historyCap + cyc] = R;
    P.cycleCount[trial] = cyc + 1;
    const int improved = (b > 0 && R < P.bestR[trial]) ? 1 : 0;
    if (improved) P.bestR[trial] = R;
    P.pending[trial] = improved;
    P.ticket[trial] = 0u;
  }
}

// After the last cycle: the best-iterate copy the next cycle's first
// transform would have made.
__global__ void __launch_bounds__(kThreads) cf_keep_kernel(const Params P) {
  const int trial = blockIdx.y;
  if (!P.pending[trial]) return;
  const float2 *src = P.grid + (long long)trial * P.cells;
  float2 *dst = P.best + (long long)trial * P.cells;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < P.cells; i += (long long)gridDim.x * kThreads)
    dst[i] = src[i];
}

}  // namespace cf
}  // namespace p6

using namespace p6;
using namespace p6::cf;

struct p6_cf_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Params P{};
  int recipCtas = 1;
  float2 *scratch = nullptr;
  std::vector<void *> allocs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;
  float lastMs = 0.f;
};

namespace {

void cf_free(p6_cf_session *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void *p : s->allocs) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

template <class T>
p6_status cf_alloc(p6_cf_session *s, T **out, size_t count) {
  void *d = nullptr;
  const cudaError_t e = cudaMalloc(&d, std::max<size_t>(1, count) * sizeof(T));
  if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
  s->allocs.push_back(d);
  *out = static_cast<T *>(d);
  return P6_OK;
}

template <class T>
p6_status cf_upload(p6_cf_session *s, const T **out, const T *src, size_t count) {
  T *d = nullptr;
  p6_status st = cf_alloc(s, &d, count);
  if (st != P6_OK) return st;
  if (count) P6_CUDA(cudaMemcpy(d, src, count * sizeof(T), cudaMemcpyHostToDevice));
  *out = d;
  return P6_OK;
}

// Launches one axis of the transform for trials [t0, t0 + trials) of `data`.
void launch_fft(const Params &P, float2 *data, int t0, int trials, int axis, int inverse, int prologue,
                int epilogue, cudaStream_t stream) {
  const dim3 grid(P.tiles, trials);
  switch (P.n) {
    case 8: cf_fft_kernel<8><<<grid, kThreads, 0, stream>>>(P, data, t0, axis, inverse, prologue, epilogue); break;
    case 16: cf_fft_kernel<16><<<grid, kThreads, 0, stream>>>(P, data, t0, axis, inverse, prologue, epilogue); break;
    case 32: cf_fft_kernel<32><<<grid, kThreads, 0, stream>>>(P, data, t0, axis, inverse, prologue, epilogue); break;
    case 64: cf_fft_kernel<64><<<grid, kThreads, 0, stream>>>(P, data, t0, axis, inverse, prologue, epilogue); break;
    default:
      cf_fft_kernel<128><<<grid, kThreads, 0, stream>>>(P, data, t0, axis, inverse, prologue, epilogue);
      break;
  }
}

// Trials per chunk: a chunk's grids (at most 32 MB, a quarter of L2) stay in
// L2 through its seven launches, so a cycle reads and writes each grid in
// HBM about once instead of once per pass.
int chunk_trials(const Params &P) {
  const long long bytes = P.cells * (long long)sizeof(float2);
  return (int)std::max<long long>(1, std::min<long long>(P.nTrials, (32LL << 20) / bytes));
}

// The seven launches of one cycle for every chunk of trials, on `stream`.
void enqueue_cycle(const p6_cf_session *s) {
  const Params &P = s->P;
  const int chunk = chunk_trials(P);
  for (int t0 = 0; t0 < P.nTrials; t0 += chunk) {
    const int nt = std::min(chunk, P.nTrials - t0);
    launch_fft(P, P.grid, t0, nt, 0, 1, PRO_KEEP, EPI_NONE, s->stream);
    launch_fft(P, P.grid, t0, nt, 1, 1, PRO_NONE, EPI_NONE, s->stream);
    launch_fft(P, P.grid, t0, nt, 2, 1, PRO_NONE, EPI_SCALE_MOMENTS, s->stream);
    launch_fft(P, P.grid, t0, nt, 2, 0, PRO_FLIP, EPI_NONE, s->stream);
    launch_fft(P, P.grid, t0, nt, 1, 0, PRO_NONE, EPI_NONE, s->stream);
    launch_fft(P, P.grid, t0, nt, 0, 0, PRO_NONE, EPI_NONE, s->stream);
    cf_reciprocal_kernel<<<dim3(s->recipCtas, nt), kThreads, 0, s->stream>>>(P, t0);
  }
}

int launches_per_cycle(const Params &P) {
  const int chunk = chunk_trials(P);
  return 7 * ((P.nTrials + chunk - 1) / chunk);
}

p6_status capture_cycle(p6_cf_session *s) {
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->exec = nullptr;
  s->graph = nullptr;
  P6_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_cycle(s);
  P6_CUDA(cudaStreamEndCapture(s->stream, &s->graph));
  P6_CUDA(cudaGraphInstantiate(&s->exec, s->graph, 0));
  return P6_OK;
}

p6_status wait_stream(p6_cf_session *s, double seconds) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s->stream);
    if (e == cudaSuccess) return P6_OK;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > seconds)
      return set_error(P6_ERR_TIMEOUT, "the device did not finish within the deadline");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

}  // namespace

extern "C" {

p6_status p6_cf_create(const p6_cf_model *m, int n_trials, const p6_cf_trial *trials, int device,
                       p6_cf_session **out) {
  clear_error();
  if (!m || !trials || !out) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  const int n = m->n;
  if (n != 8 && n != 16 && n != 32 && n != 64 && n != 128)
    return set_error(P6_ERR_INVALID_ARG, "grid edge must be 8, 16, 32, 64 or 128");
  if (n_trials < 1 || n_trials > kMaxTrials) return set_error(P6_ERR_CAPACITY, "1 to 4096 trials");
  if (m->n_orbits < 1 || m->n_clusters < 1 || m->n_members < 1 || m->n_absent < 0)
    return set_error(P6_ERR_INVALID_ARG, "empty reflection model");
  if (!m->orbit_start || !m->orbit_count || !m->orbit_idx || !m->phase || !m->cluster_orbit_start ||
      !m->cluster_n_orbits || !m->cluster_obs_i || (m->n_absent > 0 && !m->absent_idx))
    return set_error(P6_ERR_INVALID_ARG, "null table pointer");
  const long long cells = (long long)n * n * n;
  // every grid point is written by at most one thread of the reciprocal step:
  // members unique, none at F(000), none absent
  std::vector<uint8_t> owner((size_t)cells, 0);
  owner[0] = 3;
  for (int i = 0; i < m->n_absent; ++i) {
    const uint32_t idx = m->absent_idx[i] & kIdxMask;
    if ((long long)idx >= cells) return set_error(P6_ERR_INVALID_ARG, "absent index outside the grid");
    owner[idx] = 2;
  }
  std::vector<uint8_t> inCluster(m->n_orbits, 0);
  for (int c = 0; c < m->n_clusters; ++c) {
    const long long a = m->cluster_orbit_start[c], b = a + (long long)m->cluster_n_orbits[c];
    if (b > m->n_orbits) return set_error(P6_ERR_INVALID_ARG, "cluster orbits outside the orbit table");
    for (long long o = a; o < b; ++o) {
      if (inCluster[o]) return set_error(P6_ERR_INVALID_ARG, "an orbit belongs to two clusters");
      inCluster[o] = 1;
    }
  }
  for (int o = 0; o < m->n_orbits; ++o) {
    const long long a = m->orbit_start[o], b = a + (long long)m->orbit_count[o];
    if (m->orbit_count[o] < 1 || b > m->n_members)
      return set_error(P6_ERR_INVALID_ARG, "orbit members outside the member table");
    for (long long p = a; p < b; ++p) {
      const uint32_t idx = m->orbit_idx[p] & kIdxMask;
      if ((long long)idx >= cells) return set_error(P6_ERR_INVALID_ARG, "member index outside the grid");
      if (owner[idx]) return set_error(P6_ERR_INVALID_ARG, "a grid point is claimed twice, absent, or F(000)");
      owner[idx] = 1;
    }
  }
  for (int t = 0; t < n_trials; ++t)
    if (!std::isfinite(trials[t].delta_sigma) || !std::isfinite(trials[t].sym_lambda))
      return set_error(P6_ERR_INVALID_ARG, "non-finite trial setting");

  p6_cf_session *s = new p6_cf_session();
  s->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { cf_free(s); return cuda_error(e, "cudaSetDevice"); }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
  if (e != cudaSuccess) { cf_free(s); return cuda_error(e, "stream / event creation"); }

  Params &P = s->P;
  P.n = n;
  P.tiles = n * n / tile_lines(n);
  P.nTrials = n_trials;
  P.cells = cells;
  P.nOrbits = m->n_orbits;
  P.nClusters = m->n_clusters;
  P.nAbsent = m->n_absent;
  s->recipCtas = std::max(1, std::min((m->n_clusters + kWarps - 1) / kWarps, 1024));
  std::vector<float> ds(n_trials), sl(n_trials);
  std::vector<uint32_t> sd(n_trials);
  std::vector<uint8_t> wk((size_t)n_trials * m->n_orbits, 0);
  bool anyWeak = false;
  for (int t = 0; t < n_trials; ++t) {
    ds[t] = trials[t].delta_sigma;
    sl[t] = trials[t].sym_lambda;
    sd[t] = trials[t].seed;
    if (trials[t].weak) {
      for (int o = 0; o < m->n_orbits; ++o) wk[(size_t)t * m->n_orbits + o] = trials[t].weak[o] ? 1 : 0;
      anyWeak = true;
    }
  }
  p6_status st = P6_OK;
#define CF_TRY(x)               \
  do {                          \
    st = (x);                   \
    if (st != P6_OK) {          \
      cf_free(s);               \
      return st;                \
    }                           \
  } while (0)
  CF_TRY(cf_upload(s, &P.orbitStart, m->orbit_start, m->n_orbits));
  CF_TRY(cf_upload(s, &P.orbitCount, m->orbit_count, m->n_orbits));
  CF_TRY(cf_upload(s, &P.orbitIdx, m->orbit_idx, m->n_members));
  CF_TRY(cf_upload(s, &P.phase, m->phase, 2 * (size_t)m->n_members));
  CF_TRY(cf_upload(s, &P.clusterOrbitStart, m->cluster_orbit_start, m->n_clusters));
  CF_TRY(cf_upload(s, &P.clusterNOrbits, m->cluster_n_orbits, m->n_clusters));
  CF_TRY(cf_upload(s, &P.clusterObs, m->cluster_obs_i, m->n_clusters));
  CF_TRY(cf_upload(s, &P.absentIdx, m->absent_idx, m->n_absent));
  CF_TRY(cf_upload(s, &P.deltaSigma, ds.data(), n_trials));
  CF_TRY(cf_upload(s, &P.symLambda, sl.data(), n_trials));
  CF_TRY(cf_upload(s, &P.seed, sd.data(), n_trials));
  if (anyWeak) CF_TRY(cf_upload(s, &P.weak, wk.data(), wk.size()));
  CF_TRY(cf_alloc(s, &P.grid, (size_t)n_trials * cells));
  CF_TRY(cf_alloc(s, &P.best, (size_t)n_trials * cells));
  CF_TRY(cf_alloc(s, &s->scratch, (size_t)cells));
  CF_TRY(cf_alloc(s, &P.moments, (size_t)n_trials * P.tiles));
  CF_TRY(cf_alloc(s, &P.rPartial, (size_t)n_trials * s->recipCtas));
  CF_TRY(cf_alloc(s, &P.ticket, n_trials));
  CF_TRY(cf_alloc(s, &P.bestR, n_trials));
  CF_TRY(cf_alloc(s, &P.pending, n_trials));
  CF_TRY(cf_alloc(s, &P.cycleCount, n_trials));
  P.historyCap = 256;
  CF_TRY(cf_alloc(s, &P.history, (size_t)n_trials * P.historyCap));
#undef CF_TRY
  std::vector<float> inf(n_trials, INFINITY);
  e = cudaMemset(P.grid, 0, (size_t)n_trials * cells * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemset(P.best, 0, (size_t)n_trials * cells * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemset(P.ticket, 0, n_trials * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(P.pending, 0, n_trials * sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(P.bestR, inf.data(), n_trials * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cf_free(s); return cuda_error(e, "session initialisation"); }
  st = capture_cycle(s);
  if (st != P6_OK) { cf_free(s); return st; }
  *out = s;
  return P6_OK;
}

p6_status p6_cf_destroy(p6_cf_session *s) {
  clear_error();
  cf_free(s);
  return P6_OK;
}

p6_status p6_cf_set_grid(p6_cf_session *s, int trial, const float *grid) {
  clear_error();
  if (!s || !grid) return set_error(P6_ERR_INVALID_ARG, "null argument");
  const Params &P = s->P;
  if (trial >= P.nTrials) return set_error(P6_ERR_INVALID_ARG, "trial out of range");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t bytes = (size_t)P.cells * sizeof(float2);
  const int t0 = trial < 0 ? 0 : trial, t1 = trial < 0 ? P.nTrials : trial + 1;
  const float inf = INFINITY;
  for (int t = t0; t < t1; ++t) {
    P6_CUDA(cudaMemcpyAsync(P.grid + (size_t)t * P.cells, grid, bytes, cudaMemcpyHostToDevice, s->stream));
    P6_CUDA(cudaMemcpyAsync(P.best + (size_t)t * P.cells, P.grid + (size_t)t * P.cells, bytes,
                            cudaMemcpyDeviceToDevice, s->stream));
    P6_CUDA(cudaMemcpyAsync(P.bestR + t, &inf, sizeof(float), cudaMemcpyHostToDevice, s->stream));
    P6_CUDA(cudaMemsetAsync(P.pending + t, 0, sizeof(int), s->stream));
  }
  return wait_stream(s, 60.0);
}

p6_status p6_cf_run(p6_cf_session *s, int cycles, float *r_history) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (cycles < 0) return set_error(P6_ERR_INVALID_ARG, "negative cycle count");
  P6_CUDA(cudaSetDevice(s->device));
  Params &P = s->P;
  if (cycles > P.historyCap) {
    float *h = nullptr;
    p6_status st = cf_alloc(s, &h, (size_t)P.nTrials * cycles);
    if (st != P6_OK) return st;
    P.history = h;   // the smaller buffer stays in the session's allocation list until destroy
    P.historyCap = cycles;
    st = capture_cycle(s);
    if (st != P6_OK) return st;
  }
  P6_CUDA(cudaMemsetAsync(P.cycleCount, 0, P.nTrials * sizeof(int), s->stream));
  P6_CUDA(cudaEventRecord(s->ev0, s->stream));
  for (int c = 0; c < cycles; ++c) P6_CUDA(cudaGraphLaunch(s->exec, s->stream));
  const int keepCtas = (int)std::min<long long>(1024, (P.cells + kThreads - 1) / kThreads);
  cf_keep_kernel<<<dim3(keepCtas, P.nTrials), kThreads, 0, s->stream>>>(P);
  P6_CUDA(cudaGetLastError());
  P6_CUDA(cudaMemsetAsync(P.pending, 0, P.nTrials * sizeof(int), s->stream));
  P6_CUDA(cudaEventRecord(s->ev1, s->stream));
  s->launches += (long long)launches_per_cycle(P) * cycles + 1;
  std::vector<float> hist;
  if (r_history && cycles > 0) {
    hist.resize((size_t)P.nTrials * P.historyCap);
    P6_CUDA(cudaMemcpyAsync(hist.data(), P.history, hist.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  }
  const double budget = 60.0 + 1e-8 * (double)cycles * (double)P.nTrials * (double)P.cells;
  p6_status st = wait_stream(s, budget);
  if (st != P6_OK) return st;
  P6_CUDA(cudaEventElapsedTime(&s->lastMs, s->ev0, s->ev1));
  if (r_history && cycles > 0)
    for (int t = 0; t < P.nTrials; ++t)
      std::copy(hist.begin() + (size_t)t * P.historyCap, hist.begin() + (size_t)t * P.historyCap + cycles,
                r_history + (size_t)t * cycles);
  return P6_OK;
}

p6_status p6_cf_best_r(p6_cf_session *s, float *best_r) {
  clear_error();
  if (!s || !best_r) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaMemcpyAsync(best_r, s->P.bestR, s->P.nTrials * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  return wait_stream(s, 60.0);
}

p6_status p6_cf_read(p6_cf_session *s, int trial, int which, float *out) {
  clear_error();
  if (!s || !out) return set_error(P6_ERR_INVALID_ARG, "null argument");
  const Params &P = s->P;
  if (trial < 0 || trial >= P.nTrials) return set_error(P6_ERR_INVALID_ARG, "trial out of range");
  if (which < 0 || which > 2) return set_error(P6_ERR_INVALID_ARG, "which must be 0, 1 or 2");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t bytes = (size_t)P.cells * sizeof(float2);
  if (which < 2) {
    const float2 *src = (which == 0 ? P.grid : P.best) + (size_t)trial * P.cells;
    P6_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, s->stream));
    return wait_stream(s, 60.0);
  }
  P6_CUDA(cudaMemcpyAsync(s->scratch, P.best + (size_t)trial * P.cells, bytes, cudaMemcpyDeviceToDevice, s->stream));
  launch_fft(P, s->scratch, 0, 1, 0, 1, PRO_NONE, EPI_NONE, s->stream);
  launch_fft(P, s->scratch, 0, 1, 1, 1, PRO_NONE, EPI_NONE, s->stream);
  launch_fft(P, s->scratch, 0, 1, 2, 1, PRO_NONE, EPI_SCALE, s->stream);
  P6_CUDA(cudaGetLastError());
  s->launches += 3;
  P6_CUDA(cudaMemcpy2DAsync(out, sizeof(float), s->scratch, sizeof(float2), sizeof(float), (size_t)P.cells,
                            cudaMemcpyDeviceToHost, s->stream));
  return wait_stream(s, 60.0);
}

p6_status p6_cf_last_ms(p6_cf_session *s, float *ms) {
  clear_error();
  if (!s || !ms) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *ms = s->lastMs;
  return P6_OK;
}

p6_status p6_cf_time_kernels(p6_cf_session *s, int cycles, float *fft_pass_ms, float *reciprocal_ms) {
  clear_error();
  if (!s || !fft_pass_ms || !reciprocal_ms || cycles < 1) return set_error(P6_ERR_INVALID_ARG, "bad argument");
  P6_CUDA(cudaSetDevice(s->device));
  const Params &P = s->P;
  cudaEvent_t ea, eb, ec;
  P6_CUDA(cudaEventCreate(&ea));
  P6_CUDA(cudaEventCreate(&eb));
  P6_CUDA(cudaEventCreate(&ec));
  double fft = 0, rec = 0;
  p6_status st = P6_OK;
  const int chunk = chunk_trials(P);
  for (int c = 0; c < cycles && st == P6_OK; ++c)
    for (int t0 = 0; t0 < P.nTrials && st == P6_OK; t0 += chunk) {
      const int nt = std::min(chunk, P.nTrials - t0);
      cudaEventRecord(ea, s->stream);
      launch_fft(P, P.grid, t0, nt, 0, 1, PRO_KEEP, EPI_NONE, s->stream);
      launch_fft(P, P.grid, t0, nt, 1, 1, PRO_NONE, EPI_NONE, s->stream);
      launch_fft(P, P.grid, t0, nt, 2, 1, PRO_NONE, EPI_SCALE_MOMENTS, s->stream);
      launch_fft(P, P.grid, t0, nt, 2, 0, PRO_FLIP, EPI_NONE, s->stream);
      launch_fft(P, P.grid, t0, nt, 1, 0, PRO_NONE, EPI_NONE, s->stream);
      launch_fft(P, P.grid, t0, nt, 0, 0, PRO_NONE, EPI_NONE, s->stream);
      cudaEventRecord(eb, s->stream);
      cf_reciprocal_kernel<<<dim3(s->recipCtas, nt), kThreads, 0, s->stream>>>(P, t0);
      cudaEventRecord(ec, s->stream);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) { st = cuda_error(e, "kernel launch"); break; }
      st = wait_stream(s, 60.0);
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, ea, eb);
      cudaEventElapsedTime(&b, eb, ec);
      fft += a;
      rec += b;
      s->launches += 7;
    }
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  cudaEventDestroy(ec);
  if (st != P6_OK) return st;
  // per pass over every trial, and per reciprocal step over every trial
  *fft_pass_ms = (float)(fft / (6.0 * cycles));
  *reciprocal_ms = (float)(rec / cycles);
  return P6_OK;
}

p6_status p6_cf_launch_count(p6_cf_session *s, long long *count) {
  clear_error();
  if (!s || !count) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *count = s->launches;
  return P6_OK;
}

}  // extern "C"
