// Parallel-tempering Rietveld trial evaluation on sm_100a.
//
// Replaces the WebGPU backend of js/pt_gpu.js (compile / create / costs /
// batch / run, :20-423): per chain, propose one coordinate (Gaussian step x
// scale x sqrt(T), reflected into the bounds), evaluate the full powder
// pattern -- reflections of the trial cell, |F|^2 over the coset
// representatives, TCH pseudo-Voigt profiles with the K-alpha-2 doublet and
// pedestal, Lorentz-polarisation, Chebyshev background -- and the weighted
// chi^2, then the Metropolis test on chi^2/2 (js/rietveld_core.js:2171-2241).
//
// B200 layout:
//  * one CTA per chain, one launch per sweep (nv proposals).  The adjacent
//    exchange of the previous sweep runs at the start of the launch: both
//    chains of a pair read the previous state (double-buffered) and derive
//    the same decision from the same counter-based draw, so nothing is
//    synchronised across CTAs and a sequence of sweeps can be captured in a
//    CUDA graph;
//  * the observed pattern is staged once per launch into shared memory;
//  * per-reflection work (geometry, widths, areas, pedestals, Lp, weights) is
//    FP64 -- a few dozen peaks per trial, and peak positions need it; the
//    per-point profile shape is FP32 on an FP64 offset from the peak, and the
//    chi^2 is accumulated and reduced in FP64;
//  * |F|^2 takes a warp per reflection with the lanes over the coset
//    representatives; the phase is reduced to one turn in FP64 before the
//    FP32 sine and cosine.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "p6_common.cuh"

namespace p6 {
namespace pt {

constexpr int kThreads = 1024;   // one CTA per chain: 32 warps hide the latency of the evaluation
constexpr int kWarps = kThreads / 32;
constexpr int kMaxNv = 32;
constexpr int kMaxFull = 64;
constexpr double kPi = 3.14159265358979323846;
constexpr double kD2R = kPi / 180.0;
constexpr double kR2D = 180.0 / kPi;
constexpr double kGconv = 0.023548200450309493;   // sqrt(8 ln 2) / 100
constexpr double kLconv = 0.01;
constexpr double kCg = 2.772588722239781;         // 4 ln 2
constexpr double kWinG = 8.0, kWinL = 25.0, kWinMax = 10.0;

enum { SCALE = 0, PA, PB, PC, PAL, PBE, PGA, PU, PV, PW, PX, PY, PZERO, PBISO, PBKG0 };

// Chain state (device, FP64); the reference layout is produced on read-back.
struct Chain {
  double x[kMaxNv];
  double best[kMaxNv];
  double cost, bestCost;
  double sweep, accepted, proposals, swaps, swapAttempts, valid, logu, unsolved, proposalCost, feasible;
};

struct Peak {            // one contribution (K-alpha-1 or K-alpha-2) of a reflection
  double x0, maxd;       // centre and truncation radius, degrees
  float inv, cL, cG, pedestal;
  float asym;            // SL / tan(theta) + HL (0: symmetric)
  int lo, hi;            // window [lo, hi) in point indices
};

struct PeakD {           // the same in FP64 throughout (least-squares finish)
  double x0, maxd;
  double inv, cL, cG, pedestal;
  double asym;
  int lo, hi;
};

struct Params {
  int nRefl, nReps, nAtoms, n, nBkg, nFull, nv, chains, cubic;
  const int *hkl;        // nRefl * 3 (envelope)
  const int *mult;
  const int *repRot;     // nReps * 9
  const double *repTrans;// nReps * 3
  const double *atomPos, *atomW, *atomOcc, *ffA, *ffB, *ffC;
  const double *tth, *y;
  const float *w;
  const double *wd;      // the weights in FP64 (least-squares finish)
  double lambda1, lambda2, ratio, polK, minFwhm, qmax;
  const double *full;    // base full parameter vector
  const int *index;      // nv -> full index
  const double *lo, *hi, *scales;
  double maxTemp;
  uint32_t seed;
  int stageObs;          // observed pattern staged in shared memory
  int *errFlag;
  int hasPo;             // March-Dollase factor on; r = v[PBKG0 + nBkg]
  int asymIdx;           // full index of SL (HL follows); -1: no asymmetry
  int shiftIdx;          // full index of the displacement (transparency follows); -1: none
  int method;            // 0 Rietveld; 1 WPPF / Le Bail: heights free, solved per evaluation by NNLS
  const int *eqStart;    // nRefl + 1
  const int *eqHkl;      // 3 per equivalent
  double poDir[3];       // reciprocal-lattice direction
  // per chain, the decisions of the last sweep: {exchange tried, swapped, la,
  // log u} then per move {j, proposed x_j, log u, cost before, cost, accepted}
  double *trace;
};
constexpr int kTraceHead = 4, kTraceMove = 6;

// ---------------------------------------------------------------------------
// Profile model (FP64 per peak).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double soft_positive(double x, double f) {
  if (!isfinite(x)) return f;
  const double h = hypot(x, 2 * f);
  return x < 0 ? f * (f / (0.5 * h - 0.5 * x)) : 0.5 * x + 0.5 * h;
}
__device__ __forceinline__ double soft_floor(double x, double f) {
  if (!isfinite(x) || !(x > 0)) return f;
  if (!(f > 0)) return x;
  const double r = x / f;
  if (r > 20) return x;
  const double r2 = r * r;
  return f * sqrt(sqrt(r2 * r2 + 1));   // f (r^4 + 1)^(1/4)
}
__device__ __forceinline__ double peak_fwhm(double gG, double gL) {
  gG = fmax(1e-9, gG != 0 ? gG : 1e-9);
  gL = fmax(1e-9, gL != 0 ? gL : 1e-9);
  const double g2 = gG * gG, g3 = g2 * gG, g4 = g2 * g2, l2 = gL * gL, l3 = l2 * gL, l4 = l2 * l2;
  const double s = g4 * gG + 2.69269 * g4 * gL + 2.42843 * g3 * l2 + 4.47163 * g2 * l3 + 0.07842 * gG * l4 + l4 * gL;
  if (s < 0 || !isfinite(s)) return fmax(fmax(gG, gL), 1e-6);
  return fmax(1e-6, pow(s, 0.2));
}
__device__ __forceinline__ double voigt64(double delta, double inv, double cL, double cG, double pedestal) {
  const double dg = (delta * inv) * (delta * inv);
  const double v = cL * (1.0 / (1.0 + 4.0 * dg)) + cG * exp(-kCg * dg) - pedestal;
  return v > 0 ? v : 0.0;
}
// SL/HL axial-divergence asymmetry (js/profile.js:737-740): one flank is
// stretched and the other compressed, delta / (1 - t), t = asym delta
// clamped at +-0.95.  asym = 0 returns delta unchanged.
__device__ __forceinline__ double asym_delta(double delta, double asym) {
  if (asym != 0 && fabs(delta) >= 1e-9) delta /= 1.0 - fmax(-0.95, fmin(0.95, asym * delta));
  return delta;
}
__device__ __forceinline__ float asym_deltaf(float delta, float asym) {
  if (asym != 0.f && fabsf(delta) >= 1e-9f) delta /= 1.0f - fmaxf(-0.95f, fminf(0.95f, asym * delta));
  return delta;
}
// asymmetryAreaCorrection (js/profile.js:799-826): the area the asymmetry adds
// to a unit-height peak of width H, mixing (cL, cG), window R.  The
// (asymmetric - symmetric) difference is integrated with 8-point
// Gauss-Legendre panels that double in width from 0.25 H out to
// D = max(R, min(0.95 / |a|, 4096 H)), split at the clamp point; beyond D the
// stretch is a constant k and both tails are closed-form.
__device__ double asym_area(double a, double H, double cL, double cG, double R) {
  if (a == 0 || !(R > 0)) return 0.0;
  const double inv = 1 / H, w = fmax(1e-6, H);
  const double clampAt = 0.95 / fabs(a), D = fmax(R, fmin(clampAt, 4096 * w));
  const double gx[4] = {0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363};
  const double gw[4] = {0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
  auto panel = [&](double lo, double hi, double side) {
    const double m = 0.5 * (lo + hi), h = 0.5 * (hi - lo);
    double s = 0;
    for (int i = 0; i < 4; ++i)
      for (int sg = -1; sg <= 1; sg += 2) {
        const double d = side * (m + sg * h * gx[i]);
        s += gw[i] * (voigt64(asym_delta(d, a), inv, cL, cG, 0.0) - voigt64(d, inv, cL, cG, 0.0));
      }
    return s * h;
  };
  auto tail = [&](double x) {
    return cL * 0.5 * H * (0.5 * kPi - atan(2 * x / H)) + cG * 0.5 * H * sqrt(kPi / kCg) * erfc(sqrt(kCg) * x / H);
  };
  double total = 0;
  for (int sd = 0; sd < 2; ++sd) {
    const double side = sd ? 1.0 : -1.0;
    double lo = 0, e = 0.25 * w;
    for (int it = 0; it < 64; ++it) {
      const double hi = fmin(e, D);
      if (clampAt > lo && clampAt < hi) {
        total += panel(lo, clampAt, side);
        lo = clampAt;
      }
      total += panel(lo, hi, side);
      lo = hi;
      if (hi >= D) break;
      e *= 2;
    }
    const double k = 1 - fmax(-0.95, fmin(0.95, a * side * D));
    total += k * tail(D / k) - tail(D);
  }
  return total;
}
// Sample displacement and transparency shift of a peak at 2-theta t
// (js/pt_gpu.js:355, :169-171): (-disp 1e-3 cos(theta) + transp sin(2 theta))
// in degrees, 0 at theta = 90 degrees and wherever it is not finite.
__host__ __device__ inline double sample_shift(double t, double disp, double transp) {
  const double th = t * kD2R * 0.5;
  if (fabs(th - 0.5 * kPi) < 1e-6) return 0.0;
  const double d = (-disp * 0.001 * cos(th) + transp * sin(2.0 * th)) / kD2R;
  return isfinite(d) ? d : 0.0;
}

// prepareVoigt, TCH branch (js/profile.js:603-722): widths at tthPeak, centre
// x0, the SL/HL asymmetry when asymIdx >= 0 (v[asymIdx] = SL, v[asymIdx + 1]
// = HL).  Returns the area of the unit-height peak (analytic, plus the
// asymmetry's correction).
template <class PK>
__device__ double prepare(const double *v, double minFwhm, double tthPeak, double x0, int asymIdx, PK &p) {
  double asym = 0;
  if (asymIdx >= 0) {
    const double SL = v[asymIdx], HL = v[asymIdx + 1];
    if ((SL != 0 || HL != 0) && tthPeak >= 0.1 && tthPeak < 180) {
      const double th = fmax(1e-6, fmin(kPi / 2.0 - 1e-6, tthPeak * (kPi / 180) / 2.0)), t = tan(th);
      if (fabs(t) >= 1e-9) asym = SL / t + HL;
    }
  }
  double gG = minFwhm, gL = minFwhm;
  const double theta = tthPeak * (kPi / 180) / 2;
  const double safe = fmin(theta, kPi / 2.0 - 1e-6);
  if (!(safe < 1e-6)) {
    const double t = tan(safe), c = cos(safe), cs = fmax(c, 1e-9);
    const double sig2 = v[PU] * t * t + v[PV] * t + v[PW];
    const double fq = 0.25 * minFwhm / kGconv, floorSq = fq * fq;
    gG = sqrt(soft_positive(sig2, floorSq)) * kGconv;
    gL = soft_positive(v[PX] / cs + v[PY] * t, 0.25 * minFwhm / kLconv) * kLconv;
  }
  gG = soft_floor(gG, minFwhm);
  gL = soft_floor(gL, minFwhm);
  const double HG = fmax(1e-9, gG), HL = fmax(1e-9, gL);
  const double fwhm = fmax(1e-9, peak_fwhm(HG, HL));
  double eta = 0;
  if (fwhm > 1e-9) {
    const double r = HL / fwhm;
    eta = fmax(0.0, fmin(1.0, 1.36603 * r - 0.47719 * (r * r) + 0.11116 * (r * r * r)));
  }
  const double g0 = 2.0 * sqrt(log(2.0) / kPi), l0 = 2.0 / kPi;
  const double e = fmax(0.0, fmin(1.0, eta));
  const double wL = e * l0 / fmax(1e-12, fwhm), wG = (1 - e) * g0 / fmax(1e-12, fwhm), s = wL + wG;
  double cL = e, cG = 1 - e;
  if (s > 0 && isfinite(s)) { cL = wL / s; cG = wG / s; }
  const double inv = 1 / fwhm;
  const double mult = kWinG + (kWinL - kWinG) * fmax(0.0, fmin(1.0, eta));
  const double R = fmin(kWinMax, mult * fmax(0.01, fmax(1e-6, fwhm)) * (asym != 0 ? 2.0 : 1.0));
  const double ped =
      fmax(voigt64(asym_delta(R, asym), inv, cL, cG, 0.0), voigt64(asym_delta(-R, asym), inv, cL, cG, 0.0));
  p.x0 = x0;
  p.maxd = R;
  using T = decltype(p.inv);
  p.inv = (T)inv;
  p.cL = (T)cL;
  p.cG = (T)cG;
  p.pedestal = (T)ped;
  p.asym = (T)asym;
  return (cL * (1 / l0) + cG * (1 / g0)) * fwhm + asym_area(asym, fwhm, cL, cG, R);
}
__device__ __forceinline__ double lp_factor(double tth, double K) {
  if (!isfinite(tth) || tth <= 0 || tth >= 180) return 1;
  const double th = 0.5 * tth * kD2R, s = sin(th), c = cos(th);
  if (s < 1e-6 || c < 1e-6) return 1;
  const double k = (isfinite(K) && K >= 0) ? K : 1;
  const double c2 = cos(tth * kD2R);
  return (1 / (s * s * c)) * ((1 + k * c2 * c2) / (1 + k));
}
__device__ __forceinline__ int lower_bound(const double *a, int n, double t) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// First index >= from with a[i] > t (the end of a window that starts at from).
__device__ __forceinline__ int upper_bound(const double *a, int n, double t, int from) {
  int lo = from, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Reciprocal metric of the cell (buildInvDsq): aa bb cc ab bc ac; false if degenerate.
__device__ bool inv_dsq_form(const double *v, double f[6]) {
  const double a = v[PA], b = v[PB], c = v[PC];
  const double al = v[PAL] * kD2R, be = v[PBE] * kD2R, ga = v[PGA] * kD2R;
  const double cA = cos(al), cB = cos(be), cG = cos(ga), sA = sin(al), sB = sin(be), sG = sin(ga);
  const double vf = 1 - cA * cA - cB * cB - cG * cG + 2 * cA * cB * cG;
  if (!(a > 0 && b > 0 && c > 0) || vf <= 1e-9 || fabs(sA) < 1e-9 || fabs(sB) < 1e-9 || fabs(sG) < 1e-9) return false;
  const double V = a * b * c * sqrt(vf);
  const double as = b * c * sA / V, bs = a * c * sB / V, cs = a * b * sG / V;
  const double cAs = (cB * cG - cA) / (sB * sG), cBs = (cA * cG - cB) / (sA * sG), cGs = (cA * cB - cG) / (sA * sB);
  f[0] = as * as; f[1] = bs * bs; f[2] = cs * cs;
  f[3] = 2 * as * bs * cGs; f[4] = 2 * bs * cs * cAs; f[5] = 2 * as * cs * cBs;
  return true;
}

// March-Dollase factor of reflection k (js/rietveld_core.js:824-853): the
// mean of (r^2 cos^2 a + sin^2 a / r)^(-3/2) over the reflection's
// equivalents, a the angle to poDir in the reciprocal metric f (the 1/d^2
// form).  Warp-collective (lanes over the equivalents); every lane returns it.
__device__ double po_factor(const Params &P, const double f[6], double r, int k, int lane) {
  if (!(r > 0) || fabs(r - 1) < 1e-12) return 1.0;
  auto g = [&](double a0, double a1, double a2, double b0, double b1, double b2) {
    return a0 * b0 * f[0] + a1 * b1 * f[1] + a2 * b2 * f[2] + (a0 * b1 + a1 * b0) * f[3] / 2 +
           (a1 * b2 + a2 * b1) * f[4] / 2 + (a0 * b2 + a2 * b0) * f[5] / 2;
  };
  const double d0 = P.poDir[0], d1 = P.poDir[1], d2 = P.poDir[2];
  const double HH = g(d0, d1, d2, d0, d1, d2);
  if (!(HH > 0)) return 1.0;
  const int e0 = P.eqStart[k], e1 = P.eqStart[k + 1];
  const double r2 = r * r, ir = 1 / r;
  double sum = 0;
  for (int e = e0 + lane; e < e1; e += 32) {
    const double h0 = P.eqHkl[3 * e], h1 = P.eqHkl[3 * e + 1], h2 = P.eqHkl[3 * e + 2];
    const double hh = g(h0, h1, h2, h0, h1, h2), c = g(h0, h1, h2, d0, d1, d2) / sqrt(hh * HH);
    const double c2 = fmin(1.0, c * c), x = r2 * c2 + (1 - c2) * ir;
    sum += 1.0 / (x * sqrt(x));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  return e1 > e0 ? sum / (e1 - e0) : 1.0;
}

// ---------------------------------------------------------------------------
// One full cost evaluation of the parameter vector in shared memory `v`.
// All threads call it; returns chi^2 on every thread (INF if invalid).
// ---------------------------------------------------------------------------
struct Shared {
  double v[kMaxFull];
  double f[6];
  int valid;
  double warpChi[kWarps];
  double chiPart;   // this CTA's share of chi^2 when a chain spans a cluster
  double chi;
};

// Per-reflection stage of one evaluation: |F|^2 (warp per reflection, lanes
// over the coset representatives) and, on lane 0, the K-alpha-1/2 peaks,
// heights and windows.  F64 = false: FP32 structure-factor sums and FP32
// peak shapes (the tempering cost); F64 = true: FP64 throughout, with the
// unit-scale heights u1 for the scale column of the least-squares finish.
template <bool F64, class PK, class H>
__device__ void reflection_stage(const Params &P, const Shared &sh, PK *pk1, PK *pk2, H *h1, H *w2, double *u1,
                                 int *act, const double *tth, const float *f2read = nullptr,
                                 float *f2write = nullptr) {
  using A_t = typename std::conditional<F64, double, float>::type;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double *v = sh.v;
  const int nR = P.nRefl;
  const bool doublet = P.ratio > 1e-6 && P.lambda2 > 1e-6 && fabs(P.lambda1 - P.lambda2) > 1e-6;
  // |F|^2: warp per reflection, lanes over the coset representatives
  for (int k = warp; k < nR; k += kWarps) {
    if (f2read) {   // |F|^2 (x March-Dollase) of these cell, Biso and r values, computed by an earlier move
      if (lane == 0) h1[k] = (H)f2read[k];
      continue;
    }
    const int hh = P.hkl[3 * k], kk = P.hkl[3 * k + 1], ll = P.hkl[3 * k + 2];
    const double q = hh * hh * sh.f[0] + kk * kk * sh.f[1] + ll * ll * sh.f[2] + hh * kk * sh.f[3] +
                     kk * ll * sh.f[4] + hh * ll * sh.f[5];
    const double s = sqrt(q), sinT = P.lambda1 * s / 2;
    const bool live = q > 0 && q <= P.qmax && sinT < 1;
    A_t A = 0, B = 0;
    if (live) {
      const double s2 = s * s, qq = (s / 2) * (s / 2);
      for (int j = 0; j < P.nAtoms; ++j) {
        double f0 = P.ffC[j];
        for (int i = 0; i < 5; ++i) f0 += P.ffA[5 * j + i] * exp(-P.ffB[5 * j + i] * qq);
        const double wj = P.atomOcc[j] * f0 * exp(-v[PBISO] * s2 / 4) * P.atomW[j];
        const double *pos = P.atomPos + 3 * j;
        A_t c = 0, sn = 0;
        for (int r = lane; r < P.nReps; r += 32) {
          const int *R = P.repRot + 9 * r;
          const double *t = P.repTrans + 3 * r;
          const double H0 = hh * R[0] + kk * R[3] + ll * R[6], H1 = hh * R[1] + kk * R[4] + ll * R[7],
                       H2 = hh * R[2] + kk * R[5] + ll * R[8];
          double turn = H0 * pos[0] + H1 * pos[1] + H2 * pos[2] + hh * t[0] + kk * t[1] + ll * t[2];
          turn -= floor(turn);
          A_t sv, cv;
          if constexpr (F64)
            sincospi(2.0 * turn, &sv, &cv);
          else
            sincospif((float)(2.0 * turn), &sv, &cv);
          c += cv;
          sn += sv;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          c += __shfl_xor_sync(0xffffffffu, c, o);
          sn += __shfl_xor_sync(0xffffffffu, sn, o);
        }
        A += (A_t)wj * c;
        B += (A_t)wj * sn;
      }
    }
    const double po = (P.hasPo && live) ? po_factor(P, sh.f, v[PBKG0 + P.nBkg], k, lane) : 1.0;
    if (lane == 0) {
      h1[k] = (H)(((double)A * A + (double)B * B) * po);   // F^2 (x March-Dollase), parked until the heights
      if (f2write) f2write[k] = (float)h1[k];
    }
  }
  __syncwarp();
  // Peaks: lane pairs over this warp's reflections, the even lane preparing
  // K-alpha-1 and the odd lane K-alpha-2 of the same reflection at once.
  const int cnt = nR > warp ? (nR - 1 - warp) / kWarps + 1 : 0;
  for (int b = 0; b < 2 * cnt; b += 32) {
    const int idx = b + lane, line = idx & 1;
    const bool mine = idx < 2 * cnt;
    const int k = warp + (idx >> 1) * kWarps;
    double area = 0.0, lp = 1.0;
    int flag = 0;
    bool live = false;
    if (mine) {
      const int hh = P.hkl[3 * k], kk = P.hkl[3 * k + 1], ll = P.hkl[3 * k + 2];
      const double q = hh * hh * sh.f[0] + kk * kk * sh.f[1] + ll * ll * sh.f[2] + hh * kk * sh.f[3] +
                       kk * ll * sh.f[4] + hh * ll * sh.f[5];
      const double sinT = P.lambda1 * sqrt(q) / 2;
      live = q > 0 && q <= P.qmax && sinT < 1;
      if (live) {
        const double bragg = 2 * asin(sinT) * kR2D;
        if (line == 0) {
          const double base =
              bragg + (P.shiftIdx >= 0 ? sample_shift(bragg, v[P.shiftIdx], v[P.shiftIdx + 1]) : 0.0) + v[PZERO];
          area = prepare(v, P.minFwhm, base, base, P.asymIdx, pk1[k]);
          lp = lp_factor(base, P.polK);
          const int lo = lower_bound(tth, P.n, base - pk1[k].maxd), hi = upper_bound(tth, P.n, base + pk1[k].maxd, lo);
          pk1[k].lo = lo;
          pk1[k].hi = hi;
          flag = (hi > lo && lo < P.n) ? 1 : 0;
        } else {
          pk2[k].lo = pk2[k].hi = 0;
          if (doublet) {
            const double sin2 = sin(bragg * kD2R / 2.0) * (P.lambda2 / P.lambda1);
            if (fabs(sin2) < 1) {
              const double b2 = 2 * asin(sin2) / kD2R;
              const double base2 =
                  b2 + (P.shiftIdx >= 0 ? sample_shift(b2, v[P.shiftIdx], v[P.shiftIdx + 1]) : 0.0) + v[PZERO];
              area = prepare(v, P.minFwhm, base2, base2, P.asymIdx, pk2[k]);
              lp = lp_factor(base2, P.polK);
              const int lo2 = lower_bound(tth, P.n, base2 - pk2[k].maxd),
                        hi2 = upper_bound(tth, P.n, base2 + pk2[k].maxd, lo2);
              pk2[k].lo = lo2;
              pk2[k].hi = hi2;
              flag = (hi2 > lo2 && lo2 < P.n) ? 2 : 0;
            }
          }
        }
      }
    }
    const double area2 = __shfl_xor_sync(0xffffffffu, area, 1), lp2 = __shfl_xor_sync(0xffffffffu, lp, 1);
    const int flag2 = __shfl_xor_sync(0xffffffffu, flag, 1);
    if (mine && line == 0) {
      act[k] = 0;
      w2[k] = 0;
      if (live) {
        const double F2 = (double)h1[k];
        const double factor = P.mult[k] * lp * 1.0 / area;
        h1[k] = (H)(v[SCALE] * (factor * F2));
        if (u1) u1[k] = factor * F2;
        if (area2 > 0) w2[k] = (H)(P.ratio * area / area2 * (lp2 / lp));
        act[k] = area > 0 ? (flag | flag2) : 0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// WPPF / Le Bail intensities (js/pt_gpu.js:259-297): every reflection's height
// is free and non-negative, solved per evaluation by NNLS against the
// observed pattern minus the background.  Column k is reflection k's unit
// height profile (K-alpha-1 plus the weighted K-alpha-2), scaled to unit
// weighted norm s_k; H = C'WC and rhs = C'W(y - bkg) in that scaling.  The
// solve follows the reference: eight rounds of {eight cycles of projected
// coordinate descent, then the KKT error; an active-set polish with a
// Cholesky factor of the passive block}, converged when the KKT error is at
// most 1e-5 of max(1, |rhs|).  Heights h_k = x_k / s_k.  Scratch: 2 m^2 + 8 m
// doubles of shared memory.  Whole-CTA; the solve itself runs on warp 0.
// ---------------------------------------------------------------------------
__host__ __device__ inline int nnls_bytes(int m) { return (2 * m * m + 8 * m) * 8; }
constexpr int kMaxFreeRefl = 64;

// Column k of the free-intensity design matrix at point i: the unit-height
// K-alpha-1 peak plus w2 times the K-alpha-2 one.  FP32 peaks (the tempering
// path) evaluate the shape exactly as the pattern does; FP64 peaks (the
// least-squares path) in FP64.
__device__ __forceinline__ float shape32(const Peak &p, double t) {
  const float d = asym_deltaf((float)(t - p.x0), p.asym) * p.inv, dg = d * d;
  const float val = p.cL * (1.0f / (1.0f + 4.0f * dg)) + p.cG * expf(-(float)kCg * dg) - p.pedestal;
  return val > 0.f ? val : 0.f;
}

template <class PK, class HT>
__device__ __forceinline__ double free_column(const PK *pk1, const PK *pk2, const HT *w2, const int *act, int k,
                                              int i, double t) {
  double c = 0;
  const int a = act[k];
  if constexpr (std::is_same<PK, Peak>::value) {
    if ((a & 1) && i >= pk1[k].lo && i < pk1[k].hi) c += (double)shape32(pk1[k], t);
    if ((a & 2) && i >= pk2[k].lo && i < pk2[k].hi) c += (double)w2[k] * (double)shape32(pk2[k], t);
    return c;
  }
  if ((a & 1) && i >= pk1[k].lo && i < pk1[k].hi) {
    const PK &p = pk1[k];
    c += voigt64(asym_delta(t - p.x0, (double)p.asym), (double)p.inv, (double)p.cL, (double)p.cG, (double)p.pedestal);
  }
  if ((a & 2) && i >= pk2[k].lo && i < pk2[k].hi) {
    const PK &p = pk2[k];
    c += (double)w2[k] *
         voigt64(asym_delta(t - p.x0, (double)p.asym), (double)p.inv, (double)p.cL, (double)p.cG, (double)p.pedestal);
  }
  return c;
}

template <class PK, class HT, class WT>
__device__ void solve_free_heights(const Params &P, const Shared &sh, const PK *pk1, const PK *pk2, HT *h1,
                                   const HT *w2, const int *act, const double *tth, const double *yobs,
                                   const WT *wobs, double *nn) {
  const int m = P.nRefl, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  double *H = nn, *Fc = H + m * m, *rhs = Fc + m * m, *sc = rhs + m, *x = sc + m, *grad = x + m, *sol = grad + m,
         *mask = sol + m, *tmp = mask + m, *pidx = tmp + m;
  const double *v = sh.v;
  const double t0 = tth[0], t1 = tth[P.n - 1], zs = t1 > t0 ? 2.0 / (t1 - t0) : 0.0;
  auto window = [&](int k, int &lo, int &hi) {
    lo = P.n;
    hi = 0;
    if (act[k] & 1) { lo = min(lo, pk1[k].lo); hi = max(hi, pk1[k].hi); }
    if (act[k] & 2) { lo = min(lo, pk2[k].lo); hi = max(hi, pk2[k].hi); }
  };
  // norms and right-hand sides: warp per reflection
  for (int k = warp; k < m; k += nw) {
    int lo, hi;
    window(k, lo, hi);
    double a = 0, r = 0;
    for (int i = lo + lane; i < hi; i += 32) {
      const double w = (double)wobs[i];
      if (!(w > 0)) continue;
      const double t = tth[i], c = free_column(pk1, pk2, w2, act, k, i, t);
      const double z = t1 > t0 ? (t - t0) * zs - 1 : 0;
      double Tm2 = 1, Tm1 = z, bk = 0;
      for (int q = 0; q < P.nBkg; ++q) {
        const double T = q == 0 ? 1 : q == 1 ? z : 2 * z * Tm1 - Tm2;
        if (q >= 2) { Tm2 = Tm1; Tm1 = T; }
        bk += v[PBKG0 + q] * T;
      }
      a += w * c * c;
      r += w * c * (yobs[i] - bk);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    if (lane == 0) {
      const double sk = sqrt(fmax(0.0, a));
      sc[k] = sk;
      rhs[k] = sk > 0 ? r / sk : 0.0;
      H[k * m + k] = sk > 0 ? 1.0 : 0.0;   // a scaled column has unit norm
    }
  }
  __syncthreads();
  // H in the scaled columns: warp per pair j <= k, over the windows' overlap
  for (int pq = warp; pq < m * m; pq += nw) {
    const int j = pq / m, k = pq % m;
    if (k <= j) continue;
    double hv = 0;
    if (sc[j] > 0 && sc[k] > 0) {
      int lj, hj, lk, hk;
      window(j, lj, hj);
      window(k, lk, hk);
      for (int i = max(lj, lk) + lane; i < min(hj, hk); i += 32) {
        const double w = (double)wobs[i];
        if (!(w > 0)) continue;
        const double t = tth[i];
        hv += w * free_column(pk1, pk2, w2, act, j, i, t) * free_column(pk1, pk2, w2, act, k, i, t);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) hv += __shfl_xor_sync(0xffffffffu, hv, o);
      hv /= sc[j] * sc[k];
    }
    if (lane == 0) {
      H[j * m + k] = hv;
      H[k * m + j] = hv;
    }
  }
  __syncthreads();
  if (warp == 0) {
    for (int j = lane; j < m; j += 32) { x[j] = 0.0; grad[j] = rhs[j]; }
    double magnitude = 1.0;
    for (int j = lane; j < m; j += 32) magnitude = fmax(magnitude, fabs(rhs[j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) magnitude = fmax(magnitude, __shfl_xor_sync(0xffffffffu, magnitude, o));
    const double tol = 1e-5 * magnitude;
    __syncwarp();
    // KKT error of x, with grad = rhs - H x refreshed (warp-collective)
    auto kkt = [&]() {
      double err = 0;
      for (int j = lane; j < m; j += 32) {
        double g = rhs[j];
        for (int k = 0; k < m; ++k) g -= H[j * m + k] * x[k];
        grad[j] = g;
        err = fmax(err, x[j] > 0 ? fabs(g) : fmax(0.0, g));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
      __syncwarp();
      return err;
    };
    bool conv = false;
    for (int round = 0; round < 8 && !conv; ++round) {
      // projected coordinate descent, eight cycles
      for (int cyc = 0; cyc < 8; ++cyc)
        for (int j = 0; j < m; ++j) {
          const double diag = H[j * m + j];
          if (!(diag > 0)) continue;
          const double old = x[j], next = fmax(0.0, old + grad[j] / diag), delta = next - old;
          __syncwarp();
          if (lane == 0) x[j] = next;
          if (delta != 0)
            for (int k = lane; k < m; k += 32) grad[k] -= H[k * m + j] * delta;
          __syncwarp();
        }
      if (kkt() <= tol) { conv = true; break; }
      // active-set polish (lane 0; the passive block is small)
      if (lane == 0) {
        for (int j = 0; j < m; ++j) mask[j] = x[j] > 0 ? 1.0 : 0.0;
        for (int it = 0; it < 8; ++it) {
          int np = 0;
          for (int j = 0; j < m; ++j) {
            sol[j] = 0.0;
            if (mask[j] > 0.5) pidx[np++] = (double)j;
          }
          for (int i = 0; i < np; ++i) {
            const int ri = (int)pidx[i];
            for (int j = 0; j <= i; ++j) {
              const int rj = (int)pidx[j];
              double a = H[ri * m + rj];
              for (int q = 0; q < j; ++q) a -= Fc[i * m + q] * Fc[j * m + q];
              if (i == j) Fc[i * m + j] = sqrt(fmax(1e-7, a));
              else Fc[i * m + j] = a / Fc[j * m + j];
            }
            double a = rhs[ri];
            for (int q = 0; q < i; ++q) a -= Fc[i * m + q] * tmp[q];
            tmp[i] = a / Fc[i * m + i];
          }
          for (int c = 0; c < np; ++c) {
            const int i = np - 1 - c;
            double a = tmp[i];
            for (int q = i + 1; q < np; ++q) a -= Fc[q * m + i] * tmp[q];
            tmp[i] = a / Fc[i * m + i];
          }
          for (int i = 0; i < np; ++i) sol[(int)pidx[i]] = tmp[i];
          double alpha = 1.0;
          int hit = -1;
          for (int j = 0; j < m; ++j)
            if (mask[j] > 0.5 && sol[j] <= 0.0) {
              const double old = x[j], den = old - sol[j];
              const double t = den > 0 ? old / fmax(1e-30, den) : 0.0;
              if (hit < 0 || t < alpha) { alpha = t; hit = j; }
            }
          if (hit >= 0) {
            for (int j = 0; j < m; ++j)
              if (mask[j] > 0.5) {
                const double next = fmax(0.0, x[j] + alpha * (sol[j] - x[j]));
                x[j] = next;
                if (next == 0.0 && sol[j] <= 0.0) mask[j] = 0.0;
              }
            x[hit] = 0.0;
            mask[hit] = 0.0;
            continue;
          }
          for (int j = 0; j < m; ++j) x[j] = mask[j] > 0.5 ? sol[j] : 0.0;
          double err = 0, violation = tol;
          int enter = -1;
          for (int j = 0; j < m; ++j) {
            double g = rhs[j];
            for (int k = 0; k < m; ++k) g -= H[j * m + k] * x[k];
            grad[j] = g;
            err = fmax(err, x[j] > 0 ? fabs(g) : fmax(0.0, g));
            if (mask[j] < 0.5 && g > violation) { violation = g; enter = j; }
          }
          if (err <= tol || enter < 0) break;
          mask[enter] = 1.0;
        }
      }
      __syncwarp();
      if (kkt() <= tol) conv = true;
    }
  }
  __syncthreads();
  for (int k = tid; k < m; k += blockDim.x) h1[k] = (HT)(sc[k] > 0 ? x[k] / sc[k] : 0.0);
  __syncthreads();
}

// split = 2: the chain's evaluation spans a two-CTA cluster.  Both CTAs do
// the reflection stage (identical inputs, identical results); the 32-point
// tiles of the pattern alternate between them (rank r takes tiles
// warp + kWarps (2 i + r)), and chi^2 = part(rank 0) + part(rank 1) in both,
// through distributed shared memory.
__device__ double evaluate(const Params &P, Shared &sh, Peak *pk1, Peak *pk2, float *h1, float *w2, int *act,
                           const double *tth, const double *yobs, const float *wobs, float *ycalc,
                           double *nn = nullptr, int split = 1, int rank = 0, const float *f2read = nullptr,
                           float *f2write = nullptr) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) sh.valid = inv_dsq_form(sh.v, sh.f) ? 1 : 0;
  __syncthreads();
  if (!sh.valid) return INFINITY;
  const double *v = sh.v;
  const int nR = P.nRefl;
  reflection_stage<false>(P, sh, pk1, pk2, h1, w2, nullptr, act, tth, f2read, f2write);
  __syncthreads();
  if (P.method == 1) solve_free_heights(P, sh, pk1, pk2, h1, w2, act, tth, yobs, wobs, nn);
  // --- pattern in warp tiles of 32 points, then chi^2 (FP64)
  double chi = 0.0;
  const double x0 = tth[0], x1 = tth[P.n - 1], zs = x1 > x0 ? 2.0 / (x1 - x0) : 0.0;
  for (int base = (warp + rank * kWarps) * 32; base < P.n; base += split * kThreads) {
    const int i = base + lane;
    const bool in = i < P.n;
    const double x = in ? tth[i] : 0.0;
    float yp = 0.f;
    const int tLo = base, tHi = min(base + 32, P.n);
    for (int k = 0; k < nR; ++k) {
      const int a = act[k];
      if (!a) continue;
      const bool o1 = (a & 1) && pk1[k].lo < tHi && pk1[k].hi > tLo;
      const bool o2 = (a & 2) && pk2[k].lo < tHi && pk2[k].hi > tLo;
      if (!o1 && !o2) continue;
      float col = 0.f;
      if (o1 && in && i >= pk1[k].lo && i < pk1[k].hi) {
        const Peak &p = pk1[k];
        const float d = asym_deltaf((float)(x - p.x0), p.asym) * p.inv, dg = d * d;
        const float val = p.cL * (1.0f / (1.0f + 4.0f * dg)) + p.cG * expf(-(float)kCg * dg) - p.pedestal;
        col += val > 0.f ? val : 0.f;
      }
      if (o2 && in && i >= pk2[k].lo && i < pk2[k].hi) {
        const Peak &p = pk2[k];
        const float d = asym_deltaf((float)(x - p.x0), p.asym) * p.inv, dg = d * d;
        const float val = p.cL * (1.0f / (1.0f + 4.0f * dg)) + p.cG * expf(-(float)kCg * dg) - p.pedestal;
        col += w2[k] * (val > 0.f ? val : 0.f);
      }
      yp = fmaf(h1[k], col, yp);
    }
    if (in) {
      const double z = x1 > x0 ? (x - x0) * zs - 1 : 0;
      double Tm2 = 1, Tm1 = z, bk = 0;
      for (int kk = 0; kk < P.nBkg; ++kk) {
        const double T = kk == 0 ? 1 : kk == 1 ? z : 2 * z * Tm1 - Tm2;
        if (kk >= 2) { Tm2 = Tm1; Tm1 = T; }
        const double b = v[PBKG0 + kk];
        if (b != 0) bk += b * T;
      }
      const double yc = bk + (double)yp;
      if (ycalc) ycalc[i] = (float)yc;
      const float w = wobs[i];
      if (w > 0.f) {
        const double r = yobs[i] - yc;
        chi += (double)w * r * r;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) chi += __shfl_xor_sync(0xffffffffu, chi, o);
  if (lane == 0) sh.warpChi[warp] = chi;
  __syncthreads();
  if (tid == 0) {
    double t = 0;
    for (int w = 0; w < kWarps; ++w) t += sh.warpChi[w];
    sh.chiPart = t;
    if (split == 1) sh.chi = isfinite(t) ? t : INFINITY;
  }
  if (split == 2) {
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    cl.sync();
    if (tid == 0) {
      const double a = *cl.map_shared_rank(&sh.chiPart, 0), b = *cl.map_shared_rank(&sh.chiPart, 1);
      const double t = a + b;
      sh.chi = isfinite(t) ? t : INFINITY;
    }
    cl.sync();   // the peer's part is read before either CTA starts the next evaluation
  }
  __syncthreads();
  return sh.chi;
}

__device__ __forceinline__ void apply(const Params &P, const double *x, double *v) {
  for (int i = 0; i < P.nFull; ++i) v[i] = P.full[i];
  for (int j = 0; j < P.nv; ++j) v[P.index[j]] = x[j];
  if (P.cubic) { v[PB] = v[PA]; v[PC] = v[PA]; }
}

__device__ __forceinline__ double reflect(double value, double low, double high) {
  if (!isfinite(value)) return NAN;
  if (low > -1e300 && high < 1e300) {
    const double span = high - low;
    if (!(span > 0)) return low;
    const double folded = fmod(fmod(value - low, 2 * span) + 2 * span, 2 * span);
    return low + (folded <= span ? folded : 2 * span - folded);
  }
  if (value < low) return low + (low - value);
  if (value > high) return high - (value - high);
  return value;
}

__device__ __forceinline__ double uniform_open(uint32_t x) { return ((double)x + 0.5) / 4294967296.0; }

// ---------------------------------------------------------------------------
// Kernels.
// ---------------------------------------------------------------------------
struct SmemLayout {
  int pk1, pk2, h1, w2, act, f2, tth, y, w, total;
};

__host__ __device__ inline SmemLayout smem_layout(int nRefl, int n, int stage) {
  SmemLayout L;
  int o = 0;
  auto take = [&](int bytes) { const int at = o; o += (bytes + 15) & ~15; return at; };
  L.pk1 = take(nRefl * (int)sizeof(Peak));
  L.pk2 = take(nRefl * (int)sizeof(Peak));
  L.h1 = take(nRefl * 4);
  L.w2 = take(nRefl * 4);
  L.act = take(nRefl * 4);
  L.f2 = take(2 * nRefl * 4);   // two banks of |F|^2 for the sweep's moves that keep the cell, Biso and r
  L.tth = stage ? take(n * 8) : 0;
  L.y = stage ? take(n * 8) : 0;
  L.w = stage ? take(n * 4) : 0;
  L.total = o;
  return L;
}

// Cost of one parameter vector per CTA (create().costs / pattern).
__global__ void __launch_bounds__(kThreads) pt_cost_kernel(const Params P, const double *vectors, double *costs,
                                                           float *ycalc) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Shared sh;
  const SmemLayout L = smem_layout(P.nRefl, P.n, 0);
  const int c = blockIdx.x;
  if (threadIdx.x == 0) apply(P, vectors + (size_t)c * P.nv, sh.v);
  __syncthreads();
  double *nn = P.method == 1 ? reinterpret_cast<double *>(smem + L.total) : nullptr;
  const double chi = evaluate(P, sh, reinterpret_cast<Peak *>(smem + L.pk1), reinterpret_cast<Peak *>(smem + L.pk2),
                              reinterpret_cast<float *>(smem + L.h1), reinterpret_cast<float *>(smem + L.w2),
                              reinterpret_cast<int *>(smem + L.act), P.tth, P.y, P.w,
                              ycalc ? ycalc + (size_t)c * P.n : nullptr, nn);
  if (threadIdx.x == 0) costs[c] = chi;
}

// One sweep: the exchange of the previous sweep (if any), then `moves`
// proposals with Metropolis.  in/out are the double-buffered chain states.
// split = 2: a chain per two-CTA cluster (launched with cluster dimension
// 2); both CTAs run the chain's logic identically and rank 0 writes it back.
__global__ void __launch_bounds__(kThreads) pt_sweep_kernel(const Params P, const Chain *in, Chain *out, int moves,
                                                            int exchangeParity, int bootstrap, int split) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Shared sh;
  __shared__ double xs[kMaxNv];
  __shared__ Chain st;
  __shared__ int drawnJ;
  // |F|^2 reuse: bank f2cur holds the current state's |F|^2 when f2valid; a move that changes
  // no parameter |F|^2 depends on (cell, Biso, March-Dollase r) reads it, any other writes the other bank
  __shared__ int f2cur, f2valid, f2mode, f2bank, f2isF;
  const SmemLayout L = smem_layout(P.nRefl, P.n, P.stageObs);
  Peak *pk1 = reinterpret_cast<Peak *>(smem + L.pk1), *pk2 = reinterpret_cast<Peak *>(smem + L.pk2);
  float *h1 = reinterpret_cast<float *>(smem + L.h1), *w2 = reinterpret_cast<float *>(smem + L.w2);
  int *act = reinterpret_cast<int *>(smem + L.act);
  float *f2 = reinterpret_cast<float *>(smem + L.f2);
  const bool reuseF2 = P.method == 0;
  if (threadIdx.x == 0) {
    f2cur = 0;
    f2valid = 0;
  }
  const double *tth = P.tth, *yobs = P.y;
  const float *wobs = P.w;
  if (P.stageObs) {
    double *t = reinterpret_cast<double *>(smem + L.tth), *y = reinterpret_cast<double *>(smem + L.y);
    float *w = reinterpret_cast<float *>(smem + L.w);
    for (int i = threadIdx.x; i < P.n; i += kThreads) { t[i] = P.tth[i]; y[i] = P.y[i]; w[i] = P.w[i]; }
    tth = t; yobs = y; wobs = w;
  }
  const int c = blockIdx.x / split, C = P.chains;
  const int rank = split == 2 ? (int)cooperative_groups::this_cluster().block_rank() : 0;
  const double T = pow(P.maxTemp, (double)c / (double)(C - 1));
  if (threadIdx.x == 0) {
    st = in[c];
    if (P.trace && rank == 0 && !bootstrap)
      for (int k = 0; k < kTraceHead; ++k) P.trace[(size_t)c * (kTraceHead + kTraceMove * P.nv) + k] = 0.0;
    // adjacent exchange of the previous sweep, even/odd pairs alternating
    if (exchangeParity >= 0) {
      const int left = ((c - exchangeParity) % 2 == 0) ? c : c - 1;
      const int right = left + 1;
      if (left >= exchangeParity && right < C) {
        const Chain &a = in[left], &b = in[right];
        const double Ta = pow(P.maxTemp, (double)left / (C - 1)), Tb = pow(P.maxTemp, (double)right / (C - 1));
        const double la = 0.5 * (1 / Ta - 1 / Tb) * (a.cost - b.cost);
        const uint4 r = philox4x32_10(make_uint4((uint32_t)a.sweep, (uint32_t)left, 0x45584348u, 3u),
                                      make_uint2(P.seed, 0x9E3779B9u));
        const double lu = log(uniform_open(r.x));
        const bool swap = la >= 0 || lu < la;
        if (P.trace && rank == 0 && !bootstrap) {
          double *tr = P.trace + (size_t)c * (kTraceHead + kTraceMove * P.nv);
          tr[0] = 1.0;
          tr[1] = swap ? 1.0 : 0.0;
          tr[2] = la;
          tr[3] = lu;
        }
        if (c == left) st.swapAttempts += 1;
        if (swap) {
          const Chain &o = (c == left) ? b : a;
          for (int j = 0; j < P.nv; ++j) st.x[j] = o.x[j];
          st.cost = o.cost;
          st.feasible = o.feasible;
          if (c == left) st.swaps += 1;
        }
      }
    }
  }
  __syncthreads();
  for (int m = 0; m < moves; ++m) {
    if (threadIdx.x == 0) {
      for (int j = 0; j < P.nv; ++j) xs[j] = st.x[j];
      if (!bootstrap) {
        const uint4 r = philox4x32_10(make_uint4((uint32_t)st.sweep, (uint32_t)c, (uint32_t)m, 1u),
                                      make_uint2(P.seed, 0x2545F491u));
        const int j = min(P.nv - 1, (int)(uniform_open(r.x) * P.nv));
        drawnJ = j;
        const double z = sqrt(-2.0 * log(uniform_open(r.y))) * cos(2.0 * kPi * uniform_open(r.z));
        xs[j] = reflect(st.x[j] + z * P.scales[j] * sqrt(T), P.lo[j], P.hi[j]);
        st.logu = log(uniform_open(r.w));
      }
      apply(P, xs, sh.v);
      const int fi = bootstrap ? -1 : P.index[drawnJ];
      f2isF = bootstrap || (fi >= PA && fi <= PGA) || fi == PBISO || (P.hasPo && fi == PBKG0 + P.nBkg);
      f2mode = !reuseF2 ? 0 : (f2valid && !f2isF ? 1 : 2);       // 0 compute only, 1 read, 2 compute and keep
      f2bank = f2mode == 1 ? f2cur : (f2valid || f2isF ? f2cur ^ 1 : f2cur);
    }
    __syncthreads();
    const int nR = P.nRefl;
    const double cost = evaluate(P, sh, pk1, pk2, h1, w2, act, tth, yobs, wobs, nullptr,
                                 P.method == 1 ? reinterpret_cast<double *>(smem + L.total) : nullptr, split, rank,
                                 f2mode == 1 ? f2 + f2bank * nR : nullptr, f2mode == 2 ? f2 + f2bank * nR : nullptr);
    if (threadIdx.x == 0) {
      st.proposalCost = cost;
      if (bootstrap) {
        if (f2mode == 2 && sh.valid) {
          f2cur = f2bank;
          f2valid = 1;
        }
        st.cost = cost;
        st.bestCost = cost;
        for (int j = 0; j < P.nv; ++j) st.best[j] = st.x[j];
      } else {
        st.proposals += 1;
        const double before = st.cost;
        const bool acc = isfinite(cost) && (cost <= st.cost || st.logu < (st.cost - cost) / (2 * T));
        if (f2mode == 2 && sh.valid && (!f2isF || acc)) {   // the bank now holds the current state's |F|^2
          f2cur = f2bank;
          f2valid = 1;
        }
        if (P.trace && rank == 0 && m < P.nv) {
          double *tr = P.trace + (size_t)c * (kTraceHead + kTraceMove * P.nv) + kTraceHead + kTraceMove * m;
          const int jm = drawnJ;
          tr[0] = (double)jm;
          tr[1] = xs[jm];
          tr[2] = st.logu;
          tr[3] = before;
          tr[4] = cost;
          tr[5] = acc ? 1.0 : 0.0;
        }
        if (acc) {
          for (int j = 0; j < P.nv; ++j) st.x[j] = xs[j];
          st.cost = cost;
          st.accepted += 1;
          if (cost < st.bestCost) {
            st.bestCost = cost;
            for (int j = 0; j < P.nv; ++j) st.best[j] = xs[j];
          }
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && rank == 0) {
    if (!bootstrap && moves > 0) st.sweep += 1;
    out[c] = st;
  }
}


// ---------------------------------------------------------------------------
// Least-squares finish (FP64): patterns for the finite-difference Jacobian,
// the normal equations J'WJ, J'W r, chi^2, and the damped Cholesky solve
// (js/rietveld_core.js:1953-2140, :1304-1335).
// ---------------------------------------------------------------------------
struct Smem64 {
  int pk1, pk2, h1, w2, u1, act, total;
};
__host__ __device__ inline Smem64 smem64_layout(int nRefl) {
  Smem64 L;
  int o = 0;
  auto take = [&](int bytes) { const int at = o; o += (bytes + 15) & ~15; return at; };
  L.pk1 = take(nRefl * (int)sizeof(PeakD));
  L.pk2 = take(nRefl * (int)sizeof(PeakD));
  L.h1 = take(nRefl * 8);
  L.w2 = take(nRefl * 8);
  L.u1 = take(nRefl * 8);
  L.act = take(nRefl * 4);
  L.total = o;
  return L;
}

// FP64 pattern of refined vector c (one CTA each): y = background + peaks,
// yu (when given; vector 0 only) = the peaks at unit scale (the scale
// column), chiOut[c] = chi^2.
__global__ void __launch_bounds__(kThreads) pt_pattern64_kernel(const Params P, const double *vectors, double *y,
                                                                double *yu, double *chiOut) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Shared sh;
  const Smem64 L = smem64_layout(P.nRefl);
  PeakD *pk1 = reinterpret_cast<PeakD *>(smem + L.pk1), *pk2 = reinterpret_cast<PeakD *>(smem + L.pk2);
  double *h1 = reinterpret_cast<double *>(smem + L.h1), *w2 = reinterpret_cast<double *>(smem + L.w2);
  double *u1 = reinterpret_cast<double *>(smem + L.u1);
  int *act = reinterpret_cast<int *>(smem + L.act);
  const int c = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double *yc = y + (size_t)c * P.n, *yq = yu ? yu + (size_t)c * P.n : nullptr;
  if (tid == 0) {
    apply(P, vectors + (size_t)c * P.nv, sh.v);
    sh.valid = inv_dsq_form(sh.v, sh.f) ? 1 : 0;
  }
  __syncthreads();
  if (!sh.valid) {
    for (int i = tid; i < P.n; i += kThreads) {
      yc[i] = NAN;
      if (yq) yq[i] = NAN;
    }
    if (tid == 0) chiOut[c] = INFINITY;
    return;
  }
  reflection_stage<true>(P, sh, pk1, pk2, h1, w2, u1, act, P.tth);
  __syncthreads();
  if (P.method == 1) {
    // free heights; no scale column (u1 = 0)
    solve_free_heights(P, sh, pk1, pk2, h1, w2, act, P.tth, P.y, P.wd, reinterpret_cast<double *>(smem + L.total));
    for (int k = tid; k < P.nRefl; k += kThreads) u1[k] = 0.0;
    __syncthreads();
  }
  const double *v = sh.v;
  const int nR = P.nRefl;
  const double x0 = P.tth[0], x1 = P.tth[P.n - 1], zs = x1 > x0 ? 2.0 / (x1 - x0) : 0.0;
  double chi = 0.0;
  for (int base = warp * 32; base < P.n; base += kThreads) {
    const int i = base + lane;
    const bool in = i < P.n;
    const double x = in ? P.tth[i] : 0.0;
    double yp = 0.0, yu1 = 0.0;
    const int tLo = base, tHi = min(base + 32, P.n);
    for (int k = 0; k < nR; ++k) {
      const int a = act[k];
      if (!a) continue;
      const bool o1 = (a & 1) && pk1[k].lo < tHi && pk1[k].hi > tLo;
      const bool o2 = (a & 2) && pk2[k].lo < tHi && pk2[k].hi > tLo;
      if (!o1 && !o2) continue;
      double col = 0.0;
      if (o1 && in && i >= pk1[k].lo && i < pk1[k].hi) {
        const PeakD &p = pk1[k];
        col += voigt64(asym_delta(x - p.x0, p.asym), p.inv, p.cL, p.cG, p.pedestal);
      }
      if (o2 && in && i >= pk2[k].lo && i < pk2[k].hi) {
        const PeakD &p = pk2[k];
        col += w2[k] * voigt64(asym_delta(x - p.x0, p.asym), p.inv, p.cL, p.cG, p.pedestal);
      }
      yp += h1[k] * col;
      yu1 += u1[k] * col;
    }
    if (in) {
      const double z = x1 > x0 ? (x - x0) * zs - 1 : 0;
      double Tm2 = 1, Tm1 = z, bk = 0;
      for (int kk = 0; kk < P.nBkg; ++kk) {
        const double T = kk == 0 ? 1 : kk == 1 ? z : 2 * z * Tm1 - Tm2;
        if (kk >= 2) { Tm2 = Tm1; Tm1 = T; }
        const double b = v[PBKG0 + kk];
        if (b != 0) bk += b * T;
      }
      const double ycal = bk + yp;
      yc[i] = ycal;
      if (yq) yq[i] = yu1;
      const double w = P.wd[i];
      if (w > 0) {
        const double r = P.y[i] - ycal;
        chi += w * r * r;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) chi += __shfl_xor_sync(0xffffffffu, chi, o);
  if (lane == 0) sh.warpChi[warp] = chi;
  __syncthreads();
  if (tid == 0) {
    double t = 0;
    for (int w = 0; w < kWarps; ++w) t += sh.warpChi[w];
    chiOut[c] = isfinite(t) ? t : INFINITY;
  }
}

// Jacobian column descriptors: 0 scale (unit-scale peaks of vector 0),
// 1 Chebyshev T_k, 2 finite difference (y[plus] - y[minus]) / step, 3 zero.
struct LmCols {
  int kind[kMaxNv];
  int plus[kMaxNv], minus[kMaxNv], bkg[kMaxNv];
  double step[kMaxNv];
};

__device__ __forceinline__ double cheb_t(int k, double z) {
  double Tm2 = 1, Tm1 = z, T = 1;
  for (int q = 0; q <= k; ++q) {
    T = q == 0 ? 1 : q == 1 ? z : 2 * z * Tm1 - Tm2;
    if (q >= 2) { Tm2 = Tm1; Tm1 = T; }
  }
  return T;
}

__device__ __forceinline__ double jcol(const Params &P, const LmCols &L, int j, int i, const double *y,
                                       const double *yu, double z) {
  switch (L.kind[j]) {
    case 0: return yu[i];
    case 1: return cheb_t(L.bkg[j], z);
    case 2: return (y[(size_t)L.plus[j] * P.n + i] - y[(size_t)L.minus[j] * P.n + i]) / L.step[j];
    default: return 0.0;
  }
}

// Normal equations: block b < nv(nv+1)/2 -> A[a][b'] (a >= b'), then nv blocks
// of g, then one block of f.  Strided FP64 sums, reduced in a fixed order.
__global__ void __launch_bounds__(kThreads) pt_normal_kernel(const Params P, const LmCols L, const double *y,
                                                             const double *yu, double *out) {
  __shared__ double part[kWarps];
  const int nv = P.nv, nPairs = nv * (nv + 1) / 2, b = blockIdx.x, tid = threadIdx.x;
  int ja = -1, jb = -1, mode;
  if (b < nPairs) {
    mode = 0;
    int a = 0, rem = b;
    while (rem > a) { rem -= a + 1; ++a; }
    ja = a; jb = rem;
  } else if (b < nPairs + nv) {
    mode = 1;
    ja = b - nPairs;
  } else {
    mode = 2;
  }
  const double x0 = P.tth[0], x1 = P.tth[P.n - 1], zs = x1 > x0 ? 2.0 / (x1 - x0) : 0.0;
  double acc = 0.0;
  for (int i = tid; i < P.n; i += kThreads) {
    const double w = P.wd[i];
    const double z = x1 > x0 ? (P.tth[i] - x0) * zs - 1 : 0;
    const double r = w > 0 ? P.y[i] - y[i] : 0.0;
    if (mode == 0)
      acc += w * jcol(P, L, ja, i, y, yu, z) * jcol(P, L, jb, i, y, yu, z);
    else if (mode == 1)
      acc += w * jcol(P, L, ja, i, y, yu, z) * r;
    else if (w > 0)
      acc += w * r * r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) part[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double t = 0;
    for (int w = 0; w < kWarps; ++w) t += part[w];
    if (mode == 0) {
      out[ja * nv + jb] = t;
      out[jb * nv + ja] = t;
    } else if (mode == 1) {
      out[nv * nv + ja] = t;
    } else {
      out[nv * nv + nv] = t;
    }
  }
}

// solveSPD on the free set F (nF indices into A, g).  mode 0: the scaled,
// damped LM system (D A_FF D + mu I) d = D g_F, result D d; mode 1: A_FF d = g_F.
// One thread; FP64 Cholesky with the growing ridge.  out[nF] = 1 on success.
__global__ void pt_lm_solve_kernel(const double *A, const double *g, int nv, const int *F, int nF, double mu, int mode,
                                   double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double M[kMaxNv * kMaxNv], Lc[kMaxNv * kMaxNv], rhs[kMaxNv], sc[kMaxNv], x[kMaxNv];
  for (int a = 0; a < nF; ++a) sc[a] = mode == 0 ? 1.0 / sqrt(A[F[a] * nv + F[a]]) : 1.0;
  for (int a = 0; a < nF; ++a) {
    rhs[a] = g[F[a]] * sc[a];
    for (int b = 0; b < nF; ++b) M[a * nF + b] = A[F[a] * nv + F[b]] * sc[a] * sc[b];
    if (mode == 0) M[a * nF + a] += mu;
  }
  auto chol = [&](double ridge) -> bool {
    for (int i = 0; i < nF; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = M[i * nF + j] + (i == j ? ridge : 0.0);
        for (int k = 0; k < j; ++k) s -= Lc[i * nF + k] * Lc[j * nF + k];
        if (i == j) {
          if (!(s > 0) || !isfinite(s)) return false;
          Lc[i * nF + i] = sqrt(s);
        } else {
          Lc[i * nF + j] = s / Lc[j * nF + j];
        }
      }
    return true;
  };
  bool ok = chol(0.0);
  if (!ok) {
    double tr = 0;
    for (int i = 0; i < nF; ++i) tr += fabs(M[i * nF + i]);
    double ridge = (tr / (nF > 1 ? nF : 1)) * 1e-12;
    if (!(ridge > 0 || ridge < 0)) ridge = 1e-300;
    for (int a = 0; a < 10 && !ok; ++a, ridge *= 100) ok = chol(ridge);
  }
  if (ok) {
    for (int i = 0; i < nF; ++i) {
      double s = rhs[i];
      for (int k = 0; k < i; ++k) s -= Lc[i * nF + k] * x[k];
      x[i] = s / Lc[i * nF + i];
    }
    for (int i = nF - 1; i >= 0; --i) {
      double s = x[i];
      for (int k = i + 1; k < nF; ++k) s -= Lc[k * nF + i] * x[k];
      x[i] = s / Lc[i * nF + i];
    }
    for (int a = 0; a < nF; ++a) out[a] = x[a] * sc[a];
  }
  out[nF] = ok ? 1.0 : 0.0;
}

}  // namespace pt
}  // namespace p6

// ===========================================================================
// Host side.
// ===========================================================================
using namespace p6;
using namespace p6::pt;

struct p6_pt_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Params P{};
  int smemSweep = 0, smemCost = 0;
  int split = 1;            // CTAs per chain in the sweep (2: a two-CTA cluster)
  Chain *dChain[2] = {nullptr, nullptr};
  int curBuf = 0;
  int pendingParity = -1;   // exchange owed by the last sweep, applied at the start of the next
  long long sweepsDone = 0;
  void *dAlloc[32] = {};
  int nAlloc = 0;
  double *dVec = nullptr, *dCost = nullptr;
  float *dY = nullptr;
  int vecCap = 0;
  long long launches = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  int graphCount = 0;
  // least-squares finish: host copies of the parameter description and FP64 scratch
  std::vector<double> fullHost, loHost, hiHost;
  std::vector<int> indexHost;
  double tthFirst = 0, tthLast = 0;
  int smem64 = 0;
  double *dLmVec = nullptr, *dLmY = nullptr, *dLmYu = nullptr, *dLmChi = nullptr, *dLmOut = nullptr;
  int *dLmF = nullptr;
  int lmCap = 0;
  double *dTrace = nullptr;   // per chain, the last sweep's decisions (p6_pt_set_trace)
};

template <typename T>
static p6_status pt_upload(p6_pt_session *s, const T *src, size_t n, const T **dst) {
  T *d = nullptr;
  P6_CUDA(cudaMalloc((void **)&d, std::max<size_t>(n, 1) * sizeof(T)));
  if (n && src) P6_CUDA(cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, s->stream));
  s->dAlloc[s->nAlloc++] = d;
  *dst = d;
  return P6_OK;
}

static void pt_free(p6_pt_session *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->graphExec) cudaGraphExecDestroy(s->graphExec);
  if (s->graph) cudaGraphDestroy(s->graph);
  for (int i = 0; i < s->nAlloc; ++i) cudaFree(s->dAlloc[i]);
  for (void *p : {(void *)s->dChain[0], (void *)s->dChain[1], (void *)s->dVec, (void *)s->dCost, (void *)s->dY,
                  (void *)s->dLmVec, (void *)s->dLmY, (void *)s->dLmYu, (void *)s->dLmChi, (void *)s->dLmOut,
                  (void *)s->dLmF, (void *)s->dTrace})
    if (p) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static p6_status pt_ensure_vectors(p6_pt_session *s, int n) {
  if (n <= s->vecCap) return P6_OK;
  if (s->dVec) cudaFree(s->dVec);
  if (s->dCost) cudaFree(s->dCost);
  if (s->dY) cudaFree(s->dY);
  s->dVec = nullptr; s->dCost = nullptr; s->dY = nullptr;
  P6_CUDA(cudaMalloc(&s->dVec, (size_t)n * s->P.nv * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dCost, (size_t)n * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dY, (size_t)n * s->P.n * sizeof(float)));
  s->vecCap = n;
  return P6_OK;
}

extern "C" {

static int pt_cluster_capacity(int smemBytes);

p6_status p6_pt_create(const p6_pt_problem *pr, int device, p6_pt_session **out) {
  clear_error();
  if (!pr || !out) return set_error(P6_ERR_INVALID_ARG, "null problem or output pointer");
  *out = nullptr;
  if (pr->n_refl <= 0 || pr->n_reps <= 0 || (pr->n_atoms <= 0 && pr->method == 0) || pr->n_atoms < 0 ||
      pr->n_points < 2)
    return set_error(P6_ERR_INVALID_ARG, "empty problem");
  if (pr->method != 0 && pr->method != 1) return set_error(P6_ERR_INVALID_ARG, "method must be 0 (Rietveld) or 1 (WPPF / Le Bail)");
  if (pr->method == 1 && pr->n_refl > kMaxFreeRefl)
    return set_error(P6_ERR_CAPACITY, "free-intensity fits hold at most 64 envelope reflections on the device");
  if (pr->nv < 1 || pr->nv > kMaxNv) return set_error(P6_ERR_CAPACITY, "1 to 32 refined parameters");
  if (pr->n_full < PBKG0 + pr->n_bkg || pr->n_full > kMaxFull)
    return set_error(P6_ERR_INVALID_ARG, "full parameter vector too short or too long");
  if (pr->chains < 2 || pr->chains > 65535) return set_error(P6_ERR_INVALID_ARG, "at least 2 chains");
  if (!(pr->max_temp > 1)) return set_error(P6_ERR_INVALID_ARG, "max_temp must exceed 1");
  if (!pr->hkl || !pr->mult || !pr->rep_rot || !pr->rep_trans || !pr->tth || !pr->y || !pr->w || !pr->full_values ||
      !pr->index || !pr->lo || !pr->hi || !pr->scales ||
      (pr->n_atoms > 0 && (!pr->atom_pos || !pr->atom_wmult || !pr->atom_occ || !pr->ff_a || !pr->ff_b || !pr->ff_c)))
    return set_error(P6_ERR_INVALID_ARG, "null table pointer");
  for (int j = 0; j < pr->nv; ++j)
    if (pr->index[j] < 0 || pr->index[j] >= pr->n_full) return set_error(P6_ERR_INVALID_ARG, "parameter index out of range");
  for (int i = 1; i < pr->n_points; ++i)
    if (!(pr->tth[i] > pr->tth[i - 1])) return set_error(P6_ERR_INVALID_ARG, "the 2-theta axis must be ascending");
  if (pr->has_asym && pr->n_full < PBKG0 + pr->n_bkg + (pr->has_po ? 1 : 0) + 2)
    return set_error(P6_ERR_INVALID_ARG, "asymmetry: the full vector has no SL, HL entries");
  if (pr->has_shift && pr->n_full < PBKG0 + pr->n_bkg + (pr->has_po ? 1 : 0) + (pr->has_asym ? 2 : 0) + 2)
    return set_error(P6_ERR_INVALID_ARG, "sample shift: the full vector has no displacement, transparency entries");
  if (pr->has_po) {
    if (!pr->eq_start || !pr->eq_hkl) return set_error(P6_ERR_INVALID_ARG, "preferred orientation without equivalents");
    if (pr->n_full < PBKG0 + pr->n_bkg + 1)
      return set_error(P6_ERR_INVALID_ARG, "preferred orientation: the full vector has no entry after the background");
    if (pr->eq_start[0] != 0) return set_error(P6_ERR_INVALID_ARG, "eq_start[0] must be 0");
    for (int k = 0; k < pr->n_refl; ++k)
      if (pr->eq_start[k + 1] < pr->eq_start[k] || pr->eq_start[k + 1] - pr->eq_start[k] > 192)
        return set_error(P6_ERR_INVALID_ARG, "eq_start must be ascending with at most 192 equivalents per reflection");
  }
  p6_pt_session *s = new p6_pt_session();
  s->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { pt_free(s); return cuda_error(e, "cudaSetDevice"); }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { pt_free(s); return cuda_error(e, "cudaStreamCreate"); }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  Params &P = s->P;
  P.nRefl = pr->n_refl; P.nReps = pr->n_reps; P.nAtoms = pr->n_atoms; P.n = pr->n_points; P.nBkg = pr->n_bkg;
  P.nFull = pr->n_full; P.nv = pr->nv; P.chains = pr->chains; P.cubic = pr->cubic;
  P.lambda1 = pr->lambda1; P.lambda2 = pr->lambda2; P.ratio = pr->ratio; P.polK = pr->pol_k;
  P.minFwhm = pr->min_fwhm > 0 ? pr->min_fwhm : 1e-3;
  P.qmax = 1.0 / (pr->dmin * pr->dmin) * (1 + 1e-9);
  P.maxTemp = pr->max_temp;
  P.seed = pr->seed;
  std::vector<float> wf(pr->n_points);
  for (int i = 0; i < pr->n_points; ++i) wf[i] = (float)pr->w[i];
  p6_status st;
#define PT_TRY(x) do { st = (x); if (st != P6_OK) { pt_free(s); return st; } } while (0)
  PT_TRY(pt_upload(s, pr->hkl, (size_t)3 * pr->n_refl, &P.hkl));
  PT_TRY(pt_upload(s, pr->mult, (size_t)pr->n_refl, &P.mult));
  PT_TRY(pt_upload(s, pr->rep_rot, (size_t)9 * pr->n_reps, &P.repRot));
  PT_TRY(pt_upload(s, pr->rep_trans, (size_t)3 * pr->n_reps, &P.repTrans));
  PT_TRY(pt_upload(s, pr->atom_pos, (size_t)3 * pr->n_atoms, &P.atomPos));
  PT_TRY(pt_upload(s, pr->atom_wmult, (size_t)pr->n_atoms, &P.atomW));
  PT_TRY(pt_upload(s, pr->atom_occ, (size_t)pr->n_atoms, &P.atomOcc));
  PT_TRY(pt_upload(s, pr->ff_a, (size_t)5 * pr->n_atoms, &P.ffA));
  PT_TRY(pt_upload(s, pr->ff_b, (size_t)5 * pr->n_atoms, &P.ffB));
  PT_TRY(pt_upload(s, pr->ff_c, (size_t)pr->n_atoms, &P.ffC));
  PT_TRY(pt_upload(s, pr->tth, (size_t)pr->n_points, &P.tth));
  PT_TRY(pt_upload(s, pr->y, (size_t)pr->n_points, &P.y));
  PT_TRY(pt_upload(s, (const float *)wf.data(), (size_t)pr->n_points, &P.w));
  PT_TRY(pt_upload(s, pr->w, (size_t)pr->n_points, &P.wd));
  PT_TRY(pt_upload(s, pr->full_values, (size_t)pr->n_full, &P.full));
  PT_TRY(pt_upload(s, pr->index, (size_t)pr->nv, &P.index));
  PT_TRY(pt_upload(s, pr->lo, (size_t)pr->nv, &P.lo));
  PT_TRY(pt_upload(s, pr->hi, (size_t)pr->nv, &P.hi));
  PT_TRY(pt_upload(s, pr->scales, (size_t)pr->nv, &P.scales));
  P.hasPo = pr->has_po ? 1 : 0;
  P.asymIdx = pr->has_asym ? PBKG0 + pr->n_bkg + P.hasPo : -1;
  P.shiftIdx = pr->has_shift ? PBKG0 + pr->n_bkg + P.hasPo + (pr->has_asym ? 2 : 0) : -1;
  if (P.hasPo) {
    PT_TRY(pt_upload(s, pr->eq_start, (size_t)pr->n_refl + 1, &P.eqStart));
    PT_TRY(pt_upload(s, pr->eq_hkl, (size_t)3 * pr->eq_start[pr->n_refl], &P.eqHkl));
    for (int i = 0; i < 3; ++i) P.poDir[i] = pr->po_dir[i];
  }
  int smemOptin = 0;
  cudaDeviceGetAttribute(&smemOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  const int staticBytes = 4096;
  P.method = pr->method;
  const int nnB = P.method == 1 ? nnls_bytes(P.nRefl) : 0;   // free-intensity scratch after each layout
  P.stageObs = smem_layout(P.nRefl, P.n, 1).total + nnB + staticBytes <= smemOptin ? 1 : 0;
  s->smemSweep = smem_layout(P.nRefl, P.n, P.stageObs).total + nnB;
  s->smemCost = smem_layout(P.nRefl, P.n, 0).total + nnB;
  if (s->smemCost + staticBytes > smemOptin) {
    pt_free(s);
    return set_error(P6_ERR_CAPACITY, "too many reflections for the shared-memory peak table");
  }
  // the FP64 peak table of the least-squares finish; 0 when it does not fit (the finish then reports CAPACITY)
  s->smem64 = smem64_layout(P.nRefl).total + nnB + staticBytes <= smemOptin ? smem64_layout(P.nRefl).total + nnB : 0;
  s->fullHost.assign(pr->full_values, pr->full_values + pr->n_full);
  s->indexHost.assign(pr->index, pr->index + pr->nv);
  s->loHost.assign(pr->lo, pr->lo + pr->nv);
  s->hiHost.assign(pr->hi, pr->hi + pr->nv);
  s->tthFirst = pr->tth[0];
  s->tthLast = pr->tth[pr->n_points - 1];
  e = cudaFuncSetAttribute(pt_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemSweep);
  if (e == cudaSuccess && s->smem64 > 0)
    e = cudaFuncSetAttribute(pt_pattern64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smem64);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(pt_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemCost);
  if (e != cudaSuccess) { pt_free(s); return cuda_error(e, "cudaFuncSetAttribute"); }
  // chains that leave half the SMs idle span two-CTA clusters when the
  // device can schedule every chain's cluster at once
  {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (2 * pr->chains <= sms && pt_cluster_capacity(s->smemSweep) >= pr->chains) s->split = 2;
  }
  for (int b = 0; b < 2; ++b) {
    e = cudaMalloc(&s->dChain[b], (size_t)pr->chains * sizeof(Chain));
    if (e != cudaSuccess) { pt_free(s); return cuda_error(e, "cudaMalloc chains"); }
    cudaMemsetAsync(s->dChain[b], 0, (size_t)pr->chains * sizeof(Chain), s->stream);
  }
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) { pt_free(s); return cuda_error(e, "upload"); }
#undef PT_TRY
  *out = s;
  return P6_OK;
}

p6_status p6_pt_destroy(p6_pt_session *s) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  pt_free(s);
  return P6_OK;
}

p6_status p6_pt_costs(p6_pt_session *s, const double *vectors, int n_vectors, double *costs, float *ycalc) {
  clear_error();
  if (!s || !vectors || !costs || n_vectors <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  p6_status st = pt_ensure_vectors(s, n_vectors);
  if (st != P6_OK) return st;
  P6_CUDA(cudaMemcpyAsync(s->dVec, vectors, (size_t)n_vectors * s->P.nv * sizeof(double), cudaMemcpyHostToDevice,
                          s->stream));
  pt_cost_kernel<<<n_vectors, kThreads, s->smemCost, s->stream>>>(s->P, s->dVec, s->dCost, ycalc ? s->dY : nullptr);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  P6_CUDA(cudaMemcpyAsync(costs, s->dCost, (size_t)n_vectors * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (ycalc)
    P6_CUDA(cudaMemcpyAsync(ycalc, s->dY, (size_t)n_vectors * s->P.n * sizeof(float), cudaMemcpyDeviceToHost,
                            s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_pt_initial(p6_pt_session *s, const double *vectors, int n_vectors) {
  clear_error();
  if (!s || !vectors || n_vectors <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  std::vector<Chain> h(s->P.chains);
  for (int c = 0; c < s->P.chains; ++c) {
    Chain &ch = h[c];
    std::memset(&ch, 0, sizeof(Chain));
    const double *v = vectors + (size_t)(c % n_vectors) * s->P.nv;
    for (int j = 0; j < s->P.nv; ++j) ch.x[j] = ch.best[j] = v[j];
    ch.cost = ch.bestCost = 3e38;
    ch.valid = 1;
  }
  P6_CUDA(cudaMemcpyAsync(s->dChain[s->curBuf], h.data(), h.size() * sizeof(Chain), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->pendingParity = -1;
  s->sweepsDone = 0;
  return P6_OK;
}

// Two-CTA clusters of the sweep kernel the device can hold at once (0 when
// the cluster launch is not possible with this shared memory).
static int pt_cluster_capacity(int smemBytes) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smemBytes;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, pt_sweep_kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// One sweep launch: exchange owed by the previous sweep, then `moves` proposals.
static cudaError_t pt_launch_sweep(p6_pt_session *s, int moves, int parity, int bootstrap) {
  Chain *in = s->dChain[s->curBuf], *out = s->dChain[s->curBuf ^ 1];
  const int split = s->split;
  if (split == 1) {
    pt_sweep_kernel<<<s->P.chains, kThreads, s->smemSweep, s->stream>>>(s->P, in, out, moves, parity, bootstrap, 1);
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(s->P.chains * split);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = s->smemSweep;
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = split;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, pt_sweep_kernel, s->P, (const Chain *)in, out, moves, parity,
                                             bootstrap, split);
    if (e != cudaSuccess) return e;
  }
  s->curBuf ^= 1;
  s->launches++;
  return cudaGetLastError();
}

p6_status p6_pt_batch(p6_pt_session *s, int count, int bootstrap) {
  clear_error();
  if (!s || count <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaEventRecord(s->ev0, s->stream));
  if (bootstrap) {
    P6_CUDA(pt_launch_sweep(s, 1, -1, 1));
  } else {
    for (int j = 0; j < count; ++j) {
      P6_CUDA(pt_launch_sweep(s, s->P.nv, s->pendingParity, 0));
      s->pendingParity = (int)(s->sweepsDone % 2);
      s->sweepsDone++;
    }
  }
  P6_CUDA(cudaEventRecord(s->ev1, s->stream));
  return P6_OK;
}

p6_status p6_pt_read_state(p6_pt_session *s, float *state, double *x, double *best, double *costs, double *counters) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  const int C = s->P.chains, nv = s->P.nv;
  std::vector<Chain> h(C);
  // the exchange owed by the last sweep is applied (exchange only, no moves) before reading
  if (s->pendingParity >= 0) {
    P6_CUDA(pt_launch_sweep(s, 0, s->pendingParity, 0));
    s->pendingParity = -1;
  }
  P6_CUDA(cudaMemcpyAsync(h.data(), s->dChain[s->curBuf], C * sizeof(Chain), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  const int stride = 3 * nv + 12;
  for (int c = 0; c < C; ++c) {
    const Chain &ch = h[c];
    if (state) {
      float *b = state + (size_t)c * stride;
      for (int j = 0; j < nv; ++j) { b[j] = (float)ch.x[j]; b[nv + j] = (float)ch.x[j]; b[2 * nv + j] = (float)ch.best[j]; }
      const double tail[12] = {ch.cost, ch.bestCost, (double)s->sweepsDone, ch.accepted, ch.proposals, ch.swaps,
                               ch.swapAttempts, ch.valid, ch.logu, ch.unsolved, ch.proposalCost, ch.feasible};
      for (int k = 0; k < 12; ++k) b[3 * nv + k] = (float)std::min(tail[k], 3e38);
    }
    for (int j = 0; j < nv; ++j) {
      if (x) x[(size_t)c * nv + j] = ch.x[j];
      if (best) best[(size_t)c * nv + j] = ch.best[j];
    }
    if (costs) { costs[2 * c] = ch.cost; costs[2 * c + 1] = ch.bestCost; }
    if (counters) {
      counters[4 * c] = ch.accepted; counters[4 * c + 1] = ch.proposals;
      counters[4 * c + 2] = ch.swaps; counters[4 * c + 3] = ch.swapAttempts;
    }
  }
  return P6_OK;
}

p6_status p6_pt_set_split(p6_pt_session *s, int ctas_per_chain) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (ctas_per_chain != 1 && ctas_per_chain != 2) return set_error(P6_ERR_INVALID_ARG, "1 or 2 CTAs per chain");
  P6_CUDA(cudaSetDevice(s->device));
  if (ctas_per_chain == 2 && pt_cluster_capacity(s->smemSweep) < s->P.chains)
    return set_error(P6_ERR_CAPACITY, "the device cannot hold every chain's two-CTA cluster at once");
  s->split = ctas_per_chain;
  return P6_OK;
}

p6_status p6_pt_get_split(p6_pt_session *s, int *ctas_per_chain) {
  clear_error();
  if (!s || !ctas_per_chain) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *ctas_per_chain = s->split;
  return P6_OK;
}

p6_status p6_pt_synchronize(p6_pt_session *s, double timeout_seconds) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s->stream);
    if (e == cudaSuccess) return P6_OK;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_seconds)
      return set_error(P6_ERR_TIMEOUT, "the device did not finish within the deadline");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

p6_status p6_pt_last_batch_ms(p6_pt_session *s, float *ms) {
  clear_error();
  if (!s || !ms) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaEventSynchronize(s->ev1));
  P6_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
  return P6_OK;
}

p6_status p6_pt_vector_capacity(p6_pt_session *s, int *n_vectors) {
  clear_error();
  if (!s || !n_vectors) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *n_vectors = s->vecCap;
  return P6_OK;
}

p6_status p6_pt_set_trace(p6_pt_session *s, int enable) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t n = (size_t)s->P.chains * (kTraceHead + kTraceMove * s->P.nv);
  if (enable && !s->dTrace) {
    P6_CUDA(cudaMalloc(&s->dTrace, n * sizeof(double)));
    P6_CUDA(cudaMemsetAsync(s->dTrace, 0, n * sizeof(double), s->stream));
  }
  s->P.trace = enable ? s->dTrace : nullptr;
  return P6_OK;
}

p6_status p6_pt_read_trace(p6_pt_session *s, double *out) {
  clear_error();
  if (!s || !out || !s->dTrace) return set_error(P6_ERR_INVALID_ARG, "tracing was not enabled");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t n = (size_t)s->P.chains * (kTraceHead + kTraceMove * s->P.nv);
  P6_CUDA(cudaMemcpyAsync(out, s->dTrace, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_pt_launch_count(p6_pt_session *s, long long *count) {
  clear_error();
  if (!s || !count) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *count = s->launches;
  return P6_OK;
}

}  // extern "C"


// ===========================================================================
// Least-squares finish (js/rietveld_core.js:1953-2140): FP64 patterns and
// normal equations on the device, the damped Cholesky solve on the device,
// the scalar control of lm() on the host.
// ===========================================================================
namespace {
enum LmKind { K_SCALE, K_CELL, K_ANGLE, K_PROFILE, K_LORENTZ, K_ZERO, K_BISO, K_BKG, K_PO, K_SL, K_HL, K_DISP, K_TRANSP };

int lm_kind(const Params &P, int fi) {
  if (P.hasPo && fi == PBKG0 + P.nBkg) return K_PO;
  if (P.shiftIdx >= 0 && fi == P.shiftIdx) return K_DISP;
  if (P.shiftIdx >= 0 && fi == P.shiftIdx + 1) return K_TRANSP;
  if (P.asymIdx >= 0 && fi == P.asymIdx) return K_SL;
  if (P.asymIdx >= 0 && fi == P.asymIdx + 1) return K_HL;
  if (fi == SCALE) return K_SCALE;
  if (fi >= PA && fi <= PC) return K_CELL;
  if (fi >= PAL && fi <= PGA) return K_ANGLE;
  if (fi >= PU && fi <= PW) return K_PROFILE;
  if (fi == PX || fi == PY) return K_LORENTZ;
  if (fi == PZERO) return K_ZERO;
  if (fi == PBISO) return K_BISO;
  return K_BKG;
}
// fdStep (js/rietveld_core.js:526-538)
double lm_fd_step(int kind, double v) {
  const double a = std::fabs(v);
  switch (kind) {
    case K_CELL: return std::max(1e-6 * a, 1e-6);
    case K_ANGLE: case K_ZERO: case K_PO: return 1e-4;
    case K_DISP: return 1e-2;
    case K_TRANSP: return 1e-6;
    default: return std::max(1e-4 * a, 1e-5);
  }
}
// defaultLimits (js/rietveld_core.js:486-508): the range a finite-difference probe may use
void lm_limits(int kind, double v, double *lo, double *hi) {
  const double inf = std::numeric_limits<double>::infinity();
  switch (kind) {
    case K_SCALE: *lo = 0; *hi = inf; return;
    case K_CELL: *lo = 0.5 * v; *hi = 2 * v; return;
    case K_ANGLE: *lo = 30; *hi = 150; return;
    case K_BISO: *lo = -2; *hi = 30; return;
    case K_ZERO: *lo = -2; *hi = 2; return;
    case K_LORENTZ: *lo = 0; *hi = inf; return;
    case K_PO: *lo = 0.1; *hi = 5; return;
    case K_SL: *lo = 0; *hi = inf; return;
    default: *lo = -inf; *hi = inf; return;
  }
}
// stepCap (js/rietveld_core.js:511-524)
double lm_step_cap(int kind, double v) {
  switch (kind) {
    case K_CELL: return 0.02 * std::fabs(v) + 1e-6;
    case K_ANGLE: return 1;
    case K_BISO: return 2;
    case K_ZERO: return 0.1;
    case K_PO: return 0.25;
    case K_SL: case K_HL: return 0.01;
    case K_DISP: return 2;
    case K_TRANSP: return 0.01;
    case K_PROFILE: case K_LORENTZ: return 0.5 * std::max(std::fabs(v), 5.0);
    default: return std::numeric_limits<double>::infinity();
  }
}

// How far the Gaussian variance U tan^2 + V tan + W falls below zero over the fitted range.
double lm_violation(const p6_pt_session *s, const double *x) {
  std::vector<double> v = s->fullHost;
  for (size_t j = 0; j < s->indexHost.size(); ++j) v[s->indexHost[j]] = x[j];
  const double t0 = std::tan(s->tthFirst * kD2R / 2), t1 = std::tan(s->tthLast * kD2R / 2);
  const double U = v[PU], V = v[PV], W = v[PW];
  double m = std::min(U * t0 * t0 + V * t0 + W, U * t1 * t1 + V * t1 + W);
  if (U > 0) {
    const double ts = -V / (2 * U);
    if (ts > t0 && ts < t1) m = std::min(m, U * ts * ts + V * ts + W);
  }
  return m < 0 ? -m : 0;
}

p6_status lm_ensure(p6_pt_session *s, int m) {
  if (s->smem64 <= 0)
    return set_error(P6_ERR_CAPACITY, "too many reflections for the FP64 peak table of the least-squares finish");
  if (m <= s->lmCap) return P6_OK;
  for (void *p : {(void *)s->dLmVec, (void *)s->dLmY, (void *)s->dLmYu, (void *)s->dLmChi, (void *)s->dLmOut,
                  (void *)s->dLmF, (void *)s->dTrace})
    if (p) cudaFree(p);
  s->dLmVec = s->dLmY = s->dLmYu = s->dLmChi = s->dLmOut = nullptr;
  s->dLmF = nullptr;
  s->lmCap = 0;
  const int nv = s->P.nv, n = s->P.n;
  P6_CUDA(cudaMalloc(&s->dLmVec, (size_t)m * nv * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dLmY, (size_t)m * n * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dLmYu, (size_t)n * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dLmChi, (size_t)m * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dLmOut, (size_t)(nv * nv + nv + 1 + kMaxNv + 1) * sizeof(double)));
  P6_CUDA(cudaMalloc(&s->dLmF, (size_t)kMaxNv * sizeof(int)));
  s->lmCap = m;
  return P6_OK;
}

// chi^2 of n refined vectors with the FP64 model (one CTA each).
p6_status lm_costs(p6_pt_session *s, const double *x, int n, double *f) {
  p6_status st = lm_ensure(s, n);
  if (st != P6_OK) return st;
  P6_CUDA(cudaMemcpyAsync(s->dLmVec, x, (size_t)n * s->P.nv * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  pt_pattern64_kernel<<<n, kThreads, s->smem64, s->stream>>>(s->P, s->dLmVec, s->dLmY, nullptr, s->dLmChi);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  P6_CUDA(cudaMemcpyAsync(f, s->dLmChi, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}
p6_status lm_cost(p6_pt_session *s, const double *x, double *f) { return lm_costs(s, x, 1, f); }

// normal() at x: A (nv x nv), g (nv), f, left on the device in dLmOut and copied to the host.
p6_status lm_normal(p6_pt_session *s, const double *x, double *A, double *g, double *f) {
  const int nv = s->P.nv;
  std::vector<double> vecs((size_t)(1 + 2 * nv) * nv);
  std::copy(x, x + nv, vecs.begin());
  LmCols L{};
  int m = 1;
  for (int j = 0; j < nv; ++j) {
    const int fi = s->indexHost[j], kind = lm_kind(s->P, fi);
    L.plus[j] = L.minus[j] = 0;
    L.step[j] = 1;
    if (kind == K_SCALE) { L.kind[j] = 0; continue; }
    if (kind == K_BKG) { L.kind[j] = 1; L.bkg[j] = fi - PBKG0; continue; }
    const double val = x[j], h = lm_fd_step(kind, val);
    double llo, lhi;
    lm_limits(kind, val, &llo, &lhi);
    // the March-Dollase column is a forward difference (js/rietveld_core.js:1271-1275)
    const bool plus = kind == K_PO || val + h <= lhi, minus = kind != K_PO && val - h >= llo;
    const double vp = plus ? val + h : val, vm = minus ? val - h : val, d = vp - vm;
    if (!(d != 0)) { L.kind[j] = 3; continue; }
    L.kind[j] = 2;
    L.step[j] = d;
    if (plus) {
      std::copy(x, x + nv, vecs.begin() + (size_t)m * nv);
      vecs[(size_t)m * nv + j] = vp;
      L.plus[j] = m++;
    }
    if (minus) {
      std::copy(x, x + nv, vecs.begin() + (size_t)m * nv);
      vecs[(size_t)m * nv + j] = vm;
      L.minus[j] = m++;
    }
  }
  p6_status st = lm_ensure(s, m);
  if (st != P6_OK) return st;
  P6_CUDA(cudaMemcpyAsync(s->dLmVec, vecs.data(), (size_t)m * nv * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  // vector 0 (with its unit-scale column), then the finite-difference probes
  pt_pattern64_kernel<<<1, kThreads, s->smem64, s->stream>>>(s->P, s->dLmVec, s->dLmY, s->dLmYu, s->dLmChi);
  P6_CUDA(cudaGetLastError());
  if (m > 1) {
    pt_pattern64_kernel<<<m - 1, kThreads, s->smem64, s->stream>>>(s->P, s->dLmVec + nv, s->dLmY + s->P.n, nullptr,
                                                                    s->dLmChi + 1);
    P6_CUDA(cudaGetLastError());
  }
  const int blocks = nv * (nv + 1) / 2 + nv + 1;
  pt_normal_kernel<<<blocks, kThreads, 0, s->stream>>>(s->P, L, s->dLmY, s->dLmYu, s->dLmOut);
  P6_CUDA(cudaGetLastError());
  s->launches += m > 1 ? 3 : 2;
  std::vector<double> h((size_t)nv * nv + nv + 1);
  double chi0 = 0;
  P6_CUDA(cudaMemcpyAsync(h.data(), s->dLmOut, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaMemcpyAsync(&chi0, s->dLmChi, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  if (!std::isfinite(chi0))
    return set_error(P6_ERR_VALIDATION, "the model is not finite at the point of the normal equations");
  std::copy(h.begin(), h.begin() + (size_t)nv * nv, A);
  std::copy(h.begin() + (size_t)nv * nv, h.begin() + (size_t)nv * nv + nv, g);
  *f = h[(size_t)nv * nv + nv];
  return P6_OK;
}

// solveSPD of the free set on the device (A, g already in dLmOut).
p6_status lm_solve(p6_pt_session *s, const int *F, int nF, double mu, int mode, double *d, bool *ok) {
  const int nv = s->P.nv;
  P6_CUDA(cudaMemcpyAsync(s->dLmF, F, nF * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  double *out = s->dLmOut + nv * nv + nv + 1;
  pt_lm_solve_kernel<<<1, 32, 0, s->stream>>>(s->dLmOut, s->dLmOut + nv * nv, nv, s->dLmF, nF, mu, mode, out);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  std::vector<double> h(nF + 1);
  P6_CUDA(cudaMemcpyAsync(h.data(), out, (nF + 1) * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  *ok = h[nF] != 0;
  std::copy(h.begin(), h.begin() + nF, d);
  return P6_OK;
}
}  // namespace

extern "C" p6_status p6_pt_normal(p6_pt_session *s, const double *x, double *A, double *g, double *f) {
  clear_error();
  if (!s || !x || !A || !g || !f) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(s->device));
  return lm_normal(s, x, A, g, f);
}

extern "C" p6_status p6_pt_model_costs(p6_pt_session *s, const double *x, int n, double *chi2) {
  clear_error();
  if (!s || !x || !chi2 || n <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  return lm_costs(s, x, n, chi2);
}

extern "C" p6_status p6_pt_linear_start(p6_pt_session *s, double *x, double *chi2) {
  clear_error();
  if (!s || !x) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(s->device));
  const int nv = s->P.nv;
  std::vector<int> lin;
  for (int j = 0; j < nv; ++j) {
    const int k = lm_kind(s->P, s->indexHost[j]);
    if (k == K_SCALE || k == K_BKG) lin.push_back(j);
  }
  std::vector<double> A((size_t)nv * nv), g(nv), d(nv + 1), xt(x, x + nv);
  double f = 0;
  p6_status st = lm_normal(s, x, A.data(), g.data(), &f);
  if (st != P6_OK) return st;
  if (!lin.empty()) {
    bool ok = false;
    st = lm_solve(s, lin.data(), (int)lin.size(), 0.0, 1, d.data(), &ok);
    if (st != P6_OK) return st;
    if (ok) {
      for (size_t a = 0; a < lin.size(); ++a) {
        const int q = lin[a];
        xt[q] = std::min(s->hiHost[q], std::max(s->loHost[q], x[q] + d[a]));
      }
      double ft = 0;
      st = lm_cost(s, xt.data(), &ft);
      if (st != P6_OK) return st;
      if (ft < f) {
        std::copy(xt.begin(), xt.end(), x);
        f = ft;
      }
    }
  }
  if (chi2) *chi2 = f;
  return P6_OK;
}

extern "C" p6_status p6_pt_lm(p6_pt_session *s, double *x, int max_iter, double tol, double *out) {
  clear_error();
  if (!s || !x || max_iter < 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  const int nv = s->P.nv, nPts = s->P.n;
  if (!(tol > 0)) tol = 1e-5;
  std::vector<double> A((size_t)nv * nv), g(nv), dx(nv + 1), xn(nv), step(nv), sc(nv), cand(nv);
  std::vector<int> F(nv);
  double f = 0;
  p6_status st = lm_cost(s, x, &f);
  if (st != P6_OK) return st;
  if (!std::isfinite(f)) return set_error(P6_ERR_VALIDATION, "the model gives non-finite values at the start values");
  double mu = 1e-3, nu = 2, curViolation = lm_violation(s, x);
  int conv = 0, it, code = 0, accepted = 0;
  bool have = false;
  for (it = 0; it < max_iter; ++it) {
    if (!have) {
      double fNE = 0;
      st = lm_normal(s, x, A.data(), g.data(), &fNE);
      if (st != P6_OK) return st;
      have = true;
    }
    int nF = 0;
    for (int j = 0; j < nv; ++j) {
      const double lo = s->loHost[j], hi = s->hiHost[j];
      const bool atLo = x[j] <= lo + 1e-12 * (1 + std::fabs(lo)), atHi = x[j] >= hi - 1e-12 * (1 + std::fabs(hi));
      if (!((atLo && g[j] < 0) || (atHi && g[j] > 0)) && A[j * nv + j] > 0) F[nF++] = j;
    }
    if (!nF) { code = 5; break; }
    double grad = 0;
    const double noise = std::sqrt(std::max(f / std::max(1, nPts - nv), 1e-30));
    for (int a = 0; a < nF; ++a) {
      sc[a] = 1 / std::sqrt(A[F[a] * nv + F[a]]);
      grad = std::max(grad, std::fabs(g[F[a]]) * sc[a] / noise);
    }
    if (f < 1e-24 || grad < 1e-4) { code = 2; break; }
    bool ok = false;
    st = lm_solve(s, F.data(), nF, mu, 0, dx.data(), &ok);
    if (st != P6_OK) return st;
    if (!ok) {
      mu *= nu; nu *= 2;
      if (mu > 1e30) { code = 3; break; }
      continue;
    }
    std::copy(x, x + nv, xn.begin());
    std::fill(step.begin(), step.end(), 0.0);
    for (int a = 0; a < nF; ++a) {
      const int q = F[a];
      const double cap = lm_step_cap(lm_kind(s->P, s->indexHost[q]), x[q]);
      const double sh = std::max(-cap, std::min(cap, dx[a]));
      xn[q] = std::min(s->hiHost[q], std::max(s->loHost[q], x[q] + sh));
      step[q] = xn[q] - x[q];
    }
    double violation = lm_violation(s, xn.data());
    bool blocked = false;
    if (curViolation == 0 && violation > 0) {
      double loA = 0, hiA = 1;
      for (int bi = 0; bi < 24; ++bi) {
        const double mid = 0.5 * (loA + hiA);
        for (int a = 0; a < nv; ++a) cand[a] = x[a] + mid * step[a];
        if (lm_violation(s, cand.data()) == 0) loA = mid; else hiA = mid;
      }
      for (int a = 0; a < nv; ++a) { xn[a] = x[a] + loA * step[a]; step[a] = xn[a] - x[a]; }
      violation = lm_violation(s, xn.data());
      blocked = true;
    }
    double pred = 0, sAs = 0;
    for (int a = 0; a < nv; ++a) {
      if (!step[a]) continue;
      pred += 2 * g[a] * step[a];
      double tt = 0;
      for (int b = 0; b < nv; ++b) tt += A[a * nv + b] * step[b];
      sAs += step[a] * tt;
    }
    pred -= sAs;
    double fn = 0;
    st = lm_cost(s, xn.data(), &fn);
    if (st != P6_OK) return st;
    if (fn < f) {
      const double rho = pred > 0 ? (f - fn) / pred : 0.5, rel = (f - fn) / f;
      bool small = true;
      const double s2 = std::max(f, 1e-30) / std::max(1, nPts - nv);
      for (int a = 0; a < nF; ++a) {
        const int q = F[a];
        if (std::fabs(step[q]) * std::sqrt(A[q * nv + q] / s2) > 0.1) { small = false; break; }
      }
      std::copy(xn.begin(), xn.end(), x);
      f = fn;
      have = false;
      curViolation = violation;
      mu *= std::max(1.0 / 3, 1 - std::pow(2 * rho - 1, 3));
      nu = 2;
      ++accepted;
      if (!blocked && rel < tol && small) {
        if (++conv >= 2) { code = 1; ++it; break; }
      } else {
        conv = 0;
      }
    } else {
      mu *= nu; nu *= 2;
      if (mu > 1e20) { code = blocked ? 6 : (grad < 1e-3 ? 2 : 4); break; }
    }
  }
  if (out) { out[0] = f; out[1] = it; out[2] = accepted; out[3] = code; }
  return P6_OK;
}

// ===========================================================================
// p6_pt_costs_static: the cost kernel on a file-scope scratch array, so the
// call allocates no device memory.
// ===========================================================================
static __device__ __align__(256) unsigned char g_pt_static_scratch[P6_PT_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_scratch_mu;
unsigned char *g_static_scratch_addr[kMaxDevices] = {};
unsigned long long g_static_scratch_ctx[kMaxDevices] = {};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Unique id of the current device's context (the driver's cuCtxGetId, reached
// through the runtime's entry-point table so the library links no driver
// stub); 0 when the driver cannot say.  A device reset replaces the primary
// context, and with it the id and the module that holds the scratch array.
unsigned long long current_context_id() {
  typedef int (*GetCurrentFn)(void **);
  typedef int (*GetIdFn)(void *, unsigned long long *);
  static GetCurrentFn getCurrent = nullptr;
  static GetIdFn getId = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      getCurrent = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      getId = reinterpret_cast<GetIdFn>(f);
  }
  void *ctx = nullptr;
  unsigned long long id = 0;
  if (!getCurrent || !getId || getCurrent(&ctx) != 0 || !ctx || getId(ctx, &id) != 0) return 0;
  return id;
}

// Address of the scratch array on `device` (the current device): looked up
// with cudaGetSymbolAddress at the first call on the device, and again only
// when the device's context has changed since (cudaDeviceReset).
p6_status static_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices) return set_error(P6_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_static_scratch_addr[device] || ctx != g_static_scratch_ctx[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_pt_static_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_pt_static_scratch)");
    g_static_scratch_addr[device] = static_cast<unsigned char *>(p);
    g_static_scratch_ctx[device] = ctx;
  }
  *out = g_static_scratch_addr[device];
  return P6_OK;
}

// Waits for the session's stream for at most P6_PT_STATIC_WAIT_SECONDS.
p6_status static_wait(p6_pt_session *s) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s->stream);
    if (e == cudaSuccess) return P6_OK;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > P6_PT_STATIC_WAIT_SECONDS)
      return set_error(P6_ERR_TIMEOUT, "p6_pt_costs_static: the device did not finish within the deadline; "
                                       "call p6_pt_synchronize before reusing the output buffers");
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}
}  // namespace

extern "C" p6_status p6_pt_costs_static(p6_pt_session *s, const double *vectors, int n_vectors, double *costs,
                                        float *ycalc) {
  clear_error();
  if (!s || !vectors || !costs || n_vectors <= 0) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  const size_t vecBytes = align256((size_t)n_vectors * s->P.nv * sizeof(double));
  const size_t costBytes = align256((size_t)n_vectors * sizeof(double));
  const size_t yBytes = ycalc ? (size_t)n_vectors * s->P.n * sizeof(float) : 0;
  const size_t need = vecBytes + costBytes + yBytes;
  if (need > P6_PT_STATIC_SCRATCH_BYTES)
    return set_error(P6_ERR_CAPACITY, "p6_pt_costs_static: " + std::to_string(n_vectors) + " vectors need " +
                                          std::to_string(need) + " bytes of scratch, more than the " +
                                          std::to_string(P6_PT_STATIC_SCRATCH_BYTES) +
                                          "-byte static scratch; pass fewer vectors per call or use p6_pt_costs");
  P6_CUDA(cudaSetDevice(s->device));
  unsigned char *base = nullptr;
  const p6_status st = static_scratch(s->device, &base);
  if (st != P6_OK) return st;
  double *dVec = reinterpret_cast<double *>(base);
  double *dCost = reinterpret_cast<double *>(base + vecBytes);
  float *dY = ycalc ? reinterpret_cast<float *>(base + vecBytes + costBytes) : nullptr;
  P6_CUDA(cudaMemcpyAsync(dVec, vectors, (size_t)n_vectors * s->P.nv * sizeof(double), cudaMemcpyHostToDevice,
                          s->stream));
  pt_cost_kernel<<<n_vectors, kThreads, s->smemCost, s->stream>>>(s->P, dVec, dCost, dY);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  P6_CUDA(cudaMemcpyAsync(costs, dCost, (size_t)n_vectors * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (ycalc)
    P6_CUDA(cudaMemcpyAsync(ycalc, dY, (size_t)n_vectors * s->P.n * sizeof(float), cudaMemcpyDeviceToHost,
                            s->stream));
  return static_wait(s);
}
