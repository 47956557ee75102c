// Wyckoff-search trial evaluation on sm_100a.
//
// One generation of the reference kernel (swarm_reflection.wgsl:601-1270) per
// replica: proposal (one free site with p = 3/4, else every site), projection
// onto the Wyckoff subspace, symmetry expansion, grouped |F|^2 against the
// observed group intensities, the scale-free weighted wR2, clash and
// restraint penalties, Metropolis acceptance, Robbins-Monro step adaptation
// and the best-ever cache.  The layout is B200-first rather than a
// translation:
//
//  * one warp owns one replica; one CTA owns one replica ladder (the rungs of
//    one assignment, js/swarm_wyckoff.js:1784-1808), so the exchange sweep
//    (js/swarm_wyckoff.js:1825-1851) is a CTA barrier plus a shared-memory
//    swap, and a whole block of generations -- or a whole search -- is one
//    launch with no host round trip;
//  * coordinates are 32-bit fixed point (x * 2^32).  The orbit image
//    R x + t, the phase h.x mod 1 and the minimum-image separation are exact
//    integer arithmetic; only the final cosine is floating point (the SFU's
//    cos.approx on the exactly reduced turn, or an FMA-pipe polynomial);
//  * the static reflection, scattering-factor and group tables are staged
//    into shared memory once per CTA with the bulk-copy engine;
//  * the group sums scc, soo, sco are accumulated and reduced in FP64;
//  * random numbers are Philox4x32-10 keyed by (chain seed, session key) and
//    counted by (generation, replica, lane, purpose): no generator state.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ct_internal.h"
#include "mlp_internal.h"
#include "p6_common.cuh"

namespace p6 {
namespace wy {

constexpr int kMaxSites = 32;
constexpr int kMaxElem = 8;
constexpr int kMaxRules = 32;
constexpr int kMaxRungs = 32;
constexpr float kNoNeighbour = 1.0e9f;
constexpr float kNoPartnerCharge = 5.0f;
constexpr float kCoordSoftA = 0.25f;
constexpr double kTwoPow32 = 4294967296.0;
constexpr float kTurnToRad = 1.46291807926715968e-09f;  // 2 pi / 2^32
constexpr uint32_t kStageWaitLimit = 1u << 24;

struct OpFix {
  int r[9];
  uint32_t t[3];
};

struct ProjFix {
  int num[9];
  int den;
  uint32_t t[3];
  int pad[2];  // pad[0] = 1: diagonal 0/1 projector with den 1 (keep or drop each coordinate)
};

struct RuleDev {
  int a, b;
  float dmin, dmax, count;
  int mode, geom, pad;
};

struct ReflRec {  // 8 bytes
  short h, k, l;
  unsigned short mult;
};

// A rigid fragment with torsions (a molecule whose atoms are the sites of the
// assignment, in order): per replica, a translation (fractional), an
// orientation quaternion and the torsion angles replace the sites' free
// coordinates as the searched parameters.
constexpr int kFragMaxAtoms = 32, kFragMaxTors = 8, kFragParams = 16;
struct FragDev {
  int nAtoms, nTors;
  int axisB[kFragMaxTors], axisC[kFragMaxTors];  // each torsion turns about the bond b -> c
  uint32_t moving[kFragMaxTors];                  // the atoms it turns (bit i = atom i)
  float ref[kFragMaxAtoms * 3];                   // Cartesian reference geometry (A), about its centroid
  float toFrac[9];                                // Cartesian -> fractional of the cell, row-major
  float transStep, angleStep;                     // per unit of the replica's step width
};

struct PState {  // mirror of p6_wy_particle_state
  float fit, cc, pen, step, temp;
  uint32_t seed, accepted, pad;
  float bestFit, bestCC, bestPen, bestPad;
};
static_assert(sizeof(PState) == 48, "state stride");

struct Params {
  const uint32_t *gen;     // reordered genPack per assignment: F atoms (site runs) first
  const uint32_t *genOrig; // genPack in the caller's order (polyhedron moves walk it)
  const int4 *runs;        // per assignment, kMaxSites runs {start, end, type, site}
  const int *nRuns;        // per assignment
  const int *nF;           // per assignment: atoms entering |F|^2
  const uint32_t *freeMask;
  const OpFix *ops;
  const ProjFix *proj;     // per (assignment, site)
  const unsigned char *blob;  // staged static tables
  int blobBytes, offRefl, offF, offGroup, offRmin, offSoo, offOps, offPairs, nPairs;
  const int2 *pairRange;   // per assignment {offset, count} of its site-representative pairs; null: all pairs
  const RuleDev *rules;
  int nRules;
  int numParticles, nTot, maxSites, nRefl, nGroups, nElem, nAssign;
  float orth[9];
  int xf[9];
  int minImageShell, countShell, centro, maxCoordSlots, geomSlots;
  float penClash, penBond, penCoord, penGeom;
  float stepUp, stepDown, stepMin, stepMax;
  uint32_t runKey;
  uint32_t *pos;           // [2][numParticles][maxSites*3]
  PState *st;
  const uint32_t *assign;
  const int *ladders;      // nLadders * rungs, -1 empty; null: consecutive particles
  int rungs, nLadders;
  const int *schedGroups;  // per generation; null: use ngaArg/penArg
  const float *schedPen;
  const float *quenchSd;   // per generation: greedy quench with this step; null: Metropolis with adapted steps
  const uint32_t *extProp; // per particle: the proposal to evaluate (learned search); null: the kernel proposes
  int ngaArg;
  float penArg;
  uint32_t *tracePos;
  float *traceRec;
  float *traceIc;          // per particle, nRefl: mult |F|^2 of the last evaluation
  unsigned long long *swapStats;  // [tried, taken]
  int *errFlag;
  float polyProb;          // share of proposals that try a polyhedron move (0 without counted rules)
  int blobGlobal;          // the static tables are read from global memory (too large to stage)
  float invOrth[9];        // Cartesian -> fractional of the cell's own basis
  int warpSmemBytes;       // per-warp shared-memory slice
  int genOff, projOff, atomsOff, icOff;  // offsets inside the slice
  int cbOff, atoms2Off, nReflPad;          // incremental site sums and the second atom bank
  int curOff, propOff, runsOff, slotOff;   // WarpView offsets
  // factored FP64 structure factors (cos mode 2): blob offsets of the monomial
  // coefficients (real, imaginary or -1 when every one is real), their table
  // indices and the FP64 scattering factors; the per-axis table shape; the
  // per-warp offsets of the site tables and their coordinate tags
  int offK, offKi, offIdx, offF64;
  int nMono, tabLen, tabE;
  int axE[3], axOff[3];
  int tabOff, tagOff;
  double *traceSums;       // per particle {scc, soo, sco} of the last traced evaluation (FP64)
  const FragDev *frag;     // rigid-fragment search: the fragment; null: the sites move independently
  float *fragState;        // per particle the current fragment parameters (kFragParams floats)
  float *fragBest;         // per particle the parameters of its best structure
  float *fragProp;         // per particle the proposed parameters of a deferred generation
  int fragOff;             // per-warp slice offset of the current and proposed parameters
  int deferAccept;         // fixed-profile search: evaluate and record the proposal, leave the decision
                           // to wy_profile_accept_kernel (the fitness is the profile chi^2)
  // fixed-profile fitness in Gram form (cos mode 2): v = P (w y) per reflection,
  // G = P W P^T as its upper band by diagonal (profG[d * profK + k] = G[k][k + d]);
  // null: the grouped-intensity fitness
  const double *profV, *profG;
  int profK, profBw;
  double profSyy;
};

// ---------------------------------------------------------------------------
// Cosine / sine of a 32-bit turn.
// ---------------------------------------------------------------------------
// cos(2 pi t) and sin(2 pi t) with the SFU: the turn is already reduced
// exactly, so the hardware sees an argument in [-pi, pi).
__device__ __forceinline__ float cos_turn_sfu(uint32_t ph) {
  return __cosf((float)(int)ph * kTurnToRad);
}
__device__ __forceinline__ void sincos_turn_sfu(uint32_t ph, float *s, float *c) {
  __sincosf((float)(int)ph * kTurnToRad, s, c);
}

// Polynomial form: quarter-turn reduction in integers, then Taylor series of
// sin and cos of phi = x pi / 2, |x| <= 1/2 (truncation below 2e-9).
constexpr double kHalfPi = 1.57079632679489661923;
__device__ __forceinline__ void sincos_turn_poly(uint32_t ph, float *s_out, float *c_out) {
  uint32_t q = (ph + 0x20000000u) >> 30;
  int r = (int)(ph - (q << 30));
  float x = (float)r * (1.0f / 1073741824.0f);
  float x2 = x * x;
  constexpr double a = kHalfPi;
  constexpr float S0 = (float)a, S1 = (float)(-a * a * a / 6.0), S2 = (float)(a * a * a * a * a / 120.0),
                  S3 = (float)(-a * a * a * a * a * a * a / 5040.0),
                  S4 = (float)(a * a * a * a * a * a * a * a * a / 362880.0);
  constexpr float C1 = (float)(-a * a / 2.0), C2 = (float)(a * a * a * a / 24.0),
                  C3 = (float)(-a * a * a * a * a * a / 720.0),
                  C4 = (float)(a * a * a * a * a * a * a * a / 40320.0),
                  C5 = (float)(-a * a * a * a * a * a * a * a * a * a / 3628800.0);
  float sp = x * fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, S4, S3), S2), S1), S0);
  float cp = fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, C5, C4), C3), C2), C1), 1.0f);
  float cs = (q & 1u) ? sp : cp;
  float sn = (q & 1u) ? cp : sp;
  if ((q + 1u) & 2u) cs = -cs;   // q = 1, 2
  if (q & 2u) sn = -sn;          // q = 2, 3
  *s_out = sn;
  *c_out = cs;
}

template <int COSMODE>
__device__ __forceinline__ float cos_turn(uint32_t ph) {
  if (COSMODE == 0) return cos_turn_sfu(ph);
  float s, c;
  sincos_turn_poly(ph, &s, &c);
  return c;
}
template <int COSMODE>
__device__ __forceinline__ void sincos_turn(uint32_t ph, float *s, float *c) {
  if (COSMODE == 0)
    sincos_turn_sfu(ph, s, c);
  else
    sincos_turn_poly(ph, s, c);
}

// ---------------------------------------------------------------------------
// Geometry helpers (fixed point).
// ---------------------------------------------------------------------------
// Exact separation i - j in the reduced basis, nearest image, as fractions.
__device__ __forceinline__ void frac_delta(const Params &P, uint4 a, uint4 b, float q[3]) {
  int d0 = (int)(a.x - b.x), d1 = (int)(a.y - b.y), d2 = (int)(a.z - b.z);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    uint32_t v = (uint32_t)P.xf[3 * i] * (uint32_t)d0 + (uint32_t)P.xf[3 * i + 1] * (uint32_t)d1 +
                 (uint32_t)P.xf[3 * i + 2] * (uint32_t)d2;
    q[i] = (float)(int)v * (1.0f / 4294967296.0f);
  }
}
__device__ __forceinline__ void cart_vec(const Params &P, const float t[3], float c[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) c[i] = P.orth[3 * i] * t[0] + P.orth[3 * i + 1] * t[1] + P.orth[3 * i + 2] * t[2];
}
__device__ __forceinline__ float cart_len(const Params &P, const float t[3]) {
  float c[3];
  cart_vec(P, t, c);
  return sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}
__device__ __forceinline__ float cart_dist(const Params &P, uint4 a, uint4 b) {
  float q[3];
  frac_delta(P, a, b, q);
  float best = 1e30f;
  const int S = P.minImageShell;
  for (int i = -S; i <= S; ++i)
    for (int j = -S; j <= S; ++j)
      for (int k = -S; k <= S; ++k) {
        float t[3] = {q[0] + i, q[1] + j, q[2] + k}, c[3];
        cart_vec(P, t, c);
        best = fminf(best, c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      }
  return sqrtf(best);
}

__device__ __forceinline__ float geom_cos_error(int code, float c) {
  switch (code) {
    case 1: return c + 1.0f;
    case 2: return c + 0.5f;
    case 3: return c + 0.3333333f;
    case 4:
    case 5: return fminf(fabsf(c), fabsf(c + 1.0f));
    default: return 0.0f;
  }
}

__device__ __forceinline__ int64_t floor_div(int64_t a, int d) {
  int64_t q = a / d;
  if ((a % d) != 0 && a < 0) --q;
  return q;
}

// ---------------------------------------------------------------------------
// Warp-level pieces of one trial.
//
// Work is issue-bound (every replica generation is a few thousand warp
// instructions for a hundred or so warp-wide cosines), so the layout below
// is chosen to minimise instructions per cosine: up to four reflections per
// lane share each broadcast atom load, the phase is three integer
// multiply-adds, inversion partners are summed once, the clash loop walks the
// site representatives' pairs on squared distances, the constant sum of
// w Iobs^2 comes from a prefix table, and the chain state lives in registers
// of lane 0.
// ---------------------------------------------------------------------------

// Per-warp shared-memory slice, sized by the session's max_sites (pointers into the slice).
struct WarpView {
  int *meta;       // A, nRuns, nF, nSites, freeMask, particle (8 ints)
  uint32_t *cur;   // current site coordinates, maxSites * 3
  uint32_t *prop;  // proposal, maxSites * 3
  int4 *runs;      // per site run of F atoms {start, end, type, site}, maxSites
  int *slot;       // incremental: physical slot of each site's sums; slot[maxSites] is the spare
};

__device__ __forceinline__ WarpView warp_view(unsigned char *base, const Params &P) {
  WarpView v;
  v.meta = reinterpret_cast<int *>(base);
  v.cur = reinterpret_cast<uint32_t *>(base + P.curOff);
  v.prop = reinterpret_cast<uint32_t *>(base + P.propOff);
  v.runs = reinterpret_cast<int4 *>(base + P.runsOff);
  v.slot = reinterpret_cast<int *>(base + P.slotOff);
  return v;
}

// ---------------------------------------------------------------------------
// Incremental structure factors.  Per replica, C_s(h) = sum over the images of
// site s entering |F|^2 of cos (and sin) 2 pi h.x is kept in shared memory in
// two banks; a proposal recomputes C_s only for the sites it moved, into the
// other bank, and |F(h)| = sum_s f_s(h) C_s(h) is re-summed in site order --
// the same order as a full evaluation, so the result is bit-identical.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int nrefl_active(const float4 *groups, int nga) {
  return nga > 0 ? (int)(groups[nga - 1].x + groups[nga - 1].y) : 0;
}

// Group sums scc, sco (FP64) from mult |F|^2 per reflection; soo from the prefix table.
__device__ __forceinline__ void group_sums(const Params &P, const float *ic, const float4 *groups,
                                           const double *sooPrefix, int nga, int lane, double sums[3]) {
  double dcc = 0.0, dco = 0.0;
  for (int g = lane; g < nga; g += 32) {
    const float4 gm = groups[g];
    if (!(gm.w > 0.f)) continue;
    const int start = (int)gm.x, cnt = (int)gm.y;
    float iCalc = 0.f;
    for (int m = 0; m < cnt; ++m) iCalc += ic[start + m];
    const double wc = (double)gm.w * (double)iCalc;
    dcc = fma(wc, (double)iCalc, dcc);
    dco = fma(wc, (double)gm.z, dco);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dcc += __shfl_xor_sync(0xffffffffu, dcc, o);
    dco += __shfl_xor_sync(0xffffffffu, dco, o);
  }
  sums[0] = dcc;
  sums[1] = sooPrefix[nga];
  sums[2] = dco;
  __syncwarp();
}

// Cosine and sine sums of one run for two reflections.  The run's first
// nPair = run.w >> 8 atoms lead inversion pairs whose partners (the run's last
// nPair atoms) are not read: a leader's cosine counts twice and its sine
// cancels.  The singles follow the leaders.
template <int COSMODE>
__device__ __forceinline__ void run_sums(const int4 run, const uint4 *atoms, bool centro, uint32_t h0, uint32_t k0,
                                         uint32_t l0, uint32_t h1, uint32_t k1, uint32_t l1, float &c0, float &s0,
                                         float &c1, float &s1) {
  const int nPair = run.w >> 8;
  const int lead = run.x + nPair, end = run.y - nPair;
  float p0 = 0.f, p1 = 0.f;
  for (int a = run.x; a < lead; ++a) {
    const uint4 at = atoms[a];
    p0 += cos_turn<COSMODE>(h0 * at.x + k0 * at.y + l0 * at.z);
    p1 += cos_turn<COSMODE>(h1 * at.x + k1 * at.y + l1 * at.z);
  }
  c0 = 2.f * p0;
  c1 = 2.f * p1;
  s0 = 0.f;
  s1 = 0.f;
  if (centro) {
    for (int a = lead; a < end; ++a) {
      const uint4 at = atoms[a];
      c0 += cos_turn<COSMODE>(h0 * at.x + k0 * at.y + l0 * at.z);
      c1 += cos_turn<COSMODE>(h1 * at.x + k1 * at.y + l1 * at.z);
    }
  } else {
    for (int a = lead; a < end; ++a) {
      const uint4 at = atoms[a];
      float sa, ca, sb, cb;
      sincos_turn<COSMODE>(h0 * at.x + k0 * at.y + l0 * at.z, &sa, &ca);
      sincos_turn<COSMODE>(h1 * at.x + k1 * at.y + l1 * at.z, &sb, &cb);
      c0 += ca; s0 += sa; c1 += cb; s1 += sb;
    }
  }
}

// C_s for the sites in `mask`, written to physical slot ws.slot[s], except
// site `spareSite` (if >= 0), written to the spare slot ws.slot[maxSites].
template <int COSMODE>
__device__ __forceinline__ void site_sums(const Params &P, const WarpView &ws, const uint4 *atoms, float *Cb,
                                          int nAct, uint32_t mask, int spareSite, const ReflRec *refl, int lane) {
  const int nRuns = ws.meta[1];
  const bool centro = P.centro != 0;
  const int comp = centro ? 1 : 2;
  const int pad = P.nReflPad;
  for (int r0 = lane; r0 < nAct; r0 += 64) {
    const int r1 = r0 + 32;
    const bool has1 = r1 < nAct;
    const ReflRec a0 = refl[r0];
    const ReflRec a1 = refl[has1 ? r1 : r0];
    const uint32_t h0 = (uint32_t)(int)a0.h, k0 = (uint32_t)(int)a0.k, l0 = (uint32_t)(int)a0.l;
    const uint32_t h1 = (uint32_t)(int)a1.h, k1 = (uint32_t)(int)a1.k, l1 = (uint32_t)(int)a1.l;
    for (int q = 0; q < nRuns; ++q) {
      const int4 run = ws.runs[q];
      const int site = run.w & 0xFF;
      if (!((mask >> site) & 1u)) continue;
      float c0, s0, c1, s1;
      run_sums<COSMODE>(run, atoms, centro, h0, k0, l0, h1, k1, l1, c0, s0, c1, s1);
      const int phys = site == spareSite ? ws.slot[P.maxSites] : ws.slot[site];
      float *dst = Cb + (size_t)phys * pad * comp;
      dst[r0 * comp] = c0;
      if (!centro) dst[r0 * comp + 1] = s0;
      if (has1) {
        dst[r1 * comp] = c1;
        if (!centro) dst[r1 * comp + 1] = s1;
      }
    }
  }
  __syncwarp();
}

// |F|^2 and the group sums from the cached site sums; site `spareSite` (if >= 0)
// is read from the spare slot.
__device__ __forceinline__ void fitness_from_banks(const Params &P, const WarpView &ws, const float *Cb,
                                                   int spareSite, float *ic, const ReflRec *refl,
                                                   const float *ftab, const float4 *groups,
                                                   const double *sooPrefix, int nga, int lane, double sums[3],
                                                   float *traceIc) {
  const int nRuns = ws.meta[1];
  const int nAct = nrefl_active(groups, nga);
  const bool centro = P.centro != 0;
  const int comp = centro ? 1 : 2;
  const int pad = P.nReflPad;
  const int nElem = P.nElem;
  for (int r = lane; r < nAct; r += 32) {
    float fr = 0.f, fi = 0.f;
    for (int q = 0; q < nRuns; ++q) {
      const int4 run = ws.runs[q];
      const int site = run.w & 0xFF;
      const int phys = site == spareSite ? ws.slot[P.maxSites] : ws.slot[site];
      const float *src = Cb + ((size_t)phys * pad + r) * comp;
      const float w = ftab[r * nElem + run.z];
      fr = fmaf(w, src[0], fr);
      if (!centro) fi = fmaf(w, src[1], fi);
    }
    const float v = (float)refl[r].mult * (fr * fr + fi * fi);
    ic[r] = v;
    if (traceIc) traceIc[r] = v;
  }
  __syncwarp();
  group_sums(P, ic, groups, sooPrefix, nga, lane, sums);
}

// Up to four reflections per lane per pass (rows base + lane + 32 j): each
// broadcast atom load feeds NR independent cosine chains.  The arithmetic per
// reflection is the same sequence as run_sums, so |F|^2 is bit-identical to
// the site-sum path.
template <int COSMODE, int NR>
__device__ __forceinline__ void fit_rows(const Params &P, const WarpView &ws, const uint4 *atoms, float *ic,
                                         const ReflRec *refl, const float *ftab, int base, int nAct, int lane,
                                         float *traceIc) {
  const int nRuns = ws.meta[1];
  const bool centro = P.centro != 0;
  const int nElem = P.nElem;
  int r[NR];
  uint32_t h[NR], k[NR], l[NR];
  float fr[NR], fi[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    r[j] = min(base + lane + 32 * j, nAct - 1);
    const ReflRec a = refl[r[j]];
    h[j] = (uint32_t)(int)a.h;
    k[j] = (uint32_t)(int)a.k;
    l[j] = (uint32_t)(int)a.l;
    fr[j] = 0.f;
    fi[j] = 0.f;
  }
  for (int q = 0; q < nRuns; ++q) {
    const int4 run = ws.runs[q];
    const int nPair = run.w >> 8;
    const int lead = run.x + nPair, end = run.y - nPair;
    float c[NR], s[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      c[j] = 0.f;
      s[j] = 0.f;
    }
    for (int a = run.x; a < lead; ++a) {
      const uint4 at = atoms[a];
#pragma unroll
      for (int j = 0; j < NR; ++j) c[j] += cos_turn<COSMODE>(h[j] * at.x + k[j] * at.y + l[j] * at.z);
    }
#pragma unroll
    for (int j = 0; j < NR; ++j) c[j] = 2.f * c[j];
    if (centro) {
      for (int a = lead; a < end; ++a) {
        const uint4 at = atoms[a];
#pragma unroll
        for (int j = 0; j < NR; ++j) c[j] += cos_turn<COSMODE>(h[j] * at.x + k[j] * at.y + l[j] * at.z);
      }
    } else {
      for (int a = lead; a < end; ++a) {
        const uint4 at = atoms[a];
#pragma unroll
        for (int j = 0; j < NR; ++j) {
          float sa, ca;
          sincos_turn<COSMODE>(h[j] * at.x + k[j] * at.y + l[j] * at.z, &sa, &ca);
          c[j] += ca;
          s[j] += sa;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      const float w = ftab[r[j] * nElem + run.z];
      fr[j] = fmaf(w, c[j], fr[j]);
      if (!centro) fi[j] = fmaf(w, s[j], fi[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if (base + lane + 32 * j < nAct) {
      const float v = (float)refl[r[j]].mult * (fr[j] * fr[j] + fi[j] * fi[j]);
      ic[r[j]] = v;
      if (traceIc) traceIc[r[j]] = v;
    }
  }
}

// |F|^2 straight from the atoms, in passes of 128, 96, 64 or 32 reflections
// (fit_rows with NR = 4, 3, 2, 1 as the remaining count needs): the same
// per-run summation order as site_sums followed by fitness_from_banks, so the
// result is bit-identical.
template <int COSMODE>
__device__ __forceinline__ void fitness_direct(const Params &P, const WarpView &ws, const uint4 *atoms, float *ic,
                                               const ReflRec *refl, const float *ftab, const float4 *groups,
                                               const double *sooPrefix, int nga, int lane, double sums[3],
                                               float *traceIc) {
  const int nAct = nrefl_active(groups, nga);
  for (int base = 0; base < nAct;) {
    const int rem = nAct - base;
    if (rem > 96) {
      fit_rows<COSMODE, 4>(P, ws, atoms, ic, refl, ftab, base, nAct, lane, traceIc);
      base += 128;
    } else if (rem > 64) {
      fit_rows<COSMODE, 3>(P, ws, atoms, ic, refl, ftab, base, nAct, lane, traceIc);
      base += 96;
    } else if (rem > 32) {
      fit_rows<COSMODE, 2>(P, ws, atoms, ic, refl, ftab, base, nAct, lane, traceIc);
      base += 64;
    } else {
      fit_rows<COSMODE, 1>(P, ws, atoms, ic, refl, ftab, base, nAct, lane, traceIc);
      base += 32;
    }
  }
  __syncwarp();
  group_sums(P, ic, groups, sooPrefix, nga, lane, sums);
}

// ---------------------------------------------------------------------------
// Factored FP64 structure factors (cos mode 2), for groups whose rotations are
// all diagonal (triclinic, monoclinic, orthorhombic).  With R_j = diag(sigma_j)
// the image phase separates by axis, e^{2 pi i h.(R_j x + t_j)} = e^{2 pi i h.t_j}
// prod_a (c_a + i sigma_ja sgn(h_a) s_a), c_a = cos 2 pi |h_a| x_a,
// s_a = sin 2 pi |h_a| x_a.  Summed over the N_p operators modulo centring, a
// site with n_s images entering |F|^2 contributes
//   S_s(h) = n_s sum_m K_m(h) prod_a (bit a of m ? s_a : c_a),
//   K_m(h) = (1/N_p) sum_j e^{2 pi i h.t_j} prod_{a in m} i sigma_ja sgn(h_a),
// because each image is reached by |stabiliser| = N_p / n_s operators.  K
// depends on the reflection alone (host-side, exact phases); an mmm group
// leaves one monomial per reflection, 2/m two.  Per site and evaluation the
// warp builds cos and sin of 2 pi n x_a for n = 0..max |h_a| from the exact
// 32-bit turn n x_a, in FP64; n_s is folded into the x table.  A table is
// rebuilt only when its site's coordinates differ from the ones it was built
// for (the tag), so a single-site move rebuilds one table.  |F|^2, the group
// sums and the fitness sums are FP64 throughout.
// ---------------------------------------------------------------------------
// sin and cos of 2 pi t for a 32-bit turn t: quarter-turn reduction in
// integers, then the Taylor series of sin and cos of phi = x pi / 2 with
// |x| <= 1/2 through x^15 and x^16 (truncation below 1e-17).
__device__ __forceinline__ void sincos_turn_f64(uint32_t ph, double *s_out, double *c_out) {
  const uint32_t q = (ph + 0x20000000u) >> 30;
  const int r = (int)(ph - (q << 30));
  const double x = (double)r * (kHalfPi / 1073741824.0);
  const double x2 = x * x;
  const double sp = x * fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, -1.0 / 1307674368000.0,
                                                                             1.0 / 6227020800.0),
                                                                     -1.0 / 39916800.0),
                                                             1.0 / 362880.0),
                                                     -1.0 / 5040.0),
                                             1.0 / 120.0),
                                     -1.0 / 6.0),
                             1.0);
  const double cp =
      fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, fma(x2, 1.0 / 20922789888000.0,
                                                                  -1.0 / 87178291200.0),
                                                          1.0 / 479001600.0),
                                                  -1.0 / 3628800.0),
                                          1.0 / 40320.0),
                                  -1.0 / 720.0),
                          1.0 / 24.0),
                  -0.5),
          1.0);
  double cs = (q & 1u) ? sp : cp;
  double sn = (q & 1u) ? cp : sp;
  if ((q + 1u) & 2u) cs = -cs;   // q = 1, 2
  if (q & 2u) sn = -sn;          // q = 2, 3
  *s_out = sn;
  *c_out = cs;
}

// Two banks of per-axis tables per site.  Bank k of site s holds, per axis a,
// cos(2 pi n x_a) for n < axE[a] then sin, starting at axOff[a], for the
// coordinates in its tag; the x table is scaled by n_s.  A site whose
// coordinates (in `sites`) match neither tag is rebuilt, one stale site at a
// time with its entries over the lanes, into the bank that does not hold the
// current coordinates' table -- so a rejected proposal leaves the current
// tables intact and an accepted one finds its own.  sel[q] is the table
// offset run q reads.
__device__ __forceinline__ void factor_tables(const Params &P, const WarpView &ws, const uint32_t *sites,
                                              double *tab, uint4 *tag, int *sel, int lane) {
  const int nRuns = ws.meta[1];
  const int ms = P.maxSites, tl = P.tabLen;
  bool need = false;
  int s = 0, bank = 0;
  if (lane < nRuns) {
    s = ws.runs[lane].w & 0xFF;
    const uint32_t X0 = sites[3 * s], X1 = sites[3 * s + 1], X2 = sites[3 * s + 2];
    const uint4 t0 = tag[s], t1 = tag[ms + s];
    if (t0.w != 0u && t0.x == X0 && t0.y == X1 && t0.z == X2) {
      bank = 0;
    } else if (t1.w != 0u && t1.x == X0 && t1.y == X1 && t1.z == X2) {
      bank = 1;
    } else {
      need = true;
      const uint32_t C0 = ws.cur[3 * s], C1 = ws.cur[3 * s + 1], C2 = ws.cur[3 * s + 2];
      bank = (t0.w != 0u && t0.x == C0 && t0.y == C1 && t0.z == C2) ? 1 : 0;
    }
    sel[lane] = (bank * ms + s) * tl;
  }
  uint32_t mask = __ballot_sync(0xffffffffu, need);
  __syncwarp();
  const int e0 = P.axE[0], e01 = P.axE[0] + P.axE[1];
  while (mask) {
    const int q = __ffs(mask) - 1;
    mask &= mask - 1u;
    const int4 run = ws.runs[q];
    const int sq = run.w & 0xFF;
    const double ns = (double)(run.y - run.x);
    double *t = tab + sel[q];
    for (int j = lane; j < P.tabE; j += 32) {
      const int a = j < e0 ? 0 : (j < e01 ? 1 : 2);
      const int n = j - (a == 0 ? 0 : (a == 1 ? e0 : e01));
      double sn, cs;
      sincos_turn_f64((uint32_t)n * sites[3 * sq + a], &sn, &cs);
      if (a == 0) {
        sn *= ns;
        cs *= ns;
      }
      t[P.axOff[a] + n] = cs;
      t[P.axOff[a] + P.axE[a] + n] = sn;
    }
  }
  if (need) tag[bank * ms + s] = make_uint4(sites[3 * s], sites[3 * s + 1], sites[3 * s + 2], 1u);
  __syncwarp();
}

// Group sums scc, sco (FP64) from FP64 mult |F|^2; soo from the prefix table.
__device__ __forceinline__ void group_sums_f64(const double *ic, const float4 *groups, const double *sooPrefix,
                                               int nga, int lane, double sums[3]) {
  double dcc = 0.0, dco = 0.0;
  for (int g = lane; g < nga; g += 32) {
    const float4 gm = groups[g];
    if (!(gm.w > 0.f)) continue;
    const int start = (int)gm.x, cnt = (int)gm.y;
    double iCalc = 0.0;
    for (int m = 0; m < cnt; ++m) iCalc += ic[start + m];
    const double wc = (double)gm.w * iCalc;
    dcc = fma(wc, iCalc, dcc);
    dco = fma(wc, (double)gm.z, dco);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dcc += __shfl_xor_sync(0xffffffffu, dcc, o);
    dco += __shfl_xor_sync(0xffffffffu, dco, o);
  }
  sums[0] = dcc;
  sums[1] = sooPrefix[nga];
  sums[2] = dco;
  __syncwarp();
}

// mult |F|^2 of reflections base + lane and base + lane + 32 from the site
// tables: F(h) = sum_k K_k(h) sum_s f_s(h) T_{s,k}(h), T a product of three
// table entries whose indices (10 bits each) the host packed per (k, h).  The
// two reflections of a lane share each run's loads; their table offsets are
// unpacked once per monomial, outside the loop over sites.
__device__ __forceinline__ void factored_rows(const Params &P, const WarpView &ws, const double *tab, const int *sel,
                                              double *ic, const ReflRec *refl, const unsigned char *stat, int base,
                                              int nAct, int lane, float *traceIc) {
  constexpr int NR = 2;
  const int nRuns = ws.meta[1];
  const int nM = P.nMono, pad = P.nReflPad;
  const double *kre = reinterpret_cast<const double *>(stat + P.offK);
  const double *kim = P.offKi >= 0 ? reinterpret_cast<const double *>(stat + P.offKi) : nullptr;
  const uint32_t *idx = reinterpret_cast<const uint32_t *>(stat + P.offIdx);
  const double *f64 = reinterpret_cast<const double *>(stat + P.offF64);
  int r[NR];
  double fr[NR], fi[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    r[j] = min(base + lane + 32 * j, nAct - 1);
    fr[j] = 0.0;
    fi[j] = 0.0;
  }
  for (int k = 0; k < nM; ++k) {
    int o0[NR], o1[NR], o2[NR];
    double acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      const uint32_t w = idx[k * pad + r[j]];
      o0[j] = (int)(w & 0x3FFu);
      o1[j] = (int)((w >> 10) & 0x3FFu);
      o2[j] = (int)(w >> 20);
      acc[j] = 0.0;
    }
#pragma unroll 4
    for (int q = 0; q < nRuns; ++q) {
      const int4 run = ws.runs[q];
      const double *t = tab + sel[q];
      const double *fq = f64 + (size_t)run.z * pad;
#pragma unroll
      for (int j = 0; j < NR; ++j) acc[j] = fma(fq[r[j]], t[o0[j]] * t[o1[j]] * t[o2[j]], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      fr[j] = fma(kre[k * pad + r[j]], acc[j], fr[j]);
      if (kim) fi[j] = fma(kim[k * pad + r[j]], acc[j], fi[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < NR; ++j)
    if (base + lane + 32 * j < nAct) {
      const double v = (double)refl[r[j]].mult * (fr[j] * fr[j] + fi[j] * fi[j]);
      ic[r[j]] = v;
      if (traceIc) traceIc[r[j]] = (float)v;
    }
}

// The factored evaluation of the coordinates in `sites`: stale site tables
// rebuilt, then |F|^2 in passes of 64 reflections, then the FP64 group sums.
__device__ __forceinline__ void fitness_factored(const Params &P, const WarpView &ws, const uint32_t *sites,
                                                 double *tab, uint4 *tag, double *ic, const ReflRec *refl,
                                                 const unsigned char *stat, const float4 *groups,
                                                 const double *sooPrefix, int nga, int lane, double sums[3],
                                                 float *traceIc) {
  int *sel = reinterpret_cast<int *>(tag + 2 * P.maxSites);
  factor_tables(P, ws, sites, tab, tag, sel, lane);
  const int nAct = nrefl_active(groups, nga);
  for (int base = 0; base < nAct; base += 64)
    factored_rows(P, ws, tab, sel, ic, refl, stat, base, nAct, lane, traceIc);
  __syncwarp();
  group_sums_f64(ic, groups, sooPrefix, nga, lane, sums);
}

// Expand the images of the sites in `mask` from `sites` into dst; copy the others from src.
__device__ __forceinline__ void expand_moved(const Params &P, const uint32_t *gen, const OpFix *ops,
                                             const uint32_t *sites, uint32_t mask, const uint4 *src, uint4 *dst,
                                             int lane) {
  const int maxT = max(min(P.nElem, kMaxElem), 1) - 1;
  for (int i = lane; i < P.nTot; i += 32) {
    const uint32_t w = gen[i];
    const int s = w & 0xFF;
    if (!((mask >> s) & 1u)) {
      dst[i] = src[i];
      continue;
    }
    const int o = (w >> 8) & 0xFFF, t = min((int)((w >> 20) & 0xF), maxT);
    const OpFix &op = ops[o];
    const uint32_t x = sites[s * 3], y = sites[s * 3 + 1], z = sites[s * 3 + 2];
    uint4 a;
    a.x = (uint32_t)op.r[0] * x + (uint32_t)op.r[1] * y + (uint32_t)op.r[2] * z + op.t[0];
    a.y = (uint32_t)op.r[3] * x + (uint32_t)op.r[4] * y + (uint32_t)op.r[5] * z + op.t[1];
    a.z = (uint32_t)op.r[6] * x + (uint32_t)op.r[7] * y + (uint32_t)op.r[8] * z + op.t[2];
    a.w = (uint32_t)t;
    dst[i] = a;
  }
  __syncwarp();
}

// Symmetry expansion of `sites` into atoms[0..nTot) (reordered genPack, ops in smem).
__device__ __forceinline__ void expand(const Params &P, const uint32_t *gen, const OpFix *ops,
                                       const uint32_t *sites, uint4 *atoms, int lane) {
  const int maxT = max(min(P.nElem, kMaxElem), 1) - 1;
  for (int i = lane; i < P.nTot; i += 32) {
    const uint32_t w = gen[i];
    const int s = w & 0xFF, o = (w >> 8) & 0xFFF, t = min((int)((w >> 20) & 0xF), maxT);
    const OpFix &op = ops[o];
    const uint32_t x = sites[s * 3], y = sites[s * 3 + 1], z = sites[s * 3 + 2];
    uint4 a;
    a.x = (uint32_t)op.r[0] * x + (uint32_t)op.r[1] * y + (uint32_t)op.r[2] * z + op.t[0];
    a.y = (uint32_t)op.r[3] * x + (uint32_t)op.r[4] * y + (uint32_t)op.r[5] * z + op.t[1];
    a.z = (uint32_t)op.r[6] * x + (uint32_t)op.r[7] * y + (uint32_t)op.r[8] * z + op.t[2];
    a.w = (uint32_t)t;
    atoms[i] = a;
  }
}

// The agreement 1 - Rwp of a structure against a fixed-profile pattern, from
// its FP64 intensities I (mult |F|^2 per reflection, all reflections): with
// y_calc = s I . P, the weighted chi^2 at the best scale is
// sum w y^2 - a^2 / b with a = v . I and b = I G I^T, G banded and symmetric
// (the diagonal plus twice the upper band).  Exact in FP64 and independent
// of the number of pattern points.  I is FP64 in the factored evaluation,
// FP32 in the cosine modes.
template <typename T>
__device__ __forceinline__ float profile_cc(const Params &P, const T *I, int lane) {
  const int K = P.profK, bw = P.profBw;
  double a = 0.0, b = 0.0;
  for (int k = lane; k < K; k += 32) {
    const double Ik = (double)I[k];
    a = fma(__ldg(P.profV + k), Ik, a);
    // the band's diagonals in two interleaved chains, so the loads and FMAs overlap
    const int dEnd = min(bw, K - 1 - k);
    double u0 = 0.0, u1 = 0.0;
    int d = 1;
#pragma unroll 4
    for (; d + 1 <= dEnd; d += 2) {
      u0 = fma(__ldg(P.profG + (size_t)d * K + k), (double)I[k + d], u0);
      u1 = fma(__ldg(P.profG + (size_t)(d + 1) * K + k), (double)I[k + d + 1], u1);
    }
    if (d <= dEnd) u0 = fma(__ldg(P.profG + (size_t)d * K + k), (double)I[k + d], u0);
    b = fma(Ik, fma(2.0, u0 + u1, __ldg(P.profG + k) * Ik), b);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  double chi = P.profSyy;
  if (a > 0.0 && b > 0.0) chi = fmax(P.profSyy - a * (a / b), 0.0);
  return 1.0f - (float)sqrt(chi / P.profSyy);
}

__device__ __forceinline__ float cc_of(const double sums[3]) {
  const double den = sums[0] * sums[1];
  if (!(den > 1e-20) || !(sums[2] > 0.0)) return 0.0f;
  double ex = fmin(1.0, fmax(0.0, sums[2] * sums[2] / den));
  double cc = 1.0 - sqrt(fmax(0.0, 1.0 - ex));
  return (float)fmin(1.0, fmax(0.0, cc));
}

// Squared nearest-image distance in the reduced basis (minimum-image shell 0).
__device__ __forceinline__ float dist2_near(const Params &P, uint4 a, uint4 b) {
  float q[3];
  frac_delta(P, a, b, q);
  float c[3];
  cart_vec(P, q, c);
  return c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
}

__device__ __forceinline__ float clash_term(const Params &P, float d, float dmin) {
  return P.penClash * (1.0f + 9.0f * ((dmin - d) / fmaxf(dmin, 1e-3f)));
}

// Clash penalty only (no distance rules): sum over pairs i < j.  With
// site-representative pairs (P.pairRange) the list holds (rep_s, j, m_s) for
// each site s and every other atom j: every image of a site has the same
// neighbours, so sum_{i<j} f(d_ij) = 1/2 sum_s m_s sum_{j != rep_s} f(d_{rep_s,j}).
// Otherwise small cells walk the balanced list of all pairs and large ones
// stripe j over the lanes.
__device__ __forceinline__ float clash_penalty(const Params &P, const uint4 *atoms, const float *rmin,
                                               const uint32_t *pairs, int nPairs, int lane) {
  float pen = 0.f;
  const int n = P.nTot, ne = P.nElem;
  if (pairs && P.pairRange) {
    for (int idx = lane; idx < nPairs; idx += 32) {
      const uint32_t e = pairs[idx];
      const uint4 ai = atoms[e & 0xFFF], aj = atoms[(e >> 12) & 0xFFF];
      const float dmin = rmin[ai.w * ne + aj.w];
      if (P.minImageShell) {
        const float d = cart_dist(P, ai, aj);
        if (d < dmin) pen += (0.5f * (float)(e >> 24)) * clash_term(P, d, dmin);
      } else {
        const float d2 = dist2_near(P, ai, aj);
        if (d2 < dmin * dmin) pen += (0.5f * (float)(e >> 24)) * clash_term(P, sqrtf(d2), dmin);
      }
    }
  } else if (pairs && P.minImageShell == 0) {
    for (int idx = lane; idx < nPairs; idx += 32) {
      const uint32_t pr = pairs[idx];
      const uint4 ai = atoms[pr & 0xFFFF], aj = atoms[pr >> 16];
      const float dmin = rmin[ai.w * ne + aj.w];
      const float d2 = dist2_near(P, ai, aj);
      if (d2 < dmin * dmin) pen += clash_term(P, sqrtf(d2), dmin);
    }
  } else {
    for (int i = 0; i < n - 1; ++i) {
      const uint4 ai = atoms[i];
      for (int j = i + 1 + lane; j < n; j += 32) {
        const uint4 aj = atoms[j];
        const float dmin = rmin[ai.w * ne + aj.w];
        const float d = P.minImageShell ? cart_dist(P, ai, aj) : sqrtf(dist2_near(P, ai, aj));
        if (d < dmin) pen += clash_term(P, d, dmin);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pen += __shfl_xor_sync(0xffffffffu, pen, o);
  return pen;
}

// Full penalty with distance rules (swarm_reflection.wgsl:913-1128), per-lane
// slot lists in local memory.  SLOTS is the compiled slot capacity.
template <int SLOTS>
__device__ float rule_penalty(const Params &P, const uint4 *atoms, const float *rmin, const float *shellLen,
                              int lane) {
  const int nRules = min(P.nRules, kMaxRules);
  int slotOff[kMaxRules], slotN[kMaxRules];
  int acc = 0;
  for (int k = 0; k < nRules; ++k) {
    slotOff[k] = acc;
    int nk = 0;
    if (P.rules[k].mode != 0) nk = min((int)P.rules[k].count, min(P.maxCoordSlots, SLOTS) - acc);
    nk = max(nk, 0);
    slotN[k] = nk;
    acc += nk;
  }
  const int slotTotal = acc;
  const bool shapes = P.geomSlots >= P.maxCoordSlots;
  float pen = 0.f;
  const int n = P.nTot, ne = P.nElem;
  for (int i = lane; i < n; i += 32) {
    const uint4 ai = atoms[i];
    const int ti = (int)ai.w;
    uint32_t myRules = 0;
    for (int k = 0; k < nRules; ++k)
      if (P.rules[k].a == ti) myRules |= 1u << k;
    float nearest[kMaxRules], inWindow[kMaxRules];
    for (int k = 0; k < kMaxRules; ++k) { nearest[k] = kNoNeighbour; inWindow[k] = 0.f; }
    float slot[SLOTS];
    float slotV[SLOTS][3];
    for (int m = 0; m < slotTotal; ++m) slot[m] = kNoNeighbour;
    for (int j = 0; j < n; ++j) {
      const uint4 aj = atoms[j];
      const int tj = (int)aj.w;
      const float d = cart_dist(P, ai, aj);
      if (j != i) {
        const float dmin = rmin[ti * ne + tj];
        if (j > i && d < dmin) pen += clash_term(P, d, dmin);
      }
      if (myRules == 0) continue;
      float qf[3];
      frac_delta(P, ai, aj, qf);
      const float dq = cart_len(P, qf);
      for (int k = 0; k < nRules; ++k) {
        if (!(myRules & (1u << k))) continue;
        const RuleDev &R = P.rules[k];
        if (R.b != tj) continue;
        const int nk = slotN[k];
        const bool counted = nk > 0;
        if (j != i) nearest[k] = fminf(nearest[k], d);
        float cutoff = R.dmax;
        if (counted) cutoff = fmaxf(cutoff, slot[slotOff[k] + nk - 1]);
        const int S = P.countShell;
        for (int sa = -S; sa <= S; ++sa)
          for (int sb = -S; sb <= S; ++sb)
            for (int sc = -S; sc <= S; ++sc) {
              const int si = (sa + 1) * 9 + (sb + 1) * 3 + (sc + 1);
              if (S == 1 && shellLen[si] - dq > cutoff) continue;
              const float t[3] = {qf[0] + sa, qf[1] + sb, qf[2] + sc};
              float dv[3];
              cart_vec(P, t, dv);
              const float dd = sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
              if (dd < 1.0e-4f && j == i) continue;
              if (dd >= R.dmin && dd <= R.dmax) inWindow[k] += 1.0f;
              if (counted) {
                const int lo = slotOff[k], hi = lo + nk;
                const bool shaped = shapes && R.geom != 0;
                if (dd < slot[hi - 1]) {
                  int m = hi - 1;
                  while (m > lo && slot[m - 1] > dd) {
                    slot[m] = slot[m - 1];
                    if (shaped) { slotV[m][0] = slotV[m - 1][0]; slotV[m][1] = slotV[m - 1][1]; slotV[m][2] = slotV[m - 1][2]; }
                    --m;
                  }
                  slot[m] = dd;
                  if (shaped) { slotV[m][0] = dv[0]; slotV[m][1] = dv[1]; slotV[m][2] = dv[2]; }
                  cutoff = fmaxf(R.dmax, slot[hi - 1]);
                }
              }
            }
      }
    }
    for (int k = 0; k < nRules; ++k) {
      if (!(myRules & (1u << k))) continue;
      const RuleDev &R = P.rules[k];
      if (R.mode == 0) {
        const float nk = nearest[k];
        if (nk < kNoNeighbour && nk > R.dmax) pen += P.penBond * (nk - R.dmax);
      } else {
        const int nk = slotN[k];
        float deficit = 0.f;
        for (int m = 0; m < nk; ++m) {
          const float dm = slot[slotOff[k] + m];
          if (dm >= kNoNeighbour) deficit += kNoPartnerCharge;
          else {
            const float miss = fmaxf(0.f, dm - R.dmax) + fmaxf(0.f, R.dmin - dm);
            deficit += miss * (1.0f + miss / kCoordSoftA);
          }
        }
        pen += P.penBond * deficit;
        if (shapes && R.geom != 0 && nk >= 2) {
          const int lo = slotOff[k];
          float g = 0.f;
          for (int m = 0; m + 1 < nk; ++m) {
            const float dm = slot[lo + m];
            if (dm >= kNoNeighbour) continue;
            for (int q = m + 1; q < nk; ++q) {
              const float dn = slot[lo + q];
              if (dn >= kNoNeighbour) continue;
              const float c = (slotV[lo + m][0] * slotV[lo + q][0] + slotV[lo + m][1] * slotV[lo + q][1] +
                               slotV[lo + m][2] * slotV[lo + q][2]) / fmaxf(dm * dn, 1e-6f);
              const float e = geom_cos_error(R.geom, c);
              g += e * e;
            }
          }
          pen += P.penBond * P.penGeom * g;
        }
        if (R.mode == 1) pen += P.penCoord * fmaxf(0.f, inWindow[k] - R.count);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pen += __shfl_xor_sync(0xffffffffu, pen, o);
  return pen;
}

template <int SLOTS>
__device__ __forceinline__ float penalty(const Params &P, const uint4 *atoms, const float *rmin,
                                         const float *shellLen, const uint32_t *pairs, int nPairs, int lane) {
  if (SLOTS == 0) return clash_penalty(P, atoms, rmin, pairs, nPairs, lane);
  return rule_penalty<(SLOTS > 0 ? SLOTS : 1)>(P, atoms, rmin, shellLen, lane);
}

// Proposal into ws.prop.  Every lane draws one Philox block in lock-step:
// lanes < maxSites turn theirs into three normal deviates for their site; the
// move choice and the Metropolis deviate come from the block of lane 31
// (a lane no site uses when maxSites <= 31), or from a second block.
// ---------------------------------------------------------------------------
// Polyhedron moves (swarm_reflection.wgsl:425-576).  A counted rule is picked
// uniformly, then a centre (an independent site of the rule's first element)
// uniformly, then the centre's nn nearest partners: every image of every
// other site of the rule's second element, nearest image.  One of three moves
// follows with probability 1/3 each: translate the centre and its partners by
// one fractional Gaussian step, rotate the shell about the centre, or snap
// the shell to one distance (the rule's ideal shape, aligned on the two
// partners that fit it best, when the rule has one).  Each moved partner site
// is the preimage, under the operator that made its image, of the image's new
// position.  Lane 0 only, with a Philox stream of its own; the new positions
// (before projection onto the Wyckoff subspaces) go to ws.prop in fixed point
// and the mask of moved sites is returned (0: no move applies).
// ---------------------------------------------------------------------------
constexpr int kMaxPoly = 12;

struct PolyRng {
  uint2 key;
  uint32_t g, p, blk;
  uint4 buf;
  int pos;
  __device__ uint32_t word() {
    if (pos == 4) {
      buf = philox4x32_10(make_uint4(g, p, 0x7000u + blk, 6u), key);
      ++blk;
      pos = 0;
    }
    const uint32_t w = pos == 0 ? buf.x : pos == 1 ? buf.y : pos == 2 ? buf.z : buf.w;
    ++pos;
    return w;
  }
  __device__ float uniform() { return u01(word()); }
  __device__ float gaussian() {
    const uint32_t a = word(), b = word();
    return sqrtf(-2.0f * __logf(u01_open(a))) * __cosf(6.28318530717958647f * u01(b));
  }
};

// Ideal directions of the shapes (rule geometry codes 1-5): linear,
// trigonal planar, tetrahedral, square planar, octahedral.
__device__ __forceinline__ int shape_count(int code) {
  switch (code) {
    case 1: return 2;
    case 2: return 3;
    case 3: case 4: return 4;
    case 5: return 6;
    default: return 0;
  }
}
__device__ __forceinline__ void shape_vertex(int code, int k, float v[3]) {
  const float s3 = 0.57735026918962576f, h3 = 0.86602540378443865f;
  float x = 0, y = 0, z = 0;
  switch (code) {
    case 1: x = k == 0 ? 1.f : -1.f; break;
    case 2:
      if (k == 0) x = 1.f;
      else { x = -0.5f; y = k == 1 ? h3 : -h3; }
      break;
    case 3: {
      const float sx[4] = {1, 1, -1, -1}, sy[4] = {1, -1, 1, -1}, sz[4] = {1, -1, -1, 1};
      x = s3 * sx[k]; y = s3 * sy[k]; z = s3 * sz[k];
      break;
    }
    case 4: {
      const float cx[4] = {1, 0, -1, 0}, cy[4] = {0, 1, 0, -1};
      x = cx[k]; y = cy[k];
      break;
    }
    default: {
      const float cx[6] = {1, 0, -1, 0, 0, 0}, cy[6] = {0, 1, 0, -1, 0, 0}, cz[6] = {0, 0, 0, 0, 1, -1};
      x = cx[k]; y = cy[k]; z = cz[k];
    }
  }
  v[0] = x; v[1] = y; v[2] = z;
}
__device__ __forceinline__ float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
// Orthonormal frame (columns F[.][c]): e1 along a, e2 in the plane of a and b, e3 = e1 x e2.
__device__ void frame_of(const float a[3], const float b[3], float F[3][3]) {
  float e1[3], pv[3], e2[3];
  const float la = rsqrtf(fmaxf(dot3(a, a), 1e-30f));
  for (int i = 0; i < 3; ++i) e1[i] = a[i] * la;
  const float bd = dot3(b, e1);
  for (int i = 0; i < 3; ++i) pv[i] = b[i] - bd * e1[i];
  if (sqrtf(dot3(pv, pv)) < 1e-4f) {   // b along a: any perpendicular
    float hv[3] = {0, 0, 0};
    hv[fabsf(e1[0]) > 0.9f ? 1 : 0] = 1.f;
    const float hd = dot3(hv, e1);
    for (int i = 0; i < 3; ++i) pv[i] = hv[i] - hd * e1[i];
  }
  const float lp = rsqrtf(fmaxf(dot3(pv, pv), 1e-30f));
  for (int i = 0; i < 3; ++i) e2[i] = pv[i] * lp;
  const float e3[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  for (int i = 0; i < 3; ++i) { F[i][0] = e1[i]; F[i][1] = e2[i]; F[i][2] = e3[i]; }
}
// The ideal vertex e carried from the ideal frame Fi into the actual frame Fa.
__device__ __forceinline__ void carry(const float Fa[3][3], const float Fi[3][3], const float e[3], float w[3]) {
  const float c0 = Fi[0][0] * e[0] + Fi[1][0] * e[1] + Fi[2][0] * e[2];
  const float c1 = Fi[0][1] * e[0] + Fi[1][1] * e[1] + Fi[2][1] * e[2];
  const float c2 = Fi[0][2] * e[0] + Fi[1][2] * e[1] + Fi[2][2] * e[2];
  for (int i = 0; i < 3; ++i) w[i] = Fa[i][0] * c0 + Fa[i][1] * c1 + Fa[i][2] * c2;
}
__device__ __forceinline__ uint32_t frac_to_fixed(float v) {
  const double f = (double)v - floor((double)v);
  double x = floor(f * 4294967296.0 + 0.5);
  if (x >= 4294967296.0) x -= 4294967296.0;
  return (uint32_t)(unsigned long long)x;
}

__device__ __noinline__ uint32_t poly_propose(const Params &P, WarpView &ws, const OpFix *ops, float sd, PolyRng &rng) {
  const int nRules = min(P.nRules, kMaxRules);
  int nCounted = 0, k = 0;
  for (int r = 0; r < nRules; ++r)
    if (P.rules[r].mode != 0) {
      ++nCounted;
      if (rng.uniform() < 1.0f / (float)nCounted) k = r;
    }
  if (nCounted == 0) return 0u;
  const RuleDev R = P.rules[k];
  const int ta = R.a, tb = R.b, geom = R.geom;
  const float rMin = fmaxf(R.dmin, 0.f), rMax = R.dmax;
  const int nn = min((int)R.count, kMaxPoly);
  const int ms = P.maxSites, A = ws.meta[0];
  const uint32_t *gen = P.genOrig + (size_t)A * P.nTot;
  // the centre
  int nCentre = 0, sc = ms;
  uint32_t seen = 0;
  for (int g = 0; g < P.nTot; ++g) {
    const uint32_t w = __ldg(gen + g);
    const int s = w & 0xFF;
    if (s >= ms || (int)((w >> 20) & 0xF) != ta || ((seen >> s) & 1u)) continue;
    seen |= 1u << s;
    ++nCentre;
    if (rng.uniform() < 1.0f / (float)nCentre) sc = s;
  }
  if (sc >= ms || nn == 0) return 0u;
  const uint4 cF = make_uint4(ws.cur[sc * 3], ws.cur[sc * 3 + 1], ws.cur[sc * 3 + 2], 0u);
  // its nn nearest partners
  float ld[kMaxPoly], lv[kMaxPoly][3];
  int ls[kMaxPoly], lo[kMaxPoly];
  for (int m = 0; m < kMaxPoly; ++m) ld[m] = kNoNeighbour;
  for (int g = 0; g < P.nTot; ++g) {
    const uint32_t w = __ldg(gen + g);
    const int s = w & 0xFF;
    if (s >= ms || s == sc || (int)((w >> 20) & 0xF) != tb) continue;
    const int o = (w >> 8) & 0xFFF;
    const OpFix &op = ops[o];
    const uint32_t x = ws.cur[s * 3], y = ws.cur[s * 3 + 1], z = ws.cur[s * 3 + 2];
    uint4 img;
    img.x = (uint32_t)op.r[0] * x + (uint32_t)op.r[1] * y + (uint32_t)op.r[2] * z + op.t[0];
    img.y = (uint32_t)op.r[3] * x + (uint32_t)op.r[4] * y + (uint32_t)op.r[5] * z + op.t[1];
    img.z = (uint32_t)op.r[6] * x + (uint32_t)op.r[7] * y + (uint32_t)op.r[8] * z + op.t[2];
    img.w = 0;
    float q[3], dv[3];
    frac_delta(P, img, cF, q);
    cart_vec(P, q, dv);
    const float d = sqrtf(dot3(dv, dv));
    if (d < 1e-4f || d >= ld[nn - 1]) continue;
    int m = nn - 1;
    while (m > 0 && ld[m - 1] > d) {
      ld[m] = ld[m - 1];
      lv[m][0] = lv[m - 1][0]; lv[m][1] = lv[m - 1][1]; lv[m][2] = lv[m - 1][2];
      ls[m] = ls[m - 1];
      lo[m] = lo[m - 1];
      --m;
    }
    ld[m] = d;
    lv[m][0] = dv[0]; lv[m][1] = dv[1]; lv[m][2] = dv[2];
    ls[m] = s;
    lo[m] = o;
  }
  int nf = 0;
  for (int m = 0; m < nn; ++m)
    if (ld[m] < kNoNeighbour) ++nf;
  if (nf == 0) return 0u;

  const float kind = rng.uniform();
  float shift[3] = {0, 0, 0};
  float nv[kMaxPoly][3];
  for (int m = 0; m < nf; ++m) { nv[m][0] = lv[m][0]; nv[m][1] = lv[m][1]; nv[m][2] = lv[m][2]; }
  if (kind < 0.3333333f) {
    // translate: one fractional step for the whole unit
    for (int i = 0; i < 3; ++i) shift[i] = rng.gaussian() * sd;
  } else if (kind < 0.6666667f) {
    // rotate the shell about its centre (Rodrigues)
    float ax[3] = {rng.gaussian(), rng.gaussian(), rng.gaussian()};
    const float la = sqrtf(dot3(ax, ax));
    if (la < 1e-6f) { ax[0] = 0; ax[1] = 0; ax[2] = 1; }
    else for (int i = 0; i < 3; ++i) ax[i] /= la;
    const float ang = rng.gaussian() * fminf(fmaxf(sd * 20.0f, 0.05f), 0.8f);
    const float c = cosf(ang), sn = sinf(ang);
    for (int m = 0; m < nf; ++m) {
      const float *v = lv[m];
      const float kv = dot3(ax, v);
      const float cr[3] = {ax[1] * v[2] - ax[2] * v[1], ax[2] * v[0] - ax[0] * v[2], ax[0] * v[1] - ax[1] * v[0]};
      for (int i = 0; i < 3; ++i) nv[m][i] = v[i] * c + cr[i] * sn + ax[i] * kv * (1.0f - c);
    }
  } else {
    // snap: one distance for the shell, and the ideal shape when the rule has one
    float mean = 0;
    for (int m = 0; m < nf; ++m) mean += ld[m];
    mean = mean / (float)nf * (1.0f + 0.03f * rng.gaussian());
    const float dT = fminf(fmaxf(mean, fmaxf(rMin, 0.3f)), rMax < 1.0e6f ? rMax : mean);
    const int nShape = shape_count(geom);
    if (nShape >= 2 && nf >= 2) {
      float u0[3] = {lv[0][0] / ld[0], lv[0][1] / ld[0], lv[0][2] / ld[0]};
      float v0[3], v1[3];
      shape_vertex(geom, 0, v0);
      shape_vertex(geom, 1, v1);
      const float cIdeal = dot3(v0, v1);
      int j1 = 1;
      float bestErr = 1.0e9f;
      for (int m = 1; m < nf; ++m) {
        const float um[3] = {lv[m][0] / ld[m], lv[m][1] / ld[m], lv[m][2] / ld[m]};
        const float e = fabsf(dot3(u0, um) - cIdeal);
        if (e < bestErr) { bestErr = e; j1 = m; }
      }
      float Fa[3][3], Fi[3][3];
      frame_of(u0, lv[j1], Fa);
      frame_of(v0, v1, Fi);
      uint32_t usedV = 3u;
      for (int m = 0; m < nf; ++m) {
        int vk;
        if (m == 0) vk = 0;
        else if (m == j1) vk = 1;
        else {
          float bestDot = -2.0f;
          vk = nShape;
          const float um[3] = {lv[m][0] / ld[m], lv[m][1] / ld[m], lv[m][2] / ld[m]};
          for (int qv = 2; qv < nShape; ++qv) {
            if ((usedV >> qv) & 1u) continue;
            float e[3], wv[3];
            shape_vertex(geom, qv, e);
            carry(Fa, Fi, e, wv);
            const float dd = dot3(wv, um);
            if (dd > bestDot) { bestDot = dd; vk = qv; }
          }
          if (vk < nShape) usedV |= 1u << vk;
        }
        if (vk < nShape) {
          float e[3], wv[3];
          shape_vertex(geom, vk, e);
          carry(Fa, Fi, e, wv);
          for (int i = 0; i < 3; ++i) nv[m][i] = wv[i] * dT;
        } else {
          for (int i = 0; i < 3; ++i) nv[m][i] = lv[m][i] / ld[m] * dT;
        }
      }
    } else {
      for (int m = 0; m < nf; ++m)
        for (int i = 0; i < 3; ++i) nv[m][i] = lv[m][i] / ld[m] * dT;
    }
  }

  // back to the independent sites: the nearest image of each site carries it
  const float cf[3] = {(float)((double)cF.x * (1.0 / 4294967296.0)), (float)((double)cF.y * (1.0 / 4294967296.0)),
                       (float)((double)cF.z * (1.0 / 4294967296.0))};
  uint32_t mask = 0;
  if (kind < 0.3333333f) {
    for (int i = 0; i < 3; ++i) ws.prop[sc * 3 + i] = frac_to_fixed(cf[i] + shift[i]);
    mask = 1u << sc;
  }
  for (int m = 0; m < nf; ++m) {
    const int s = ls[m];
    if ((mask >> s) & 1u) continue;
    float dest[3];
    for (int i = 0; i < 3; ++i)
      dest[i] = cf[i] + (P.invOrth[3 * i] * nv[m][0] + P.invOrth[3 * i + 1] * nv[m][1] + P.invOrth[3 * i + 2] * nv[m][2]) +
                shift[i];
    // R^-1 (dest - t) by the adjugate
    const OpFix &op = ops[lo[m]];
    const float m0 = op.r[0], m1 = op.r[1], m2 = op.r[2], m3 = op.r[3], m4 = op.r[4], m5 = op.r[5], m6 = op.r[6],
                m7 = op.r[7], m8 = op.r[8];
    const float c00 = m4 * m8 - m5 * m7, c01 = m5 * m6 - m3 * m8, c02 = m3 * m7 - m4 * m6;
    const float det = m0 * c00 + m1 * c01 + m2 * c02;
    const float dn = fabsf(det) < 1e-6f ? 1.0f : det;
    float wv[3];
    for (int i = 0; i < 3; ++i) wv[i] = (dest[i] - (float)((double)op.t[i] * (1.0 / 4294967296.0))) / dn;
    const float out[3] = {c00 * wv[0] + (m2 * m7 - m1 * m8) * wv[1] + (m1 * m5 - m2 * m4) * wv[2],
                          c01 * wv[0] + (m0 * m8 - m2 * m6) * wv[1] + (m2 * m3 - m0 * m5) * wv[2],
                          c02 * wv[0] + (m1 * m6 - m0 * m7) * wv[1] + (m0 * m4 - m1 * m3) * wv[2]};
    for (int i = 0; i < 3; ++i) ws.prop[s * 3 + i] = frac_to_fixed(out[i]);
    mask |= 1u << s;
  }
  return mask;
}

// SLOTS > 0: the distance-rule variants, the only ones whose problems can
// have counted rules and so polyhedron moves.
// Fragment parameters -> fixed-point site coordinates (lane i: atom i).
// The torsions are applied from the reference geometry outward in their
// order, each about its bond as the earlier torsions left it (forward
// kinematics; the axis atoms are read from their lanes), then the rotation of
// the unit quaternion q = (w, x, y, z), then Cartesian -> fractional plus the
// translation.  prm: t[3], q[4], torsion angles.
__device__ __noinline__ void frag_atoms(const FragDev &F, const float *prm, uint32_t *out, int lane) {
  const bool mine = lane < F.nAtoms;
  float x = mine ? F.ref[3 * lane] : 0.f, y = mine ? F.ref[3 * lane + 1] : 0.f, z = mine ? F.ref[3 * lane + 2] : 0.f;
  for (int t = 0; t < F.nTors; ++t) {
    const int b = F.axisB[t], c = F.axisC[t];
    const float bx = __shfl_sync(0xffffffffu, x, b), by = __shfl_sync(0xffffffffu, y, b),
                bz = __shfl_sync(0xffffffffu, z, b);
    const float cx = __shfl_sync(0xffffffffu, x, c), cy = __shfl_sync(0xffffffffu, y, c),
                cz = __shfl_sync(0xffffffffu, z, c);
    if ((F.moving[t] >> lane) & 1u) {
      float ux = cx - bx, uy = cy - by, uz = cz - bz;
      const float inv = rsqrtf(ux * ux + uy * uy + uz * uz);
      ux *= inv; uy *= inv; uz *= inv;
      float sn, cs;
      sincosf(prm[7 + t], &sn, &cs);
      // Rodrigues: v' = v cos + (u x v) sin + u (u.v)(1 - cos), v about b
      const float vx = x - bx, vy = y - by, vz = z - bz;
      const float d = ux * vx + uy * vy + uz * vz;
      const float wx = uy * vz - uz * vy, wy = uz * vx - ux * vz, wz = ux * vy - uy * vx;
      x = bx + vx * cs + wx * sn + ux * d * (1.f - cs);
      y = by + vy * cs + wy * sn + uy * d * (1.f - cs);
      z = bz + vz * cs + wz * sn + uz * d * (1.f - cs);
    }
  }
  if (!mine) return;
  const float qw = prm[3], qx = prm[4], qy = prm[5], qz = prm[6];
  const float r00 = 1.f - 2.f * (qy * qy + qz * qz), r01 = 2.f * (qx * qy - qw * qz), r02 = 2.f * (qx * qz + qw * qy);
  const float r10 = 2.f * (qx * qy + qw * qz), r11 = 1.f - 2.f * (qx * qx + qz * qz), r12 = 2.f * (qy * qz - qw * qx);
  const float r20 = 2.f * (qx * qz - qw * qy), r21 = 2.f * (qy * qz + qw * qx), r22 = 1.f - 2.f * (qx * qx + qy * qy);
  const float X = r00 * x + r01 * y + r02 * z, Y = r10 * x + r11 * y + r12 * z, Z = r20 * x + r21 * y + r22 * z;
  const float *T = F.toFrac;
  out[3 * lane] = frac_to_fixed(T[0] * X + T[1] * Y + T[2] * Z + prm[0]);
  out[3 * lane + 1] = frac_to_fixed(T[3] * X + T[4] * Y + T[5] * Z + prm[1]);
  out[3 * lane + 2] = frac_to_fixed(T[6] * X + T[7] * Y + T[8] * Z + prm[2]);
}

// A fragment proposal: with probability 1/4 every parameter moves, otherwise
// one group -- the translation, the orientation or one torsion -- chosen
// uniformly.  Gaussian steps of the replica's width sd: translation sd x
// transStep per axis, orientation a turn of sd x angleStep about a random
// axis, torsion sd x angleStep.  Lane 0 draws (Philox, its own counters) and
// writes the proposed parameters; every lane then maps them to coordinates.
__device__ __noinline__ void frag_propose(const Params &P, float *fcur, float *fprop, uint32_t *prop, int g, int p,
                                          int lane, float sd, uint2 key, float *uMetro) {
  const FragDev &F = *P.frag;
  if (lane == 0) {
    const uint4 a = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xF7A60000u, 1u), key);
    const uint4 b = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xF7A60000u, 2u), key);
    const uint4 c = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xF7A60000u, 3u), key);
    for (int k = 0; k < kFragParams; ++k) fprop[k] = fcur[k];
    const bool all = u01(a.x) < 0.25f;
    const int pick = min(1 + F.nTors, (int)(u01(a.y) * (float)(2 + F.nTors)));
    const float2 n0 = gauss2(b.x, b.y), n1 = gauss2(b.z, b.w), n2 = gauss2(c.x, c.y), n3 = gauss2(c.z, c.w);
    if (all || pick == 0) {
      fprop[0] += n0.x * sd * F.transStep;
      fprop[1] += n0.y * sd * F.transStep;
      fprop[2] += n1.x * sd * F.transStep;
      for (int k = 0; k < 3; ++k) fprop[k] -= floorf(fprop[k]);
    }
    if (all || pick == 1) {
      float ax = n1.y, ay = n2.x, az = n2.y;
      const float nn = rsqrtf(fmaxf(ax * ax + ay * ay + az * az, 1e-20f));
      ax *= nn; ay *= nn; az *= nn;
      float sn, cs;
      sincosf(0.5f * n3.x * sd * F.angleStep, &sn, &cs);
      const float dw = cs, dx = ax * sn, dy = ay * sn, dz = az * sn;
      const float qw = fcur[3], qx = fcur[4], qy = fcur[5], qz = fcur[6];
      float w = dw * qw - dx * qx - dy * qy - dz * qz, x = dw * qx + dx * qw + dy * qz - dz * qy,
            y = dw * qy - dx * qz + dy * qw + dz * qx, z = dw * qz + dx * qy - dy * qx + dz * qw;
      const float qn = rsqrtf(w * w + x * x + y * y + z * z);
      fprop[3] = w * qn; fprop[4] = x * qn; fprop[5] = y * qn; fprop[6] = z * qn;
    }
    for (int t = 0; t < F.nTors; ++t)
      if (all || pick == 2 + t) {
        const uint4 d = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xF7A60000u, 4u + (uint32_t)t), key);
        float v = fprop[7 + t] + gauss2(d.x, d.y).x * sd * F.angleStep;
        v -= 6.28318530717958647f * floorf(v * 0.159154943091895336f + 0.5f);   // into [-pi, pi)
        fprop[7 + t] = v;
      }
    *uMetro = u01(a.z);
  }
  *uMetro = __shfl_sync(0xffffffffu, *uMetro, 0);
  __syncwarp();
  frag_atoms(F, fprop, prop, lane);
  __syncwarp();
}

template <int SLOTS>
__device__ __forceinline__ void propose(const Params &P, WarpView &ws, const ProjFix *proj, const OpFix *ops, int g,
                                        int p, int lane, float sd, uint32_t seed, float *uMetro) {
  const uint2 key = make_uint2(seed, P.runKey);
  if (P.frag) {
    float *fp = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(ws.meta) + P.fragOff);
    frag_propose(P, fp, fp + kFragParams, ws.prop, g, p, lane, sd, key, uMetro);
    return;
  }
  uint32_t polyMask = 0;
  if (SLOTS > 0 && P.polyProb > 0.f) {
    if (lane == 0) {
      PolyRng rng{key, (uint32_t)g, (uint32_t)p, 0u, make_uint4(0, 0, 0, 0), 4};
      if (rng.uniform() < P.polyProb) polyMask = poly_propose(P, ws, ops, sd, rng);
    }
    polyMask = __shfl_sync(0xffffffffu, polyMask, 0);
    __syncwarp();
  }
  const uint4 c = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, (uint32_t)lane, 2u), key);
  uint4 cc = make_uint4(__shfl_sync(0xffffffffu, c.x, 31), __shfl_sync(0xffffffffu, c.y, 31),
                        __shfl_sync(0xffffffffu, c.z, 31), __shfl_sync(0xffffffffu, c.w, 31));
  if (P.maxSites >= 32) cc = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xFFFFu, 1u), key);
  const uint32_t free = (uint32_t)ws.meta[4];
  const int nFree = __popc(free);
  int pick = -1;
  if (!polyMask && u01(cc.x) < 0.75f && nFree > 0) {
    const int kth = min(nFree - 1, (int)(u01(cc.y) * (float)nFree));
    pick = __fns(free, 0, kth + 1);
  }
  *uMetro = u01(cc.z);
  if (lane < P.maxSites) {
    const int s = lane;
    const bool moving = polyMask ? ((polyMask >> s) & 1u) != 0 : (pick < 0) || (pick == s);
    if (moving) {
      const float2 n01 = gauss2(c.x, c.y);
      const float2 n23 = gauss2(c.z, c.w);
      const float gz[3] = {n01.x, n01.y, n23.x};
      const float scale = sd * 4294967296.0f;
      int64_t pos[3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
        pos[i] = polyMask ? (int64_t)ws.prop[s * 3 + i] : (int64_t)ws.cur[s * 3 + i] + __float2ll_rn(gz[i] * scale);
      const ProjFix &pr = proj[s];
      if (pr.pad[0]) {  // diagonal 0/1 projector: keep or drop each coordinate
#pragma unroll
        for (int i = 0; i < 3; ++i)
          ws.prop[s * 3 + i] = (pr.num[4 * i] ? (uint32_t)pos[i] : 0u) + pr.t[i];
      } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          int64_t acc = (int64_t)pr.num[3 * i] * pos[0] + (int64_t)pr.num[3 * i + 1] * pos[1] +
                        (int64_t)pr.num[3 * i + 2] * pos[2];
          if (pr.den != 1) acc = floor_div(acc, pr.den);
          ws.prop[s * 3 + i] = (uint32_t)(acc + (int64_t)pr.t[i]);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i) ws.prop[s * 3 + i] = ws.cur[s * 3 + i];
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
// A ladder held by RANKS CTAs of one thread-block cluster (RANKS = 2: four
// rungs each, so 512 ladders become 1024 CTAs that spread evenly over 148
// SMs).  The exchange energies live in rank 0's shared memory and a swap
// across the two CTAs moves coordinates through distributed shared memory;
// with RANKS = 1 these are the CTA's own arrays and the syncs are
// __syncthreads.
template <int RANKS>
__device__ __forceinline__ void ladder_sync() {
  if constexpr (RANKS > 1)
    cooperative_groups::this_cluster().sync();
  else
    __syncthreads();
}
template <int RANKS, class T>
__device__ __forceinline__ T *ladder_peer(T *p, int rank) {
  if constexpr (RANKS > 1)
    return cooperative_groups::this_cluster().map_shared_rank(p, rank);
  else
    return p;
}

// One CTA's share of a search: ladders L0, L0 + Lstep, ... of the problem P,
// generations [gen0, gen0 + nGen).  Returns false (on every thread) when the
// static tables could not be staged in time.
// GT = 1: the static tables are read from global memory (too large to stage);
// a template parameter so that the staged path keeps shared-memory loads.
template <int COSMODE, int SLOTS, int INCR, int RANKS = 1, int GT = 0>
__device__ __forceinline__ bool wy_cta(const Params &P, int L0, int Lstep, int gen0, int nGen, int mcmc,
                                       int swapEvery, int reevalFirst) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t stageBar;
  __shared__ float shellLen[27];
  __shared__ float exFit[kMaxRungs], exCC[kMaxRungs], exPen[kMaxRungs], exTemp[kMaxRungs], exE[kMaxRungs];
  __shared__ int exSwap[kMaxRungs];
  __shared__ int stagedFlag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nWarps = blockDim.x >> 5;
  const int rank = RANKS > 1 ? (int)cooperative_groups::this_cluster().block_rank() : 0;
  const int rung = warp + rank * nWarps;   // this warp's rung of the ladder

  // Stage the static tables once per CTA with the bulk-copy engine, unless
  // they are too large to share the CTA's shared memory with the replica
  // slices: then every table read goes to global memory (through L1).
  constexpr bool stage = GT == 0;
  const unsigned char *stat = GT ? P.blob : smem;
  const int blobPad = stage ? (P.blobBytes + 127) & ~127 : 0;
  if (stage && threadIdx.x == 0) {
    mbar_init(&stageBar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (stage && threadIdx.x == 0) {
    mbar_arrive_expect_tx(&stageBar, (uint32_t)P.blobBytes);
    for (int off = 0; off < P.blobBytes; off += 65536) {
      const int n = min(65536, P.blobBytes - off);
      bulk_g2s(smem + off, P.blob + off, (uint32_t)n, &stageBar);
    }
  }
  if (threadIdx.x < 27) {
    const float t[3] = {(float)((int)threadIdx.x / 9 - 1), (float)(((int)threadIdx.x / 3) % 3 - 1),
                        (float)((int)threadIdx.x % 3 - 1)};
    shellLen[threadIdx.x] = cart_len(P, t);
  }
  bool staged = !stage || __syncthreads_and(mbar_wait_bounded(&stageBar, 0, kStageWaitLimit) ? 1 : 0) != 0;
  if (!stage) __syncthreads();
  if constexpr (RANKS > 1) {
    // both CTAs of the ladder go on, or both return
    if (threadIdx.x == 0) stagedFlag = staged ? 1 : 0;
    ladder_sync<RANKS>();
    staged = staged && *ladder_peer<RANKS>(&stagedFlag, rank ^ 1) != 0;
    ladder_sync<RANKS>();
  }
  if (!staged) {
    if (threadIdx.x == 0) raise_flag(P.errFlag, DEV_STAGE_TIMEOUT);
    mbar_wait_bounded(&stageBar, 0, kStageWaitLimit);   // copies still in flight land before the CTA moves on
    return false;
  }
  const ReflRec *refl = reinterpret_cast<const ReflRec *>(stat + P.offRefl);
  const float *ftab = reinterpret_cast<const float *>(stat + P.offF);
  const float4 *groups = reinterpret_cast<const float4 *>(stat + P.offGroup);
  const float *rmin = reinterpret_cast<const float *>(stat + P.offRmin);
  const double *sooPrefix = reinterpret_cast<const double *>(stat + P.offSoo);
  const OpFix *ops = reinterpret_cast<const OpFix *>(stat + P.offOps);
  const uint32_t *pairs =
      (P.nPairs > 0 || P.pairRange) ? reinterpret_cast<const uint32_t *>(stat + P.offPairs) : nullptr;

  unsigned char *wbase = smem + blobPad + (size_t)warp * P.warpSmemBytes;
  WarpView ws = warp_view(wbase, P);
  uint4 *atoms = reinterpret_cast<uint4 *>(wbase + P.atomsOff);
  float *ic = reinterpret_cast<float *>(wbase + P.icOff);
  uint32_t *gen = reinterpret_cast<uint32_t *>(wbase + P.genOff);
  ProjFix *proj = reinterpret_cast<ProjFix *>(wbase + P.projOff);

  const int rungs = P.rungs;
  const int nLadders = P.nLadders;
  const size_t curStride = (size_t)P.maxSites * 3;
  uint32_t *bestBase = P.pos + (size_t)P.numParticles * curStride;

  float *Cb = INCR ? reinterpret_cast<float *>(wbase + P.cbOff) : nullptr;
  double *ftabs = COSMODE == 2 ? reinterpret_cast<double *>(wbase + P.tabOff) : nullptr;
  uint4 *ftags = COSMODE == 2 ? reinterpret_cast<uint4 *>(wbase + P.tagOff) : nullptr;
  double *ic64 = reinterpret_cast<double *>(wbase + P.icOff);
  float *fcurW = reinterpret_cast<float *>(wbase + P.fragOff);   // fragment parameters: current, then proposed
  uint4 *atomsB[2] = {atoms, INCR ? reinterpret_cast<uint4 *>(wbase + P.atoms2Off) : atoms};

  for (int L = L0; L < nLadders; L += Lstep) {
    int p = -1;
    if (rung < rungs) {
      if (P.ladders)
        p = P.ladders[(size_t)L * rungs + rung];
      else {
        const int q = L * rungs + rung;
        p = q < P.numParticles ? q : -1;
      }
    }
    const bool active = p >= 0;
    const uint32_t *myPairs = pairs;
    int myNPairs = P.nPairs;
    // chain state in registers (meaningful on lane 0)
    float fit = 0.f, cc0 = 0.f, pen0 = 0.f, step = 0.f, temp = 0.f, bestFit = -1e30f, bestCC = 0.f, bestPen = 0.f;
    uint32_t seed = 0, accepted = 0;
    if (active) {
      const int A = (int)P.assign[p];
      if (pairs && P.pairRange) {
        const int2 pr = P.pairRange[A];
        myPairs = pairs + pr.x;
        myNPairs = pr.y;
      }
      if (lane == 0) {
        ws.meta[0] = A;
        ws.meta[1] = P.nRuns[A];
        ws.meta[2] = P.nF[A];
        ws.meta[4] = (int)P.freeMask[A];
        ws.meta[5] = p;
        const PState st = P.st[p];
        fit = st.fit; cc0 = st.cc; pen0 = st.pen; step = st.step; temp = st.temp;
        seed = st.seed; accepted = st.accepted;
        bestFit = st.bestFit; bestCC = st.bestCC; bestPen = st.bestPen;
      }
      seed = __shfl_sync(0xffffffffu, seed, 0);
      if (lane < P.maxSites) ws.runs[lane] = P.runs[(size_t)A * kMaxSites + lane];
      if (INCR) for (int j = lane; j <= P.maxSites; j += 32) ws.slot[j] = j;
      for (int j = lane; j < (int)curStride; j += 32) ws.cur[j] = P.pos[(size_t)p * curStride + j];
      for (int j = lane; j < P.nTot; j += 32) gen[j] = __ldg(P.gen + (size_t)A * P.nTot + j);
      for (int j = lane; j < P.maxSites; j += 32) proj[j] = P.proj[(size_t)A * P.maxSites + j];
      if constexpr (COSMODE == 2)
        for (int j = lane; j < 2 * P.maxSites; j += 32) ftags[j] = make_uint4(0u, 0u, 0u, 0u);
      if (P.frag && lane < kFragParams) fcurW[lane] = P.fragState[(size_t)p * kFragParams + lane];
    }
    __syncwarp();
    const uint32_t allSites = P.maxSites >= 32 ? 0xffffffffu : ((1u << P.maxSites) - 1u);
    int prevNga = -1;
    int cachedAct = -1;       // reflections the site sums cover; -1: none
    int cb = 0;               // atom bank holding the current cell
    for (int gi = 0; gi < nGen; ++gi) {
      const int g = gen0 + gi;
      const int nga = P.schedGroups ? P.schedGroups[g] : P.ngaArg;
      const float penScale = P.schedGroups ? P.schedPen[g] : P.penArg;
      // the Gram-form profile fitness needs every reflection: no resolution ramp
      const int ngaC = P.profV ? P.nGroups : max(0, min(nga, P.nGroups));
      if (active) {
        float *tIc = P.traceIc ? P.traceIc + (size_t)p * P.nRefl : nullptr;
        const bool reeval = mcmc && ((gi == 0 && reevalFirst) || (gi > 0 && nga != prevNga));
        if constexpr (INCR) {
          const int nAct = nrefl_active(groups, ngaC);
          if (cachedAct != nAct) {
            // (re)fill the site sums of the current cell for the active reflections
            expand(P, gen, ops, ws.cur, atomsB[cb], lane);
            __syncwarp();
            site_sums<COSMODE>(P, ws, atomsB[cb], Cb, nAct, allSites, -1, refl, lane);
            cachedAct = nAct;
          }
          if (reeval || !mcmc) {
            double sums[3];
            fitness_from_banks(P, ws, Cb, -1, ic, refl, ftab, groups, sooPrefix, ngaC, lane, sums, tIc);
            const float cc = P.profV ? profile_cc(P, ic, lane) : cc_of(sums);
            const float pen = penalty<SLOTS>(P, atomsB[cb], rmin, shellLen, myPairs, myNPairs, lane) * penScale;
            fit = cc - pen;
            cc0 = cc;
            pen0 = pen / fmaxf(penScale, 1e-9f);
          }
        } else {
          if (reeval || !mcmc) {
            // evaluate the current state (dispatchCoords(null, false))
            expand(P, gen, ops, ws.cur, atoms, lane);
            __syncwarp();
            double sums[3];
            if constexpr (COSMODE == 2)
              fitness_factored(P, ws, ws.cur, ftabs, ftags, ic64, refl, stat, groups, sooPrefix, ngaC, lane, sums,
                               tIc);
            else
              fitness_direct<COSMODE>(P, ws, atoms, ic, refl, ftab, groups, sooPrefix, ngaC, lane, sums, tIc);
            if (P.traceSums && lane == 0)
              for (int k = 0; k < 3; ++k) P.traceSums[(size_t)p * 3 + k] = sums[k];
            const float cc = P.profV ? (COSMODE == 2 ? profile_cc(P, ic64, lane) : profile_cc(P, ic, lane)) : cc_of(sums);
            const float pen = penalty<SLOTS>(P, atoms, rmin, shellLen, myPairs, myNPairs, lane) * penScale;
            fit = cc - pen;
            cc0 = cc;
            pen0 = pen / fmaxf(penScale, 1e-9f);
          }
        }
        if (mcmc) {
          float uMetro;
          const float sd = P.quenchSd ? P.quenchSd[g] : __shfl_sync(0xffffffffu, step, 0);
          if (P.extProp) {
            // a proposal chosen outside (the learned search): the Metropolis draw stays ours
            for (int j = lane; j < (int)curStride; j += 32) ws.prop[j] = P.extProp[(size_t)p * curStride + j];
            const uint4 u = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, 0xFFFEu, 3u), make_uint2(seed, P.runKey));
            uMetro = u01(u.x);
            __syncwarp();
          } else {
            propose<SLOTS>(P, ws, proj, ops, g, p, lane, sd, seed, &uMetro);
          }
          double sums[3];
          uint32_t moved = 0;
          const uint4 *evalAtoms;
          if constexpr (INCR) {
            bool diff = false;
            if (lane < P.maxSites)
              diff = ws.prop[lane * 3] != ws.cur[lane * 3] || ws.prop[lane * 3 + 1] != ws.cur[lane * 3 + 1] ||
                     ws.prop[lane * 3 + 2] != ws.cur[lane * 3 + 2];
            moved = __ballot_sync(0xffffffffu, diff);
            expand_moved(P, gen, ops, ws.prop, moved, atomsB[cb], atomsB[cb ^ 1], lane);
            if (__popc(moved) <= 1) {
              // one site moved (or none): its sums go to the spare slot, the rest are reused
              const int spare = moved ? __ffs(moved) - 1 : -1;
              if (moved) site_sums<COSMODE>(P, ws, atomsB[cb ^ 1], Cb, cachedAct, moved, spare, refl, lane);
              fitness_from_banks(P, ws, Cb, spare, ic, refl, ftab, groups, sooPrefix, ngaC, lane, sums, tIc);
            } else {
              // a collective move: full evaluation, the cache is refilled if it is accepted
              fitness_direct<COSMODE>(P, ws, atomsB[cb ^ 1], ic, refl, ftab, groups, sooPrefix, ngaC, lane, sums,
                                      tIc);
            }
            evalAtoms = atomsB[cb ^ 1];
          } else {
            expand(P, gen, ops, ws.prop, atoms, lane);
            __syncwarp();
            if constexpr (COSMODE == 2)
              fitness_factored(P, ws, ws.prop, ftabs, ftags, ic64, refl, stat, groups, sooPrefix, ngaC, lane, sums,
                               tIc);
            else
              fitness_direct<COSMODE>(P, ws, atoms, ic, refl, ftab, groups, sooPrefix, ngaC, lane, sums, tIc);
            evalAtoms = atoms;
          }
          if (P.traceSums && lane == 0)
            for (int k = 0; k < 3; ++k) P.traceSums[(size_t)p * 3 + k] = sums[k];
          const float cc = P.profV ? (COSMODE == 2 ? profile_cc(P, ic64, lane) : profile_cc(P, ic, lane)) : cc_of(sums);
          const float pen = penalty<SLOTS>(P, evalAtoms, rmin, shellLen, myPairs, myNPairs, lane) * penScale;
          int acc = 0, best = 0;
          if (P.deferAccept) {
            // fixed-profile search: the proposal's intensities went to traceIc;
            // its penalty and Metropolis draw wait for the profile chi^2
            if (lane == 0 && P.traceRec) {
              float *rec = P.traceRec + (size_t)p * 8;
              rec[0] = cc - pen; rec[1] = cc; rec[2] = pen; rec[3] = uMetro;
              rec[4] = 0.f; rec[5] = 0.f; rec[6] = temp; rec[7] = step;
            }
            if (P.frag && P.fragProp && lane < kFragParams)
              P.fragProp[(size_t)p * kFragParams + lane] = fcurW[kFragParams + lane];
          } else if (lane == 0) {
            const float fNew = cc - pen;
            float fOld = fit;
            if (fOld > -1.0e29f) fOld = cc0 - pen0 * penScale;
            const float stepBefore = step;
            if (P.quenchSd)
              acc = fNew > fOld ? 1 : 0;   // quench: only improvements (js/swarm_wyckoff.js:2069-2075)
            else if (fNew >= fOld)
              acc = 1;
            else if (uMetro < expf((fNew - fOld) / fmaxf(temp, 1e-9f)))
              acc = 1;
            if (acc) {
              fit = fNew;
              cc0 = cc;
              pen0 = pen / fmaxf(penScale, 1e-9f);
              accepted += 1u;
              const bool hasBest = bestFit > -1.0e29f;
              const float bestR = hasBest ? bestCC - bestPen * penScale : -1.0e30f;
              if (fNew > bestR) {
                bestFit = fNew;
                bestCC = cc;
                bestPen = pen / fmaxf(penScale, 1e-9f);
                best = 1;
              }
            }
            if (!P.quenchSd) step = fminf(fmaxf(step * (acc ? P.stepUp : P.stepDown), P.stepMin), P.stepMax);
            if (P.traceRec) {
              float *rec = P.traceRec + (size_t)p * 8;
              rec[0] = fNew; rec[1] = cc; rec[2] = pen; rec[3] = uMetro;
              rec[4] = (float)acc; rec[5] = fOld; rec[6] = temp; rec[7] = stepBefore;
            }
          }
          acc = __shfl_sync(0xffffffffu, acc, 0);
          best = __shfl_sync(0xffffffffu, best, 0);
          if (P.tracePos)
            for (int j = lane; j < (int)curStride; j += 32) P.tracePos[(size_t)p * curStride + j] = ws.prop[j];
          if (acc) {
            for (int j = lane; j < (int)curStride; j += 32) ws.cur[j] = ws.prop[j];
            if (P.frag && lane < kFragParams) fcurW[lane] = fcurW[kFragParams + lane];
            if constexpr (INCR) {
              cb ^= 1;
              if (__popc(moved) == 1) {
                if (lane == 0) {
                  const int site = __ffs(moved) - 1, t = ws.slot[site];
                  ws.slot[site] = ws.slot[P.maxSites];
                  ws.slot[P.maxSites] = t;
                }
              } else if (moved) {
                cachedAct = -1;
              }
            }
          }
          if (best) {
            for (int j = lane; j < (int)curStride; j += 32) bestBase[(size_t)p * curStride + j] = ws.prop[j];
            if (P.frag && lane < kFragParams) P.fragBest[(size_t)p * kFragParams + lane] = fcurW[kFragParams + lane];
          }
          __syncwarp();
        } else if (lane == 0 && P.traceRec) {
          float *rec = P.traceRec + (size_t)p * 8;
          rec[0] = fit; rec[1] = cc0; rec[2] = pen0 * penScale;
        }
      }
      prevNga = nga;
      // replica exchange inside the ladder (js/swarm_wyckoff.js:1825-1851)
      if (swapEvery > 0 && mcmc && P.ladders && ((g + 1) % swapEvery) == 0) {
        float *eFit = ladder_peer<RANKS>(exFit, 0), *eCC = ladder_peer<RANKS>(exCC, 0);
        float *ePen = ladder_peer<RANKS>(exPen, 0);
        const int *eSwap = ladder_peer<RANKS>(exSwap, 0);
        if (active && lane == 0) {
          eFit[rung] = fit; eCC[rung] = cc0; ePen[rung] = pen0; ladder_peer<RANKS>(exTemp, 0)[rung] = temp;
          ladder_peer<RANKS>(exE, 0)[rung] = isfinite(cc0) ? cc0 - pen0 * penScale : fit;
        }
        if (rank == 0 && threadIdx.x < kMaxRungs) exSwap[threadIdx.x] = -1;
        ladder_sync<RANKS>();
        if (rank == 0 && threadIdx.x == 0) {
          const int parity = ((g + 1) / swapEvery) & 1;
          unsigned long long tried = 0, taken = 0;
          for (int r = parity; r + 1 < rungs; r += 2) {
            const int a = P.ladders[(size_t)L * rungs + r], b = P.ladders[(size_t)L * rungs + r + 1];
            if (a < 0 || b < 0) continue;
            const float fa = exE[r], fb = exE[r + 1];
            if (!isfinite(fa) || !isfinite(fb)) continue;
            ++tried;
            const float d = (1.0f / exTemp[r] - 1.0f / exTemp[r + 1]) * (fb - fa);
            if (d < 0.f) {
              const uint4 c = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)L, (uint32_t)r, 7u),
                                            make_uint2(P.runKey, 0x45584348u));
              if (u01(c.x) >= expf(d)) continue;
            }
            ++taken;
            exSwap[r] = r + 1;
            float t = exFit[r]; exFit[r] = exFit[r + 1]; exFit[r + 1] = t;
            t = exCC[r]; exCC[r] = exCC[r + 1]; exCC[r + 1] = t;
            t = exPen[r]; exPen[r] = exPen[r + 1]; exPen[r + 1] = t;
          }
          if (P.swapStats && tried) {
            atomicAdd(P.swapStats, tried);
            atomicAdd(P.swapStats + 1, taken);
          }
        }
        ladder_sync<RANKS>();
        // the energies after the decisions; a rung that received other
        // coordinates refills its site sums
        if (active) {
          if (lane == 0) { fit = eFit[rung]; cc0 = eCC[rung]; pen0 = ePen[rung]; }
          const bool swapped = eSwap[rung] >= 0 || (rung > 0 && eSwap[rung - 1] == rung);
          if (swapped) cachedAct = -1;
        }
        // each pair (r, r+1) swaps coordinates, by rung r's warp; rungs keep temp and step
        if (rung < rungs && eSwap[rung] >= 0) {
          const int r1 = rung + 1;
          unsigned char *mine = smem + blobPad + (size_t)warp * P.warpSmemBytes;
          unsigned char *other =
              ladder_peer<RANKS>(smem + blobPad + (size_t)(r1 % nWarps) * P.warpSmemBytes, r1 / nWarps);
          const WarpView wa = warp_view(mine, P);
          const WarpView wb = warp_view(other, P);
          for (int j = lane; j < (int)curStride; j += 32) {
            const uint32_t t = wa.cur[j];
            wa.cur[j] = wb.cur[j];
            wb.cur[j] = t;
          }
          if (P.frag && lane < kFragParams) {
            float *fa = reinterpret_cast<float *>(mine + P.fragOff), *fb = reinterpret_cast<float *>(other + P.fragOff);
            const float t = fa[lane];
            fa[lane] = fb[lane];
            fb[lane] = t;
          }
        }
        ladder_sync<RANKS>();
      }
    }
    if (active) {
      for (int j = lane; j < (int)curStride; j += 32) P.pos[(size_t)p * curStride + j] = ws.cur[j];
      if (P.frag && lane < kFragParams) P.fragState[(size_t)p * kFragParams + lane] = fcurW[lane];
      if (lane == 0) {
        PState st;
        st.fit = fit; st.cc = cc0; st.pen = pen0; st.step = step; st.temp = temp;
        st.seed = seed; st.accepted = accepted; st.pad = 0;
        st.bestFit = bestFit; st.bestCC = bestCC; st.bestPen = bestPen; st.bestPad = 0.f;
        P.st[p] = st;
      }
    }
    __syncthreads();
  }
  // the staging barrier is set up afresh by the next call on this CTA
  if (stage && threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&stageBar)) : "memory");
  ladder_sync<RANKS>();   // no CTA leaves while its partner may still reach its shared memory
  return true;
}

template <int COSMODE, int SLOTS, int INCR, int GT = 0>
__global__ void __launch_bounds__(256, 4) wy_kernel(const __grid_constant__ Params P, int gen0, int nGen, int mcmc,
                                                    int swapEvery, int reevalFirst) {
  wy_cta<COSMODE, SLOTS, INCR, 1, GT>(P, blockIdx.x, gridDim.x, gen0, nGen, mcmc, swapEvery, reevalFirst);
}

// The same search with each ladder of 8 on a cluster of two 4-warp CTAs
// (launched with cluster dimension 2): ladder = cluster index.
template <int COSMODE, int SLOTS, int INCR>
__global__ void __launch_bounds__(128, 7) wy_kernel_pair(const __grid_constant__ Params P, int gen0, int nGen,
                                                         int mcmc, int swapEvery, int reevalFirst) {
  wy_cta<COSMODE, SLOTS, INCR, 2>(P, blockIdx.x >> 1, gridDim.x >> 1, gen0, nGen, mcmc, swapEvery, reevalFirst);
}

// Per-problem generation range of a batched launch.
struct RunArgs {
  int gen0, nGen, mcmc, swapEvery, reevalFirst, pad[3];
};

// Many independent searches in one persistent launch: each CTA takes the
// next (problem, ladder) item from a list ordered by estimated cost, copies
// that problem's parameters into shared memory, stages its tables and runs
// the ladder through its generations.
template <int COSMODE, int SLOTS, int INCR>
__global__ void __launch_bounds__(256, 4) wy_batch_kernel(const Params *probs, const RunArgs *args, const int2 *items,
                                                          int nItems, int *counter) {
  __shared__ __align__(16) Params Ps;
  __shared__ int item;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = item;
    if (it >= nItems) break;
    const int2 w = items[it];
    const int *src = reinterpret_cast<const int *>(probs + w.x);
    int *dst = reinterpret_cast<int *>(&Ps);
    for (int i = threadIdx.x; i < (int)(sizeof(Params) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    const RunArgs a = args[w.x];
    // Lstep = nLadders: this ladder only
    const bool ok = Ps.blobGlobal
                        ? wy_cta<COSMODE, SLOTS, INCR, 1, 1>(Ps, w.y, Ps.nLadders, a.gen0, a.nGen, a.mcmc, a.swapEvery,
                                                             a.reevalFirst)
                        : wy_cta<COSMODE, SLOTS, INCR, 1, 0>(Ps, w.y, Ps.nLadders, a.gen0, a.nGen, a.mcmc, a.swapEvery,
                                                             a.reevalFirst);
    if (!ok) break;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Learned search: K candidate proposals per replica with their features, and
// the choice among them by the proposal network's predicted gain.
// ---------------------------------------------------------------------------
constexpr int kFeat = 64;   // feature vector of one candidate

// One thread per (particle, candidate): the plain search's move (one free
// site with probability 0.75, else every site; Gaussian steps of the
// replica's width, projected onto the Wyckoff subspace) and its features:
// one-hot moved site, collective flag, the site's position and its
// candidate (sin, cos of 2 pi x), the step in units of the width, and the
// replica's cc, penalty, fitness, log width and temperature.
__global__ void wy_candidates_kernel(const Params P, int g, int K, uint32_t *cand, float *feat) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)P.numParticles * K) return;
  const int p = (int)(t / K), c = (int)(t % K);
  const size_t stride = (size_t)P.maxSites * 3;
  const uint32_t *cur = P.pos + (size_t)p * stride;
  uint32_t *out = cand + (size_t)t * stride;
  float *f = feat + (size_t)t * kFeat;
  for (int i = 0; i < kFeat; ++i) f[i] = 0.f;
  const PState st = P.st[p];
  const int A = (int)P.assign[p];
  const uint32_t free = P.freeMask[A];
  const int nFree = __popc(free);
  const uint2 key = make_uint2(st.seed, P.runKey);
  const uint4 r0 = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, (uint32_t)c, 9u), key);
  int pick = -1;
  if (u01(r0.x) < 0.75f && nFree > 0) {
    const int kth = min(nFree - 1, (int)(u01(r0.y) * (float)nFree));
    pick = __fns(free, 0, kth + 1);
  }
  const float sd = st.step;
  const float scale = sd * 4294967296.0f;
  constexpr float kTwoPiTurn = 6.28318530717958647f / 4294967296.0f;
  for (size_t j = 0; j < stride; ++j) out[j] = cur[j];
  for (int s = 0; s < P.maxSites; ++s) {
    if (!(pick < 0 || pick == s)) continue;
    if (!((free >> s) & 1u) && pick < 0) continue;   // fixed sites do not move
    const uint4 r = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)p, ((uint32_t)c << 8) | (uint32_t)s, 10u), key);
    const float2 n01 = gauss2(r.x, r.y), n23 = gauss2(r.z, r.w);
    const float gz[3] = {n01.x, n01.y, n23.x};
    int64_t pos[3];
    for (int i = 0; i < 3; ++i) pos[i] = (int64_t)cur[s * 3 + i] + __float2ll_rn(gz[i] * scale);
    const ProjFix &pr = P.proj[(size_t)A * P.maxSites + s];
    uint32_t nw[3];
    if (pr.pad[0]) {
      for (int i = 0; i < 3; ++i) nw[i] = (pr.num[4 * i] ? (uint32_t)pos[i] : 0u) + pr.t[i];
    } else {
      for (int i = 0; i < 3; ++i) {
        int64_t acc = (int64_t)pr.num[3 * i] * pos[0] + (int64_t)pr.num[3 * i + 1] * pos[1] +
                      (int64_t)pr.num[3 * i + 2] * pos[2];
        if (pr.den != 1) acc = floor_div(acc, pr.den);
        nw[i] = (uint32_t)(acc + (int64_t)pr.t[i]);
      }
    }
    for (int i = 0; i < 3; ++i) out[s * 3 + i] = nw[i];
    if (pick == s) {
      if (s < 32) f[s] = 1.f;
      for (int i = 0; i < 3; ++i) {
        float sv, cv;
        __sincosf((float)(int)cur[s * 3 + i] * kTwoPiTurn, &sv, &cv);
        f[33 + 2 * i] = sv;
        f[34 + 2 * i] = cv;
        f[39 + i] = gz[i];
        __sincosf((float)(int)nw[i] * kTwoPiTurn, &sv, &cv);
        f[42 + 2 * i] = sv;
        f[43 + 2 * i] = cv;
      }
    }
  }
  f[32] = pick < 0 ? 1.f : 0.f;
  f[48] = isfinite(st.cc) ? st.cc : 0.f;
  f[49] = isfinite(st.pen) ? st.pen : 0.f;
  f[50] = isfinite(st.fit) && st.fit > -1e29f ? st.fit : 0.f;
  f[51] = __logf(fmaxf(sd, 1e-6f));
  f[52] = st.temp * 100.f;
}

// Per particle: the candidate with the largest predicted gain (score column 0
// of d_out), or candidate 0 without a network; its proposal and features.
__global__ void wy_select_kernel(const Params P, int K, const float *score, int dOut, const uint32_t *cand,
                                 const float *feat, uint32_t *ext, float *chosenFeat, float *chosenScore) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.numParticles) return;
  int best = 0;
  float bs = score ? score[(size_t)p * K * dOut] : 0.f;
  if (score)
    for (int c = 1; c < K; ++c) {
      const float v = score[((size_t)p * K + c) * dOut];
      if (v > bs) { bs = v; best = c; }
    }
  const size_t stride = (size_t)P.maxSites * 3;
  const size_t src = (size_t)p * K + best;
  for (size_t j = 0; j < stride; ++j) ext[(size_t)p * stride + j] = cand[src * stride + j];
  for (int i = 0; i < kFeat; ++i) chosenFeat[(size_t)p * kFeat + i] = feat[src * kFeat + i];
  chosenScore[p] = bs;
}

// Generated cell of one particle in genPack order (parity support).
__global__ void wy_expand_one(const Params P, const uint32_t *genOrig, int particle, uint32_t *out) {
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= P.nTot) return;
  const int A = (int)P.assign[particle];
  const uint32_t w = genOrig[(size_t)A * P.nTot + i];
  const int s = w & 0xFF, o = (w >> 8) & 0xFFF;
  const OpFix &op = P.ops[o];
  const uint32_t *x = P.pos + (size_t)particle * P.maxSites * 3 + s * 3;
  for (int c = 0; c < 3; ++c)
    out[i * 3 + c] = (uint32_t)op.r[3 * c] * x[0] + (uint32_t)op.r[3 * c + 1] * x[1] +
                     (uint32_t)op.r[3 * c + 2] * x[2] + op.t[c];
}

__global__ void philox_one(uint4 c, uint2 k, uint4 *out) { *out = philox4x32_10(c, k); }

// One warp per parameter vector: the fragment's fixed-point coordinates.
__global__ void wy_fragment_atoms_kernel(const FragDev *F, const float *prm, int n, uint32_t *out) {
  const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (v >= n) return;
  __shared__ uint32_t buf[8][kFragMaxAtoms * 3];
  uint32_t *o = buf[threadIdx.x >> 5];
  frag_atoms(*F, prm + (size_t)v * kFragParams, o, lane);
  __syncwarp();
  for (int j = lane; j < F->nAtoms * 3; j += 32) out[(size_t)v * F->nAtoms * 3 + j] = o[j];
}

// Acceptance step of a fixed-profile search: the Metropolis test, best
// tracking, step adaptation and ladder exchange of the fused search
// (js/swarm_wyckoff.js:1825-1851 for the exchange) with the profile chi^2 as
// the energy.  A replica's agreement is 1 - Rwp, Rwp = sqrt(chi^2 / sum w y^2)
// at its best scale, and its fitness is agreement - penalty, the place cc -
// penalty holds in the intensity search.  One warp per ladder, lane r on rung
// r; the proposals and their penalties and uniforms come from the search
// kernel's deferred generation (tracePos, traceRec).  init != 0: chi^2 is of
// the current structures, which become the chains' energies.
constexpr int kAcceptWarps = 4;
__global__ void __launch_bounds__(32 * kAcceptWarps) wy_profile_accept_kernel(const Params P, const double2 *part,
                                                                             int nParts, double syy, int g,
                                                                             int swapEvery, int init) {
  __shared__ float sE[kAcceptWarps][kMaxRungs], sT[kAcceptWarps][kMaxRungs];
  __shared__ int sSwap[kAcceptWarps][kMaxRungs];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = blockIdx.x * kAcceptWarps + w;
  if (L >= P.nLadders) return;   // whole warps leave together
  const int rungs = P.rungs;
  const size_t stride = (size_t)P.maxSites * 3;
  uint32_t *bestBase = P.pos + (size_t)P.numParticles * stride;
  const float penScale = P.schedGroups ? P.schedPen[g] : P.penArg;
  const float ps = fmaxf(penScale, 1e-9f);
  int p = -1;
  if (lane < rungs) {
    if (P.ladders) {
      p = P.ladders[(size_t)L * rungs + lane];
    } else {
      const int q = L * rungs + lane;
      p = q < P.numParticles ? q : -1;
    }
  }
  // chi^2 of each rung's replica at its best scale from the contraction's
  // partials {a = sum w y Y, b = sum w Y^2}: the rungs' rows are read at
  // once, lpr lanes per rung (lane l: rung l / lpr, partials l % lpr, + lpr,
  // ... in order), then a fixed butterfly inside each group of lpr lanes;
  // chi^2 = sum w y^2 - a^2 / b (no positive scale: sum w y^2)
  int lpr = 32;
  while (lpr > 1 && lpr * rungs > 32) lpr >>= 1;
  const int myRung = lane / lpr, sub = lane % lpr;
  const int q = __shfl_sync(0xffffffffu, p, myRung);
  double a = 0.0, b = 0.0;
  if (myRung < rungs && q >= 0) {
    const double2 *row = part + (size_t)q * nParts;
    for (int t = sub; t < nParts; t += lpr) {
      const double2 v = row[t];
      a += v.x;
      b += v.y;
    }
  }
  for (int o = lpr >> 1; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  double chiGroup = syy;
  if (a > 0.0 && b > 0.0) chiGroup = fmax(syy - a * (a / b), 0.0);
  const double chi = __shfl_sync(0xffffffffu, chiGroup, lane < rungs ? lane * lpr : 0);
  int acc = 0, best = 0;
  PState st{};
  if (p >= 0) {
    st = P.st[p];
    float *rec = P.traceRec + (size_t)p * 8;
    const float pen = rec[2];
    const float cc = 1.0f - (float)sqrt(chi / syy);
    const float fNew = cc - pen;
    if (init) {
      st.fit = fNew; st.cc = cc; st.pen = pen / ps;
      acc = 1;
    } else {
      float fOld = st.fit;
      if (fOld > -1.0e29f) fOld = st.cc - st.pen * penScale;
      const float u = rec[3];
      if (P.quenchSd)
        acc = fNew > fOld ? 1 : 0;
      else if (fNew >= fOld)
        acc = 1;
      else if (u < expf((fNew - fOld) / fmaxf(st.temp, 1e-9f)))
        acc = 1;
      if (acc) {
        st.fit = fNew; st.cc = cc; st.pen = pen / ps;
        st.accepted += 1u;
      }
      if (!P.quenchSd) st.step = fminf(fmaxf(st.step * (acc ? P.stepUp : P.stepDown), P.stepMin), P.stepMax);
      rec[4] = (float)acc;
      rec[5] = fOld;
    }
    rec[0] = fNew;
    rec[1] = cc;
    if (acc) {
      const float bestR = st.bestFit > -1.0e29f ? st.bestCC - st.bestPen * penScale : -1.0e30f;
      if (fNew > bestR) {
        st.bestFit = fNew; st.bestCC = cc; st.bestPen = pen / ps;
        best = 1;
      }
    }
  }
  // accepted proposals become current (init keeps the current structures);
  // new bests are copied from the current bank
  const unsigned accMask = init ? 0u : __ballot_sync(0xffffffffu, acc);
  const unsigned bestMask = __ballot_sync(0xffffffffu, best);
  // (a rigid fragment's parameters follow its coordinates)
  const bool frag = P.frag && P.fragState && P.fragBest && P.fragProp;
  for (unsigned m = accMask; m; m &= m - 1) {
    const int q = __shfl_sync(0xffffffffu, p, __ffs(m) - 1);
    for (int j = lane; j < (int)stride; j += 32) P.pos[(size_t)q * stride + j] = P.tracePos[(size_t)q * stride + j];
    if (frag && lane < kFragParams)
      P.fragState[(size_t)q * kFragParams + lane] = P.fragProp[(size_t)q * kFragParams + lane];
  }
  __syncwarp();
  for (unsigned m = bestMask; m; m &= m - 1) {
    const int q = __shfl_sync(0xffffffffu, p, __ffs(m) - 1);
    for (int j = lane; j < (int)stride; j += 32) bestBase[(size_t)q * stride + j] = P.pos[(size_t)q * stride + j];
    if (frag && lane < kFragParams)
      P.fragBest[(size_t)q * kFragParams + lane] = P.fragState[(size_t)q * kFragParams + lane];
  }
  __syncwarp();
  if (swapEvery > 0 && !init && ((g + 1) % swapEvery) == 0) {
    if (p >= 0) {
      sE[w][lane] = isfinite(st.cc) ? st.cc - st.pen * penScale : st.fit;
      sT[w][lane] = st.temp;
    }
    if (lane < kMaxRungs) sSwap[w][lane] = -1;
    __syncwarp();
    if (lane == 0) {
      const int parity = ((g + 1) / swapEvery) & 1;
      unsigned long long tried = 0, taken = 0;
      for (int r = parity; r + 1 < rungs; r += 2) {
        const int a = P.ladders ? P.ladders[(size_t)L * rungs + r] : L * rungs + r;
        const int b = P.ladders ? P.ladders[(size_t)L * rungs + r + 1] : L * rungs + r + 1;
        if (a < 0 || b < 0 || a >= P.numParticles || b >= P.numParticles) continue;
        const float fa = sE[w][r], fb = sE[w][r + 1];
        if (!isfinite(fa) || !isfinite(fb)) continue;
        ++tried;
        const float d = (1.0f / sT[w][r] - 1.0f / sT[w][r + 1]) * (fb - fa);
        if (d < 0.f) {
          const uint4 c = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)L, (uint32_t)r, 7u),
                                        make_uint2(P.runKey, 0x45584348u));
          if (u01(c.x) >= expf(d)) continue;
        }
        ++taken;
        sSwap[w][r] = r + 1;
      }
      if (P.swapStats && tried) {
        atomicAdd(P.swapStats, tried);
        atomicAdd(P.swapStats + 1, taken);
      }
    }
    __syncwarp();
    // energies follow the coordinates; temperature and step stay with the rung
    int partner = lane;
    if (lane < rungs) {
      if (sSwap[w][lane] >= 0) partner = lane + 1;
      else if (lane > 0 && sSwap[w][lane - 1] == lane) partner = lane - 1;
    }
    const float oFit = __shfl_sync(0xffffffffu, st.fit, partner);
    const float oCC = __shfl_sync(0xffffffffu, st.cc, partner);
    const float oPen = __shfl_sync(0xffffffffu, st.pen, partner);
    if (partner != lane && p >= 0) {
      st.fit = oFit; st.cc = oCC; st.pen = oPen;
    }
    for (int r = 0; r + 1 < rungs; ++r) {
      if (sSwap[w][r] < 0) continue;
      const int a = __shfl_sync(0xffffffffu, p, r), b = __shfl_sync(0xffffffffu, p, r + 1);
      for (int j = lane; j < (int)stride; j += 32) {
        const uint32_t t = P.pos[(size_t)a * stride + j];
        P.pos[(size_t)a * stride + j] = P.pos[(size_t)b * stride + j];
        P.pos[(size_t)b * stride + j] = t;
      }
      if (frag && lane < kFragParams) {
        const float t = P.fragState[(size_t)a * kFragParams + lane];
        P.fragState[(size_t)a * kFragParams + lane] = P.fragState[(size_t)b * kFragParams + lane];
        P.fragState[(size_t)b * kFragParams + lane] = t;
      }
    }
  }
  if (p >= 0) P.st[p] = st;
}

}  // namespace wy
}  // namespace p6

// ===========================================================================
// Host side: the session.
// ===========================================================================
using namespace p6;
using namespace p6::wy;

struct p6_wy_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Params P{};
  int cosMode = 0;
  int slots = 0;  // 0: clash only; 64 / 256: rule variants
  int incremental = 0;  // site sums cached per replica (two banks) in shared memory
  uint32_t *dGen = nullptr, *dGenOrig = nullptr, *dFree = nullptr, *dPos = nullptr, *dAssign = nullptr;
  int4 *dRuns = nullptr;
  int2 *dPairRange = nullptr;
  int *dNRuns = nullptr, *dNF = nullptr, *dLadders = nullptr, *dSchedG = nullptr, *dErr = nullptr;
  float *dSchedP = nullptr, *dTraceRec = nullptr, *dTraceIc = nullptr, *dQuench = nullptr;
  double *dTraceSums = nullptr;   // per particle {scc, soo, sco} of the last traced evaluation
  FragDev *dFrag = nullptr;       // rigid-fragment search (p6_wy_set_fragment)
  float *dFragState = nullptr, *dFragBest = nullptr, *dFragProp = nullptr;
  int quenchLen = 0;
  // learned search: candidates, features, scores, the chosen proposal
  uint32_t *dCand = nullptr, *dExt = nullptr;
  float *dFeat = nullptr, *dScore = nullptr, *dChosenFeat = nullptr, *dChosenScore = nullptr;
  int learnK = 0, learnOut = 0;
  uint32_t *dTracePos = nullptr;
  OpFix *dOps = nullptr;
  ProjFix *dProj = nullptr;
  unsigned char *dBlob = nullptr;
  RuleDev *dRules = nullptr;
  PState *dSt = nullptr;
  unsigned long long *dSwap = nullptr;
  int nLadders = 0, rungs = 8, schedLen = 0;
  int nga = 0;
  float penScale = 1.0f;
  bool trace = false;
  long long launches = 0;
  std::vector<uint32_t> hostAssign;
  std::vector<uint32_t> siteCountOfAssign;
  std::vector<ProjFix> projHost;     // Wyckoff projectors per (assignment, site), for the refinement
  std::vector<float4> groupsHost;    // {start, count, Iobs, weight} per reflection group
  int smemBytes = 0;
  int maxGrid = 0;
  int smemPair = 0;      // per CTA when a ladder spans a cluster of two CTAs
  int ladderSplit = 2;   // CTAs per ladder of 8 in the fused search (1 or 2)
  std::vector<float> schedPenHost;   // the penalty schedule (fixed-profile search)
  double *dProfV = nullptr, *dProfG = nullptr;   // Gram-form fixed-profile fitness (p6_wy_set_profile)
  p6_ct_session *linkedCt = nullptr; // contraction of the last fixed-profile run (its waits are checked too)
};

namespace {

thread_local std::string g_err;
int g_inject_code = 0, g_inject_after = -1;

}  // namespace

namespace p6 {
p6_status set_error(p6_status code, const std::string &msg) {
  g_err = msg;
  return code;
}
p6_status cuda_error(cudaError_t e, const char *what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorIllegalAddress || e == cudaErrorLaunchFailure || e == cudaErrorDevicesUnavailable ||
      e == cudaErrorHardwareStackError || e == cudaErrorIllegalInstruction || e == cudaErrorMisalignedAddress)
    return P6_ERR_DEVICE_LOST;
  return P6_ERR_CUDA;
}
void clear_error() { g_err.clear(); }
}  // namespace p6

static p6_status injected() {
  if (g_inject_after < 0 || g_inject_code == 0) return P6_OK;
  if (g_inject_after-- == 0) {
    const int c = g_inject_code;
    g_inject_code = 0;
    g_inject_after = -1;
    return set_error((p6_status)c, "injected failure (host-side fault injection)");
  }
  return P6_OK;
}

#define P6_ENTRY()                      \
  do {                                  \
    clear_error();                      \
    p6_status _inj = injected();        \
    if (_inj != P6_OK) return _inj;     \
  } while (0)

static uint32_t to_fixed(double x) {
  double f = x - std::floor(x);
  double v = std::floor(f * kTwoPow32 + 0.5);
  if (v >= kTwoPow32) v -= kTwoPow32;
  return (uint32_t)(uint64_t)v;
}
static float from_fixed(uint32_t x) {
  float f = (float)((double)x / kTwoPow32);
  return f >= 1.0f ? 0.0f : f;
}
// Translation snapped to a multiple of 1/24 when it is one, then fixed point.
static uint32_t trans_fixed(double t) {
  double s = t * 24.0, r = std::floor(s + 0.5);
  if (std::fabs(s - r) < 1e-4) {
    long long n = ((long long)r % 24 + 24) % 24;
    return (uint32_t)((n * 4294967296LL + 12) / 24);
  }
  return to_fixed(t);
}
// Smallest denominator (<= 24) making every entry of P an integer.
static bool rationalise(const float *p, int n, int *num, int *den) {
  static const int dens[] = {1, 2, 3, 4, 6, 8, 12, 24};
  for (int d : dens) {
    bool ok = true;
    for (int i = 0; i < n && ok; ++i) {
      double v = (double)p[i] * d;
      if (std::fabs(v - std::floor(v + 0.5)) > 1e-4) ok = false;
    }
    if (ok) {
      for (int i = 0; i < n; ++i) num[i] = (int)std::floor((double)p[i] * d + 0.5);
      *den = d;
      return true;
    }
  }
  return false;
}

template <typename T>
static p6_status upload(T **dst, const T *src, size_t n, cudaStream_t s) {
  P6_CUDA(cudaMalloc((void **)dst, std::max<size_t>(n, 1) * sizeof(T)));
  if (n) P6_CUDA(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return P6_OK;
}

static void free_session(p6_wy_session *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  void *ptrs[] = {s->dGen, s->dGenOrig, s->dFree, s->dPos, s->dAssign, s->dRuns, s->dNRuns, s->dNF,
                  s->dLadders, s->dSchedG, s->dErr, s->dSchedP, s->dQuench, s->dTraceRec, s->dTraceIc, s->dTraceSums, s->dFrag, s->dFragState, s->dFragBest, s->dFragProp, s->dTracePos, s->dOps,
                  s->dProj, s->dBlob, s->dRules, s->dSt, s->dSwap, s->dCand, s->dExt, s->dFeat, s->dScore,
                  s->dChosenFeat, s->dChosenScore, s->dPairRange, s->dProfV, s->dProfG};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

template <int C, int S, int I>
static cudaError_t launch_variant(p6_wy_session *s, int grid, int block, int gen0, int nGen, int mcmc,
                                  int swapEvery, int reevalFirst) {
  // global tables only without incremental sums (those need the shared memory anyway)
  auto k = wy_kernel<C, S, I, 0>;
  if constexpr (I == 0)
    if (s->P.blobGlobal) k = wy_kernel<C, S, I, 1>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemBytes);
  if (e != cudaSuccess) return e;
  k<<<grid, block, s->smemBytes, s->stream>>>(s->P, gen0, nGen, mcmc, swapEvery, reevalFirst);
  return cudaGetLastError();
}

// A ladder of 8 on a cluster of two 4-warp CTAs, one cluster per ladder.
template <int C, int I>
static cudaError_t launch_pair(p6_wy_session *s, int gen0, int nGen, int mcmc, int swapEvery, int reevalFirst) {
  auto k = wy_kernel_pair<C, 0, I>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemPair);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * s->P.nLadders, 1, 1);
  cfg.blockDim = dim3(128, 1, 1);
  cfg.dynamicSmemBytes = (size_t)s->smemPair;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, k, s->P, gen0, nGen, mcmc, swapEvery, reevalFirst);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

template <int C, int S>
static cudaError_t launch_incr(p6_wy_session *s, int grid, int block, int gen0, int nGen, int mcmc, int swapEvery,
                               int reevalFirst) {
  if (s->incremental) return launch_variant<C, S, 1>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  return launch_variant<C, S, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
}

static cudaError_t launch(p6_wy_session *s, int gen0, int nGen, int mcmc, int swapEvery, int reevalFirst) {
  Params &P = s->P;
  const int rungs = P.rungs;
  const int block = 32 * rungs;
  int grid = std::min(P.nLadders, s->maxGrid > 0 ? s->maxGrid : P.nLadders);
  grid = std::max(grid, 1);
  cudaError_t e;
  const int C = s->cosMode, S = s->slots;
  if (s->ladderSplit == 2 && P.ladders && rungs == 8 && S == 0 && !s->incremental && s->smemPair > 0 &&
      !P.blobGlobal) {
    e = C == 0   ? launch_pair<0, 0>(s, gen0, nGen, mcmc, swapEvery, reevalFirst)
        : C == 1 ? launch_pair<1, 0>(s, gen0, nGen, mcmc, swapEvery, reevalFirst)
                 : launch_pair<2, 0>(s, gen0, nGen, mcmc, swapEvery, reevalFirst);
    if (e == cudaSuccess) s->launches++;
    return e;
  }
  if (C == 2)   // the factored evaluation has no incremental form
    e = S == 0    ? launch_variant<2, 0, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst)
        : S == 64 ? launch_variant<2, 64, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst)
                  : launch_variant<2, 256, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else if (C == 0 && S == 0) e = launch_incr<0, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else if (C == 1 && S == 0) e = launch_incr<1, 0>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else if (C == 0 && S == 64) e = launch_incr<0, 64>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else if (C == 1 && S == 64) e = launch_incr<1, 64>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else if (C == 0) e = launch_incr<0, 256>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  else e = launch_incr<1, 256>(s, grid, block, gen0, nGen, mcmc, swapEvery, reevalFirst);
  if (e == cudaSuccess) s->launches++;
  return e;
}

static p6_status check_device_flag(p6_wy_session *s) {
  int flag = 0;
  P6_CUDA(cudaMemcpyAsync(&flag, s->dErr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  if (flag == DEV_STAGE_TIMEOUT) return set_error(P6_ERR_TIMEOUT, "static-table staging did not complete in time");
  if (flag) return set_error(P6_ERR_CAPACITY, "device reported a capacity error");
  return P6_OK;
}

extern "C" {

const char *p6_last_error(void) { return g_err.c_str(); }
int p6_abi_version(void) { return 1; }
void p6_debug_inject_failure(int code, int after_calls) {
  g_inject_code = code;
  g_inject_after = code ? after_calls : -1;
}

p6_status p6_philox_device(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  clear_error();
  uint4 *d = nullptr;
  P6_CUDA(cudaMalloc(&d, sizeof(uint4)));
  philox_one<<<1, 1>>>(make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]), make_uint2(key[0], key[1]), d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(uint4), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_error(e, "philox_one");
  return P6_OK;
}

p6_status p6_wy_create(const p6_wy_problem *pr, int device, p6_wy_session **out) {
  P6_ENTRY();
  if (!pr || !out) return set_error(P6_ERR_INVALID_ARG, "null problem or output pointer");
  *out = nullptr;
  if (pr->num_particles <= 0 || pr->n_assign <= 0 || pr->n_tot <= 0 || pr->n_ops <= 0 || pr->max_sites <= 0)
    return set_error(P6_ERR_INVALID_ARG, "empty problem");
  if (!pr->gen_pack || !pr->sym_packed || !pr->site_proj || !pr->refl_pack || !pr->group_meta || !pr->f_tab ||
      !pr->restraint_tables)
    return set_error(P6_ERR_INVALID_ARG, "null table pointer");
  if (pr->max_sites > kMaxSites)
    return set_error(P6_ERR_CAPACITY, "more than 32 independent sites per assignment");
  if (pr->n_elem < 1 || pr->n_elem > kMaxElem) return set_error(P6_ERR_CAPACITY, "1 to 8 elements are supported");
  if (pr->n_ops > 4096) return set_error(P6_ERR_CAPACITY, "more than 4096 operators");
  if (pr->n_rules > kMaxRules) return set_error(P6_ERR_CAPACITY, "more than 32 distance rules");
  if (pr->max_coord_slots > 256) return set_error(P6_ERR_CAPACITY, "more than 256 neighbour slots");
  if (pr->group_stride != 3 && pr->group_stride != 4) return set_error(P6_ERR_INVALID_ARG, "group stride must be 3 or 4");
  if (!(pr->poly_prob >= 0.f && pr->poly_prob <= 1.f)) return set_error(P6_ERR_INVALID_ARG, "poly_prob must lie in [0, 1]");
  if (pr->n_tot > 4096) return set_error(P6_ERR_CAPACITY, "more than 4096 generated atoms");
  if (pr->cos_mode < 0 || pr->cos_mode > 2) return set_error(P6_ERR_INVALID_ARG, "cos_mode must be 0, 1 or 2");
  if (pr->cos_mode == 2 && pr->incremental == 1)
    return set_error(P6_ERR_INVALID_ARG, "the factored evaluation (cos_mode 2) has no incremental form");
  if (pr->incremental < -1 || pr->incremental > 1)
    return set_error(P6_ERR_INVALID_ARG, "incremental must be -1 (auto), 0 or 1");

  const int nA = pr->n_assign, nTot = pr->n_tot, ms = pr->max_sites, nE = pr->n_elem;
  // --- validate and convert host tables -----------------------------------
  std::vector<uint32_t> genR((size_t)nA * nTot);
  std::vector<int4> runs((size_t)nA * kMaxSites, make_int4(0, 0, 0, 0));
  std::vector<int> nRuns(nA), nF(nA);
  for (int A = 0; A < nA; ++A) {
    const uint32_t *g = pr->gen_pack + (size_t)A * nTot;
    int w = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int i = 0; i < nTot; ++i) {
        const uint32_t word = g[i];
        const int site = word & 0xFF, op = (word >> 8) & 0xFFF, skip = (word >> 24) & 1;
        if (site >= ms || op >= pr->n_ops)
          return set_error(P6_ERR_INVALID_ARG, "genPack entry names a site or operator out of range");
        if ((skip != 0) == (pass == 0)) continue;
        genR[(size_t)A * nTot + w++] = word;
      }
    int nf = 0, nr = 0;
    for (int i = 0; i < nTot; ++i)
      if (!((g[i] >> 24) & 1)) ++nf;
    for (int i = 0; i < nf; ++i) {
      const uint32_t word = genR[(size_t)A * nTot + i];
      const int site = word & 0xFF, ty = std::min<int>((word >> 20) & 0xF, nE - 1);
      if (nr > 0 && runs[(size_t)A * kMaxSites + nr - 1].w == site && runs[(size_t)A * kMaxSites + nr - 1].y == i) {
        runs[(size_t)A * kMaxSites + nr - 1].y = i + 1;
      } else {
        if (nr >= kMaxSites) return set_error(P6_ERR_CAPACITY, "a site's images are not contiguous in genPack");
        runs[(size_t)A * kMaxSites + nr++] = make_int4(i, i + 1, ty, site);
      }
    }
    nRuns[A] = nr;
    nF[A] = nf;
    // Inversion pairs: two images of one site whose positions sum to a lattice
    // vector at every point of the site's subspace have equal cosines and
    // opposite sines for every integer hkl.  Each run is reordered as
    // [leaders | singles | partners] and the number of pairs goes to bits 8+
    // of run.w; the |F|^2 sums read only the leaders (cosine counted twice,
    // sine cancelled) and the singles.  The test uses two generic points of
    // the subspace in FP64, so a pair holds wherever the site sits.
    for (int q = 0; q < nr; ++q) {
      int4 &run = runs[(size_t)A * kMaxSites + q];
      const int site = run.w, len = run.y - run.x;
      const float *pj = pr->site_proj + ((size_t)A * ms + site) * 12;
      double img[2][64][3];
      if (len > 64) continue;
      for (int p = 0; p < 2; ++p) {
        const double u[3] = {p ? 0.2718281 : 0.1234567, p ? 0.5772156 : 0.3456789, p ? 0.6931471 : 0.7654321};
        double x[3];
        for (int k = 0; k < 3; ++k)
          x[k] = (double)pj[3 * k] * u[0] + (double)pj[3 * k + 1] * u[1] + (double)pj[3 * k + 2] * u[2] + pj[9 + k];
        for (int i = 0; i < len; ++i) {
          const int op = (genR[(size_t)A * nTot + run.x + i] >> 8) & 0xFFF;
          const float *b = pr->sym_packed + op * 12;
          for (int k = 0; k < 3; ++k)
            img[p][i][k] = (double)b[3 * k] * x[0] + (double)b[3 * k + 1] * x[1] + (double)b[3 * k + 2] * x[2] + b[9 + k];
        }
      }
      auto inverse = [&](int i, int j) {
        for (int p = 0; p < 2; ++p)
          for (int k = 0; k < 3; ++k) {
            const double v = img[p][i][k] + img[p][j][k];
            if (std::fabs(v - std::floor(v + 0.5)) > 1e-7) return false;
          }
        return true;
      };
      int partner[64];
      for (int i = 0; i < len; ++i) partner[i] = -2;  // -2 unassigned, -1 single
      for (int i = 0; i < len; ++i) {
        if (partner[i] != -2) continue;
        partner[i] = -1;
        if (inverse(i, i)) continue;  // an image on an inversion centre stands alone
        for (int j = i + 1; j < len; ++j)
          if (partner[j] == -2 && inverse(i, j)) {
            partner[i] = j;
            partner[j] = i;
            break;
          }
      }
      std::vector<uint32_t> lead, single, part;
      for (int i = 0; i < len; ++i) {
        const uint32_t word = genR[(size_t)A * nTot + run.x + i];
        if (partner[i] < 0) single.push_back(word);
        else if (partner[i] > i) lead.push_back(word);
      }
      for (int i = 0; i < len; ++i)
        if (partner[i] >= 0 && partner[i] < i) part.push_back(genR[(size_t)A * nTot + run.x + i]);
      int w = run.x;
      for (uint32_t v : lead) genR[(size_t)A * nTot + w++] = v;
      for (uint32_t v : single) genR[(size_t)A * nTot + w++] = v;
      for (uint32_t v : part) genR[(size_t)A * nTot + w++] = v;
      run.w = site | ((int)lead.size() << 8);
    }
  }
  std::vector<OpFix> ops(pr->n_ops);
  for (int o = 0; o < pr->n_ops; ++o) {
    const float *b = pr->sym_packed + o * 12;
    for (int k = 0; k < 9; ++k) {
      const double v = b[k];
      if (std::fabs(v - std::floor(v + 0.5)) > 1e-6)
        return set_error(P6_ERR_INVALID_ARG, "operator with a non-integer rotation part");
      ops[o].r[k] = (int)std::floor(v + 0.5);
    }
    for (int k = 0; k < 3; ++k) ops[o].t[k] = trans_fixed(b[9 + k]);
  }
  std::vector<ProjFix> proj((size_t)nA * ms);
  std::vector<uint32_t> freeMask(nA, 0);
  for (int A = 0; A < nA; ++A)
    for (int si = 0; si < ms; ++si) {
      const float *b = pr->site_proj + ((size_t)A * ms + si) * 12;
      ProjFix &f = proj[(size_t)A * ms + si];
      if (!rationalise(b, 9, f.num, &f.den))
        return set_error(P6_ERR_INVALID_ARG, "a Wyckoff projector is not a rational matrix with denominator <= 24");
      for (int k = 0; k < 3; ++k) f.t[k] = trans_fixed(b[9 + k]);
      f.pad[0] = f.pad[1] = 0;
      if (f.den == 1) {
        bool diag = true;
        for (int k = 0; k < 9 && diag; ++k)
          diag = (k % 4 == 0) ? (f.num[k] == 0 || f.num[k] == 1) : f.num[k] == 0;
        f.pad[0] = diag ? 1 : 0;
      }
      double norm = 0;
      for (int k = 0; k < 9; ++k) norm += std::fabs(b[k]);
      if (norm > 1e-6) freeMask[A] |= 1u << si;
    }
  // --- factored FP64 structure factors (cos mode 2) ---------------------------
  const bool factored = pr->cos_mode == 2;
  const int nReflPad = (pr->n_refl + 3) & ~3;
  int nMono = 0, axE[3] = {1, 1, 1}, axOff[3] = {0, 0, 0}, tabLen = 0, tabE = 0;
  bool complexK = false;
  std::vector<double> monoRe, monoIm, f64;
  std::vector<uint32_t> monoIdx;
  if (factored) {
    for (int o = 0; o < pr->n_ops; ++o)
      for (int k = 0; k < 9; ++k)
        if (k % 4 != 0 && ops[o].r[k] != 0)
          return set_error(P6_ERR_INVALID_ARG,
                           "the factored evaluation (cos_mode 2) needs a group whose rotations are all diagonal");
    for (int A = 0; A < nA; ++A) {
      uint32_t seen = 0;
      for (int q = 0; q < nRuns[A]; ++q) {
        const int site = runs[(size_t)A * kMaxSites + q].w & 0xFF;
        if (seen & (1u << site))
          return set_error(P6_ERR_INVALID_ARG, "factored evaluation: a site's images are not contiguous");
        seen |= 1u << site;
      }
    }
    // operators modulo the centring translations (translations in 1/24, exact)
    std::vector<std::array<int, 3>> tn(pr->n_ops);
    for (int o = 0; o < pr->n_ops; ++o)
      for (int k = 0; k < 3; ++k) {
        const double v = (double)pr->sym_packed[o * 12 + 9 + k] * 24.0;
        tn[o][k] = (((int)std::floor(v + 0.5)) % 24 + 24) % 24;
      }
    std::vector<int> cen, reps;
    for (int o = 0; o < pr->n_ops; ++o)
      if (ops[o].r[0] == 1 && ops[o].r[4] == 1 && ops[o].r[8] == 1) cen.push_back(o);
    for (int o = 0; o < pr->n_ops; ++o) {
      bool dup = false;
      for (int j : reps) {
        if (ops[j].r[0] != ops[o].r[0] || ops[j].r[4] != ops[o].r[4] || ops[j].r[8] != ops[o].r[8]) continue;
        for (int c : cen) {
          bool same = true;
          for (int k = 0; k < 3; ++k) same &= ((tn[o][k] - tn[j][k] - tn[c][k]) % 24 + 48) % 24 == 0;
          if (same) { dup = true; break; }
        }
        if (dup) break;
      }
      if (!dup) reps.push_back(o);
    }
    std::vector<std::array<int, 3>> hkl(pr->n_refl);
    for (int r = 0; r < pr->n_refl; ++r) {
      const uint32_t pk = pr->refl_pack[2 * r];
      hkl[r] = {(int)(pk & 0x3FF) - 512, (int)((pk >> 10) & 0x3FF) - 512, (int)((pk >> 20) & 0x3FF) - 512};
      for (int a = 0; a < 3; ++a) axE[a] = std::max(axE[a], std::abs(hkl[r][a]) + 1);
    }
    axOff[0] = 0;
    axOff[1] = 2 * axE[0];
    axOff[2] = axOff[1] + 2 * axE[1];
    tabLen = axOff[2] + 2 * axE[2];
    tabE = axE[0] + axE[1] + axE[2];
    if (tabLen > 1024) return set_error(P6_ERR_CAPACITY, "factored evaluation: Miller indices too large for the site tables");
    // K_m(h) = (1/N_p) sum_j e^{2 pi i h.t_j} prod_{a in m} (i sigma_ja sgn h_a)
    const double kTwoPi = 6.283185307179586476925286766559;
    std::vector<std::vector<std::pair<int, std::pair<double, double>>>> mono(pr->n_refl);
    for (int r = 0; r < pr->n_refl; ++r) {
      const int *h = hkl[r].data();
      for (int m = 0; m < 8; ++m) {
        bool zero = false;
        for (int a = 0; a < 3; ++a) zero |= ((m >> a) & 1) && h[a] == 0;
        if (zero) continue;
        double re = 0.0, im = 0.0;
        for (int j : reps) {
          const int ph = ((h[0] * tn[j][0] + h[1] * tn[j][1] + h[2] * tn[j][2]) % 24 + 24) % 24;
          double cr = std::cos(kTwoPi * ph / 24.0), ci = std::sin(kTwoPi * ph / 24.0);
          for (int a = 0; a < 3; ++a)
            if ((m >> a) & 1) {   // times i sigma sgn(h): (cr + i ci) i g = -ci g + i cr g
              const double g = (double)ops[j].r[4 * a] * (h[a] > 0 ? 1.0 : -1.0);
              const double nr = -ci * g, ni = cr * g;
              cr = nr;
              ci = ni;
            }
          re += cr;
          im += ci;
        }
        re /= (double)reps.size();
        im /= (double)reps.size();
        if (std::fabs(re) < 1e-9) re = 0.0;
        if (std::fabs(im) < 1e-9) im = 0.0;
        if (re != 0.0 || im != 0.0) mono[r].push_back({m, {re, im}});
        complexK |= im != 0.0;
      }
      nMono = std::max(nMono, (int)mono[r].size());
    }
    nMono = std::max(nMono, 1);
    if (nMono > 4)
      return set_error(P6_ERR_INVALID_ARG, "factored evaluation: more than four monomials per reflection "
                                           "(use cos_mode 0 or 1 for this group)");
    monoRe.assign((size_t)nMono * nReflPad, 0.0);
    monoIm.assign(complexK ? (size_t)nMono * nReflPad : 0, 0.0);
    monoIdx.assign((size_t)nMono * nReflPad, 0u);
    for (int r = 0; r < pr->n_refl; ++r)
      for (size_t k = 0; k < mono[r].size(); ++k) {
        const int m = mono[r][k].first;
        uint32_t word = 0;
        for (int a = 0; a < 3; ++a)
          word |= (uint32_t)(axOff[a] + ((m >> a) & 1) * axE[a] + std::abs(hkl[r][a])) << (10 * a);
        monoRe[k * nReflPad + r] = mono[r][k].second.first;
        if (complexK) monoIm[k * nReflPad + r] = mono[r][k].second.second;
        monoIdx[k * nReflPad + r] = word;
      }
    f64.assign((size_t)nE * nReflPad, 0.0);
    for (int r = 0; r < pr->n_refl; ++r)
      for (int t = 0; t < nE; ++t) f64[(size_t)t * nReflPad + r] = (double)pr->f_tab[(size_t)r * nE + t];
  }
  // --- static blob: reflections | f table | groups | rMin | soo prefix | ops | pairs [| factored] ---
  auto pad16 = [](size_t n) { return (n + 15) & ~(size_t)15; };
  // Clash pairs.  The space group maps the cell's atoms onto themselves, and
  // rounding in the reduced basis is the nearest image out to every
  // threshold (otherwise the minimum-image shell search is on), so all the
  // images of one site see the same neighbours: the pairs (rep_s, j), j != rep_s,
  // with weight m_s / 2 (m_s = the site's atoms in the cell) give the sum over
  // all pairs i < j from nSites x (nTot - 1) distances instead of nTot^2 / 2.
  std::vector<uint32_t> repPairs;
  std::vector<int2> pairRange(nA);
  bool useRep = true;
  for (int A = 0; A < nA && useRep; ++A) {
    std::vector<int> first(ms, -1), mult(ms, 0);
    for (int i = 0; i < nTot; ++i) {
      const int s = genR[(size_t)A * nTot + i] & 0xFF;
      if (first[s] < 0) first[s] = i;
      ++mult[s];
    }
    pairRange[A].x = (int)repPairs.size();
    for (int s = 0; s < ms && useRep; ++s) {
      if (!mult[s]) continue;
      if (mult[s] > 255) useRep = false;
      for (int j = 0; j < nTot && useRep; ++j)
        if (j != first[s]) repPairs.push_back((uint32_t)first[s] | ((uint32_t)j << 12) | ((uint32_t)mult[s] << 24));
    }
    pairRange[A].y = (int)repPairs.size() - pairRange[A].x;
    if (repPairs.size() > 4608) useRep = false;
  }
  if (!useRep) repPairs.clear();
  const int nPairs = useRep ? 0 : (nTot <= 96 ? nTot * (nTot - 1) / 2 : 0);
  const size_t pairWords = useRep ? repPairs.size() : (size_t)nPairs;
  const size_t offRefl = 0, szRefl = pad16((size_t)pr->n_refl * sizeof(ReflRec));
  const size_t offF = offRefl + szRefl, szF = pad16((size_t)pr->n_refl * nE * sizeof(float));
  const size_t offG = offF + szF, szG = pad16((size_t)pr->n_groups * sizeof(float4));
  const size_t offR = offG + szG, szR = pad16((size_t)nE * nE * sizeof(float));
  const size_t offS = offR + szR, szS = pad16((size_t)(pr->n_groups + 1) * sizeof(double));
  const size_t offO = offS + szS, szO = pad16((size_t)pr->n_ops * sizeof(OpFix));
  const size_t offP = offO + szO, szP = pad16(pairWords * sizeof(uint32_t));
  const size_t offK = offP + szP, szK = pad16(monoRe.size() * sizeof(double));
  const size_t offKi = offK + szK, szKi = pad16(monoIm.size() * sizeof(double));
  const size_t offIdx = offKi + szKi, szIdx = pad16(monoIdx.size() * sizeof(uint32_t));
  const size_t offF64 = offIdx + szIdx, szF64 = pad16(f64.size() * sizeof(double));
  const size_t blobBytes = offF64 + szF64;
  std::vector<unsigned char> blob(blobBytes, 0);
  for (int r = 0; r < pr->n_refl; ++r) {
    const uint32_t pk = pr->refl_pack[2 * r];
    ReflRec rec;
    rec.h = (short)((int)(pk & 0x3FF) - 512);
    rec.k = (short)((int)((pk >> 10) & 0x3FF) - 512);
    rec.l = (short)((int)((pk >> 20) & 0x3FF) - 512);
    const uint32_t m = pr->refl_pack[2 * r + 1];
    if (m > 65535) return set_error(P6_ERR_INVALID_ARG, "multiplicity out of range");
    rec.mult = (unsigned short)m;
    std::memcpy(&blob[offRefl + r * sizeof(ReflRec)], &rec, sizeof(rec));
  }
  std::memcpy(&blob[offF], pr->f_tab, (size_t)pr->n_refl * nE * sizeof(float));
  std::vector<double> soo(pr->n_groups + 1, 0.0);
  for (int gI = 0; gI < pr->n_groups; ++gI) {
    const float *gm = pr->group_meta + (size_t)gI * pr->group_stride;
    float4 v = make_float4(gm[0], gm[1], gm[2], pr->group_stride >= 4 ? gm[3] : 1.0f);
    if (v.x < 0 || v.y < 0 || (int)v.x + (int)v.y > pr->n_refl)
      return set_error(P6_ERR_INVALID_ARG, "group range outside the reflection list");
    if (gI > 0) {
      const float *pg = pr->group_meta + (size_t)(gI - 1) * pr->group_stride;
      if ((int)v.x != (int)pg[0] + (int)pg[1])
        return set_error(P6_ERR_INVALID_ARG, "groups must be contiguous and in order");
    }
    std::memcpy(&blob[offG + gI * sizeof(float4)], &v, sizeof(v));
    // sum of w Iobs^2 over the first gI+1 groups: constant for a given number of active groups
    soo[gI + 1] = soo[gI] + ((v.w > 0.f) ? (double)v.w * (double)v.z * (double)v.z : 0.0);
  }
  std::memcpy(&blob[offS], soo.data(), soo.size() * sizeof(double));
  for (int i = 0; i < nE * nE; ++i) {
    const float v = pr->restraint_tables[pr->r_min_off + i];
    std::memcpy(&blob[offR + i * sizeof(float)], &v, sizeof(float));
  }
  std::memcpy(&blob[offO], ops.data(), ops.size() * sizeof(OpFix));
  {
    int q = 0;
    if (useRep && !repPairs.empty()) std::memcpy(&blob[offP], repPairs.data(), repPairs.size() * sizeof(uint32_t));
    for (int i = 0; i < nTot && nPairs; ++i)
      for (int j = i + 1; j < nTot; ++j) {
        const uint32_t v = (uint32_t)i | ((uint32_t)j << 16);
        std::memcpy(&blob[offP + (size_t)(q++) * sizeof(uint32_t)], &v, sizeof(v));
      }
  }
  if (factored) {
    std::memcpy(&blob[offK], monoRe.data(), monoRe.size() * sizeof(double));
    if (complexK) std::memcpy(&blob[offKi], monoIm.data(), monoIm.size() * sizeof(double));
    std::memcpy(&blob[offIdx], monoIdx.data(), monoIdx.size() * sizeof(uint32_t));
    std::memcpy(&blob[offF64], f64.data(), f64.size() * sizeof(double));
  }
  std::vector<RuleDev> rules(std::max(pr->n_rules, 1));
  for (int k = 0; k < pr->n_rules; ++k) {
    const float *rb = pr->restraint_tables + pr->rule_off + 7 * k;
    rules[k] = RuleDev{(int)rb[0], (int)rb[1], rb[2], rb[3], rb[4], (int)rb[5], (int)rb[6], 0};
  }
  // --- shared memory plan ----------------------------------------------------
  // Per warp: state and run tables, the assignment's genPack row and projectors,
  // one or two atom banks, |F|^2 per reflection, and (incremental) two banks of
  // site sums (only when the caller asks for incremental evaluation).
  const int rungs = 8;
  const int comp = pr->centro ? 1 : 2;
  const size_t curOff = 32;
  const size_t propOff = curOff + (((size_t)ms * 3 * sizeof(uint32_t) + 15) & ~(size_t)15);
  const size_t runsOff = propOff + (((size_t)ms * 3 * sizeof(uint32_t) + 15) & ~(size_t)15);
  const size_t slotOff = runsOff + (size_t)ms * sizeof(int4);
  const size_t genOff = slotOff + (((size_t)(ms + 1) * sizeof(int) + 15) & ~(size_t)15);
  const size_t projOff = (genOff + (size_t)nTot * sizeof(uint32_t) + 15) & ~(size_t)15;
  const size_t atomsOff = (projOff + (size_t)ms * sizeof(ProjFix) + 15) & ~(size_t)15;
  const size_t icOff = atomsOff + (size_t)nTot * sizeof(uint4);
  // the factored evaluation keeps FP64 |F|^2 and, per site, its axis tables and their coordinate tags
  const size_t icEnd = icOff + (size_t)nReflPad * (factored ? sizeof(double) : sizeof(float));
  const size_t tabOff = (icEnd + 15) & ~(size_t)15;
  const size_t tagOff = tabOff + (factored ? (size_t)2 * ms * tabLen * sizeof(double) : 0);
  // two banks of tags, then the table offset each run reads
  const size_t fragOff =
      ((factored ? tagOff + (size_t)2 * ms * sizeof(uint4) + (size_t)ms * sizeof(int) : icEnd) + 15) & ~(size_t)15;
  const size_t baseEnd = fragOff + 2 * kFragParams * sizeof(float);   // fragment parameters: current, proposed
  const size_t atoms2Off = (baseEnd + 15) & ~(size_t)15;
  const size_t cbOff = atoms2Off + (size_t)nTot * sizeof(uint4);
  const size_t incrEnd = cbOff + (size_t)(ms + 1) * nReflPad * comp * sizeof(float);
  const size_t blobPadded = (blobBytes + 127) & ~(size_t)127;
  const size_t smemFull = blobPadded + ((baseEnd + 127) & ~(size_t)127) * rungs;
  const size_t smemIncr = blobPadded + ((incrEnd + 127) & ~(size_t)127) * rungs;
  const bool incrFits4 = smemIncr <= (size_t)56 * 1024;
  // Auto keeps the full evaluation: on the benchmark problem the gather of cached
  // sums measured slower than recomputing every image (75.5 vs 66.8 ms per search).
  const int useIncr = pr->incremental < 0 ? 0 : (pr->incremental ? 1 : 0);
  if (useIncr && !incrFits4 && smemIncr > (size_t)200 * 1024)
    return set_error(P6_ERR_CAPACITY, "incremental site sums do not fit in shared memory");
  const size_t warpBytes = ((useIncr ? incrEnd : baseEnd) + 127) & ~(size_t)127;
  size_t smem = useIncr ? smemIncr : smemFull;

  p6_wy_session *s = new p6_wy_session();
  s->device = device;
  s->cosMode = pr->cos_mode;
  s->incremental = useIncr;
  const int slotsNeeded = pr->n_rules > 0 ? (pr->max_coord_slots <= 64 ? 64 : 256) : 0;
  s->slots = slotsNeeded;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaSetDevice"); }
  int smemOptin = 0, nSM = 0;
  cudaDeviceGetAttribute(&smemOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, device);
  // Shared memory: the staged tables once, plus one slice per rung (8 warps);
  // when both do not fit, the tables stay in global memory.
  int blobGlobal = 0;
  if (!useIncr && (int)smem > smemOptin - 1024 && (int)(warpBytes * rungs) <= smemOptin - 1024) {
    blobGlobal = 1;
    smem = warpBytes * rungs;
  }
  if ((int)smem > smemOptin - 1024) {
    free_session(s);
    return set_error(P6_ERR_CAPACITY, "the reflection table and generated cell do not fit in shared memory");
  }
  s->smemBytes = (int)smem;
  s->smemPair = (int)((blobGlobal ? 0 : blobPadded) + warpBytes * (rungs / 2));
  p6_status st;
#define P6_TRY(x)                   \
  do {                              \
    st = (x);                       \
    if (st != P6_OK) {              \
      free_session(s);              \
      return st;                    \
    }                               \
  } while (0)
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaStreamCreate"); }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  P6_TRY(upload(&s->dGen, genR.data(), genR.size(), s->stream));
  P6_TRY(upload(&s->dGenOrig, pr->gen_pack, (size_t)nA * nTot, s->stream));
  P6_TRY(upload(&s->dRuns, runs.data(), runs.size(), s->stream));
  if (useRep) P6_TRY(upload(&s->dPairRange, pairRange.data(), pairRange.size(), s->stream));
  P6_TRY(upload(&s->dNRuns, nRuns.data(), nRuns.size(), s->stream));
  P6_TRY(upload(&s->dNF, nF.data(), nF.size(), s->stream));
  P6_TRY(upload(&s->dFree, freeMask.data(), freeMask.size(), s->stream));
  P6_TRY(upload(&s->dOps, ops.data(), ops.size(), s->stream));
  P6_TRY(upload(&s->dProj, proj.data(), proj.size(), s->stream));
  s->projHost = proj;
  s->groupsHost.resize(pr->n_groups);
  for (int gI = 0; gI < pr->n_groups; ++gI) {
    const float *gm = pr->group_meta + (size_t)gI * pr->group_stride;
    s->groupsHost[gI] = make_float4(gm[0], gm[1], gm[2], pr->group_stride >= 4 ? gm[3] : 1.0f);
  }
  P6_TRY(upload(&s->dBlob, blob.data(), blob.size(), s->stream));
  P6_TRY(upload(&s->dRules, rules.data(), rules.size(), s->stream));
  const size_t posWords = (size_t)2 * pr->num_particles * ms * 3;
  e = cudaMalloc(&s->dPos, posWords * sizeof(uint32_t));
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaMalloc positions"); }
  cudaMemsetAsync(s->dPos, 0, posWords * sizeof(uint32_t), s->stream);
  e = cudaMalloc(&s->dSt, (size_t)pr->num_particles * sizeof(PState));
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaMalloc state"); }
  cudaMemsetAsync(s->dSt, 0, (size_t)pr->num_particles * sizeof(PState), s->stream);
  std::vector<uint32_t> assign0(pr->num_particles, 0);
  P6_TRY(upload(&s->dAssign, assign0.data(), assign0.size(), s->stream));
  s->hostAssign = assign0;
  e = cudaMalloc(&s->dErr, sizeof(int));
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaMalloc flag"); }
  cudaMemsetAsync(s->dErr, 0, sizeof(int), s->stream);
  e = cudaMalloc(&s->dSwap, 2 * sizeof(unsigned long long));
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "cudaMalloc swap stats"); }
  cudaMemsetAsync(s->dSwap, 0, 2 * sizeof(unsigned long long), s->stream);

  Params &P = s->P;
  P.gen = s->dGen;
  P.genOrig = s->dGenOrig;
  P.runs = s->dRuns;
  P.nRuns = s->dNRuns;
  P.nF = s->dNF;
  P.freeMask = s->dFree;
  P.ops = s->dOps;
  P.proj = s->dProj;
  P.blob = s->dBlob;
  P.blobBytes = (int)blobBytes;
  P.offRefl = (int)offRefl;
  P.offF = (int)offF;
  P.offGroup = (int)offG;
  P.offRmin = (int)offR;
  P.offSoo = (int)offS;
  P.offOps = (int)offO;
  P.offPairs = (int)offP;
  P.nPairs = nPairs;
  P.pairRange = useRep ? s->dPairRange : nullptr;
  P.rules = s->dRules;
  P.nRules = pr->n_rules;
  P.numParticles = pr->num_particles;
  P.nTot = nTot;
  P.maxSites = ms;
  P.nRefl = pr->n_refl;
  P.nGroups = pr->n_groups;
  P.nElem = nE;
  P.nAssign = nA;
  bool counted = false;
  for (int k = 0; k < pr->n_rules; ++k) counted |= (int)pr->restraint_tables[pr->rule_off + 7 * k + 5] != 0;
  P.polyProb = counted ? pr->poly_prob : 0.f;   // no counted rule: nothing to move as a unit
  for (int i = 0; i < 9; ++i) {
    P.invOrth[i] = (float)pr->inv_orth[i];
    P.orth[i] = (float)pr->orth[i];
    const double x = pr->xform[i];
    if (std::fabs(x - std::floor(x + 0.5)) > 1e-9) {
      free_session(s);
      return set_error(P6_ERR_INVALID_ARG, "xform must be an integer matrix");
    }
    P.xf[i] = (int)std::floor(x + 0.5);
  }
  P.minImageShell = pr->min_image_shell ? 1 : 0;
  P.countShell = pr->count_shell ? 1 : 0;
  P.centro = pr->centro;
  P.maxCoordSlots = pr->max_coord_slots;
  P.geomSlots = pr->geom_slots;
  P.penClash = pr->pen_clash;
  P.penBond = pr->pen_bond;
  P.penCoord = pr->pen_coord;
  P.penGeom = pr->pen_geom;
  P.stepUp = pr->step_up;
  P.stepDown = pr->step_down;
  P.stepMin = pr->step_min;
  P.stepMax = pr->step_max;
  P.runKey = pr->run_key;
  P.pos = s->dPos;
  P.st = s->dSt;
  P.assign = s->dAssign;
  P.ladders = nullptr;
  P.rungs = 8;
  P.nLadders = (pr->num_particles + 7) / 8;
  P.schedGroups = nullptr;
  P.schedPen = nullptr;
  P.ngaArg = pr->n_groups;
  P.penArg = 1.0f;
  P.swapStats = s->dSwap;
  P.errFlag = s->dErr;
  P.warpSmemBytes = (int)warpBytes;
  P.blobGlobal = blobGlobal;
  P.offK = (int)offK;
  P.offKi = complexK ? (int)offKi : -1;
  P.offIdx = (int)offIdx;
  P.offF64 = (int)offF64;
  P.nMono = nMono;
  P.tabLen = tabLen;
  P.tabE = tabE;
  for (int a = 0; a < 3; ++a) {
    P.axE[a] = axE[a];
    P.axOff[a] = axOff[a];
  }
  P.tabOff = (int)tabOff;
  P.tagOff = (int)tagOff;
  P.traceSums = nullptr;
  P.frag = nullptr;
  P.fragState = nullptr;
  P.fragBest = nullptr;
  P.fragOff = (int)fragOff;
  P.genOff = (int)genOff;
  P.projOff = (int)projOff;
  P.atomsOff = (int)atomsOff;
  P.icOff = (int)icOff;
  P.cbOff = (int)cbOff;
  P.atoms2Off = (int)atoms2Off;
  P.nReflPad = nReflPad;
  P.curOff = (int)curOff;
  P.propOff = (int)propOff;
  P.runsOff = (int)runsOff;
  P.slotOff = (int)slotOff;
  s->nga = pr->n_groups;
  // Resident CTAs: the persistent grid covers the GPU once.
  int occ = 0;
  if (useIncr) {
    cudaFuncSetAttribute(wy_kernel<0, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemBytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wy_kernel<0, 0, 1>, 256, s->smemBytes);
  } else {
    cudaFuncSetAttribute(wy_kernel<0, 0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, s->smemBytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wy_kernel<0, 0, 0>, 256, s->smemBytes);
  }
  s->maxGrid = std::max(1, occ) * std::max(1, nSM);
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) { free_session(s); return cuda_error(e, "session upload"); }
  *out = s;
  return P6_OK;
#undef P6_TRY
}

p6_status p6_wy_destroy(p6_wy_session *s) {
  clear_error();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  free_session(s);
  return P6_OK;
}

p6_status p6_wy_set_assign(p6_wy_session *s, const uint32_t *assign_of) {
  P6_ENTRY();
  if (!s || !assign_of) return set_error(P6_ERR_INVALID_ARG, "null argument");
  for (int i = 0; i < s->P.numParticles; ++i)
    if ((int)assign_of[i] >= s->P.nAssign) return set_error(P6_ERR_INVALID_ARG, "assignment index out of range");
  P6_CUDA(cudaSetDevice(s->device));
  s->hostAssign.assign(assign_of, assign_of + s->P.numParticles);
  P6_CUDA(cudaMemcpyAsync(s->dAssign, s->hostAssign.data(), s->hostAssign.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_set_params(p6_wy_session *s, int n_groups_active, float pen_scale) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  s->nga = n_groups_active;
  s->penScale = pen_scale;
  return P6_OK;
}

static p6_status write_positions_f32(p6_wy_session *s, const float *positions, bool resetBest) {
  const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
  std::vector<uint32_t> fx(resetBest ? 2 * n : n);
  for (size_t i = 0; i < n; ++i) fx[i] = to_fixed(positions[i]);
  if (resetBest)
    for (size_t i = 0; i < n; ++i) fx[n + i] = fx[i];
  P6_CUDA(cudaMemcpyAsync(s->dPos, fx.data(), fx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_sync_state(p6_wy_session *s, const float *positions, const p6_wy_particle_state *state) {
  P6_ENTRY();
  if (!s || !positions || !state) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(s->device));
  p6_status st = write_positions_f32(s, positions, true);
  if (st != P6_OK) return st;
  P6_CUDA(cudaMemcpyAsync(s->dSt, state, (size_t)s->P.numParticles * sizeof(PState), cudaMemcpyHostToDevice,
                          s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_read_state(p6_wy_session *s, float *positions, float *best_positions, p6_wy_particle_state *state) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
  std::vector<uint32_t> fx(2 * n);
  P6_CUDA(cudaMemcpyAsync(fx.data(), s->dPos, fx.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  if (state)
    P6_CUDA(cudaMemcpyAsync(state, s->dSt, (size_t)s->P.numParticles * sizeof(PState), cudaMemcpyDeviceToHost,
                            s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  if (positions)
    for (size_t i = 0; i < n; ++i) positions[i] = from_fixed(fx[i]);
  if (best_positions)
    for (size_t i = 0; i < n; ++i) best_positions[i] = from_fixed(fx[n + i]);
  return P6_OK;
}

p6_status p6_wy_write_positions_fixed(p6_wy_session *s, const uint32_t *current) {
  P6_ENTRY();
  if (!s || !current) return set_error(P6_ERR_INVALID_ARG, "null argument");
  const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
  P6_CUDA(cudaMemcpyAsync(s->dPos, current, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaMemcpyAsync(s->dPos + n, current, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_set_ladder_split(p6_wy_session *s, int ctas_per_ladder) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (ctas_per_ladder != 1 && ctas_per_ladder != 2) return set_error(P6_ERR_INVALID_ARG, "ctas_per_ladder must be 1 or 2");
  s->ladderSplit = ctas_per_ladder;
  return P6_OK;
}

p6_status p6_wy_write_state_fixed(p6_wy_session *s, const uint32_t *current, const uint32_t *best,
                                  const p6_wy_particle_state *state) {
  P6_ENTRY();
  if (!s || !current || !best || !state) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
  P6_CUDA(cudaMemcpyAsync(s->dPos, current, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaMemcpyAsync(s->dPos + n, best, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaMemcpyAsync(s->dSt, state, (size_t)s->P.numParticles * sizeof(PState), cudaMemcpyHostToDevice,
                          s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_read_positions_fixed(p6_wy_session *s, uint32_t *current, uint32_t *best) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
  if (current) P6_CUDA(cudaMemcpyAsync(current, s->dPos, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  if (best) P6_CUDA(cudaMemcpyAsync(best, s->dPos + n, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_set_trace(p6_wy_session *s, int enable) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (enable && !s->dTracePos) {
    P6_CUDA(cudaMalloc(&s->dTracePos, (size_t)s->P.numParticles * s->P.maxSites * 3 * sizeof(uint32_t)));
    P6_CUDA(cudaMalloc(&s->dTraceRec, (size_t)s->P.numParticles * 8 * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dTraceIc, (size_t)s->P.numParticles * std::max(s->P.nRefl, 1) * sizeof(float)));
    P6_CUDA(cudaMemsetAsync(s->dTraceIc, 0, (size_t)s->P.numParticles * std::max(s->P.nRefl, 1) * sizeof(float),
                            s->stream));
    P6_CUDA(cudaMalloc(&s->dTraceSums, (size_t)s->P.numParticles * 3 * sizeof(double)));
    P6_CUDA(cudaMemsetAsync(s->dTraceSums, 0, (size_t)s->P.numParticles * 3 * sizeof(double), s->stream));
  }
  s->trace = enable != 0;
  return P6_OK;
}

p6_status p6_wy_read_trace(p6_wy_session *s, uint32_t *proposals, float *records) {
  P6_ENTRY();
  if (!s || !s->dTracePos) return set_error(P6_ERR_INVALID_ARG, "tracing was not enabled");
  P6_CUDA(cudaSetDevice(s->device));
  if (proposals)
    P6_CUDA(cudaMemcpyAsync(proposals, s->dTracePos, (size_t)s->P.numParticles * s->P.maxSites * 3 * 4,
                            cudaMemcpyDeviceToHost, s->stream));
  if (records)
    P6_CUDA(cudaMemcpyAsync(records, s->dTraceRec, (size_t)s->P.numParticles * 8 * 4, cudaMemcpyDeviceToHost,
                            s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

static p6_status dispatch_impl(p6_wy_session *s, int mcmc) {
  Params &P = s->P;
  Params saved = P;
  P.ladders = nullptr;
  P.rungs = 8;
  P.nLadders = (P.numParticles + 7) / 8;
  P.schedGroups = nullptr;
  P.schedPen = nullptr;
  P.ngaArg = s->nga;
  P.penArg = s->penScale;
  P.tracePos = s->trace ? s->dTracePos : nullptr;
  P.traceRec = s->trace ? s->dTraceRec : nullptr;
  P.traceIc = s->trace ? s->dTraceIc : nullptr;
  P.traceSums = s->trace ? s->dTraceSums : nullptr;
  P6_CUDA(cudaEventRecord(s->ev0, s->stream));
  cudaError_t e = launch(s, 0, 1, mcmc, 0, 0);
  P = saved;
  if (e != cudaSuccess) return cuda_error(e, "wy_kernel launch");
  P6_CUDA(cudaEventRecord(s->ev1, s->stream));
  return P6_OK;
}

p6_status p6_wy_dispatch(p6_wy_session *s, const float *coords, int mcmc) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (coords) {
    const size_t n = (size_t)s->P.numParticles * s->P.maxSites * 3;
    std::vector<uint32_t> fx(n);
    for (size_t i = 0; i < n; ++i) fx[i] = to_fixed(coords[i]);
    P6_CUDA(cudaMemcpyAsync(s->dPos, fx.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    P6_CUDA(cudaStreamSynchronize(s->stream));
  }
  return dispatch_impl(s, mcmc);
}

p6_status p6_wy_evaluate_sync(p6_wy_session *s, const float *coords, int mcmc, float *fit_cc) {
  P6_ENTRY();
  if (!s || !fit_cc) return set_error(P6_ERR_INVALID_ARG, "null argument");
  p6_status st = p6_wy_dispatch(s, coords, mcmc);
  if (st != P6_OK) return st;
  std::vector<PState> h(s->P.numParticles);
  P6_CUDA(cudaMemcpyAsync(h.data(), s->dSt, h.size() * sizeof(PState), cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  for (int i = 0; i < s->P.numParticles; ++i) {
    fit_cc[i] = h[i].fit;
    fit_cc[s->P.numParticles + i] = h[i].cc;
  }
  return check_device_flag(s);
}

p6_status p6_wy_set_ladders(p6_wy_session *s, const int32_t *ladders, int n_ladders, int rungs) {
  P6_ENTRY();
  if (!s || !ladders || n_ladders <= 0) return set_error(P6_ERR_INVALID_ARG, "null or empty ladder table");
  if (rungs < 1 || rungs > 8) return set_error(P6_ERR_INVALID_ARG, "rungs must be 1..8 (one warp per rung)");
  std::vector<int> seen(s->P.numParticles, 0);
  for (int i = 0; i < n_ladders * rungs; ++i) {
    const int p = ladders[i];
    if (p < -1 || p >= s->P.numParticles) return set_error(P6_ERR_INVALID_ARG, "ladder entry out of range");
    if (p >= 0 && seen[p]++) return set_error(P6_ERR_INVALID_ARG, "a particle appears in two ladder slots");
  }
  P6_CUDA(cudaSetDevice(s->device));
  if (s->dLadders) cudaFree(s->dLadders);
  s->dLadders = nullptr;
  p6_status st = upload(&s->dLadders, ladders, (size_t)n_ladders * rungs, s->stream);
  if (st != P6_OK) return st;
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->nLadders = n_ladders;
  s->rungs = rungs;
  return P6_OK;
}

p6_status p6_wy_set_schedule(p6_wy_session *s, const int32_t *sched_groups, const float *sched_pen, int n_gen) {
  P6_ENTRY();
  if (!s || !sched_groups || !sched_pen || n_gen <= 0) return set_error(P6_ERR_INVALID_ARG, "empty schedule");
  P6_CUDA(cudaSetDevice(s->device));
  if (s->dSchedG) cudaFree(s->dSchedG);
  if (s->dSchedP) cudaFree(s->dSchedP);
  s->dSchedG = nullptr;
  s->dSchedP = nullptr;
  p6_status st = upload(&s->dSchedG, sched_groups, (size_t)n_gen, s->stream);
  if (st != P6_OK) return st;
  st = upload(&s->dSchedP, sched_pen, (size_t)n_gen, s->stream);
  if (st != P6_OK) return st;
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->schedLen = n_gen;
  s->schedPenHost.assign(sched_pen, sched_pen + n_gen);
  return P6_OK;
}

p6_status p6_wy_set_quench(p6_wy_session *s, const float *step_sd, int n_gen) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (s->dQuench) cudaFree(s->dQuench);
  s->dQuench = nullptr;
  s->quenchLen = 0;
  if (!step_sd) return P6_OK;
  if (n_gen <= 0) return set_error(P6_ERR_INVALID_ARG, "empty quench schedule");
  p6_status st = upload(&s->dQuench, step_sd, (size_t)n_gen, s->stream);
  if (st != P6_OK) return st;
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->quenchLen = n_gen;
  return P6_OK;
}

p6_status p6_wy_run(p6_wy_session *s, int gen0, int n_gen, int swap_every, int reeval_first) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (!s->dLadders) return set_error(P6_ERR_INVALID_ARG, "no ladders set (p6_wy_set_ladders)");
  if (!s->dSchedG || gen0 < 0 || n_gen <= 0 || gen0 + n_gen > s->schedLen)
    return set_error(P6_ERR_INVALID_ARG, "generation range outside the schedule");
  P6_CUDA(cudaSetDevice(s->device));
  Params &P = s->P;
  Params saved = P;
  P.ladders = s->dLadders;
  P.rungs = s->rungs;
  P.nLadders = s->nLadders;
  P.schedGroups = s->dSchedG;
  P.schedPen = s->dSchedP;
  P.quenchSd = nullptr;
  if (s->dQuench) {
    if (gen0 + n_gen > s->quenchLen) {
      P = saved;
      return set_error(P6_ERR_INVALID_ARG, "generation range outside the quench schedule");
    }
    P.quenchSd = s->dQuench;
  }
  // with tracing on, the records hold the last generation of the run
  P.tracePos = s->trace ? s->dTracePos : nullptr;
  P.traceRec = s->trace ? s->dTraceRec : nullptr;
  P.traceIc = s->trace ? s->dTraceIc : nullptr;
  P.traceSums = s->trace ? s->dTraceSums : nullptr;
  P6_CUDA(cudaEventRecord(s->ev0, s->stream));
  cudaError_t e = launch(s, gen0, n_gen, 1, swap_every, reeval_first ? 1 : 0);
  P = saved;
  if (e != cudaSuccess) return cuda_error(e, "wy_kernel launch");
  P6_CUDA(cudaEventRecord(s->ev1, s->stream));
  return P6_OK;
}

p6_status p6_wy_run_host(p6_wy_session *s, const float *positions_in, const p6_wy_particle_state *state_in, int gen0,
                         int n_gen, int swap_every, int reeval_first, float *positions_out, float *best_out,
                         p6_wy_particle_state *state_out) {
  P6_ENTRY();
  if (!s || !positions_in || !state_in) return set_error(P6_ERR_INVALID_ARG, "null argument");
  p6_status st = p6_wy_sync_state(s, positions_in, state_in);
  if (st != P6_OK) return st;
  st = p6_wy_run(s, gen0, n_gen, swap_every, reeval_first);
  if (st != P6_OK) return st;
  st = p6_wy_read_state(s, positions_out, best_out, state_out);
  if (st != P6_OK) return st;
  return check_device_flag(s);
}

p6_status p6_wy_synchronize(p6_wy_session *s, double timeout_seconds) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(s->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > timeout_seconds) return set_error(P6_ERR_TIMEOUT, "the device did not finish within the deadline");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  if (s->linkedCt) {
    p6_status st = ct::check(s->linkedCt);
    s->linkedCt = nullptr;
    if (st != P6_OK) return st;
  }
  return check_device_flag(s);
}

p6_status p6_wy_read_trace_ic(p6_wy_session *s, float *ic) {
  P6_ENTRY();
  if (!s || !s->dTraceIc || !ic) return set_error(P6_ERR_INVALID_ARG, "tracing was not enabled");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaMemcpyAsync(ic, s->dTraceIc, (size_t)s->P.numParticles * s->P.nRefl * sizeof(float),
                          cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_set_fragment(p6_wy_session *s, const p6_wy_fragment *f) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (!f) {
    s->P.frag = nullptr;
    return P6_OK;
  }
  if (s->P.nAssign != 1) return set_error(P6_ERR_INVALID_ARG, "a fragment search takes one assignment");
  if (f->n_atoms < 1 || f->n_atoms > kFragMaxAtoms || f->n_atoms > s->P.maxSites)
    return set_error(P6_ERR_CAPACITY, "the fragment has more atoms than the sites (or than 32)");
  if (f->n_tors < 0 || f->n_tors > kFragMaxTors) return set_error(P6_ERR_CAPACITY, "at most 8 torsions");
  FragDev h{};
  h.nAtoms = f->n_atoms;
  h.nTors = f->n_tors;
  for (int t = 0; t < f->n_tors; ++t) {
    if (f->axis_b[t] < 0 || f->axis_b[t] >= f->n_atoms || f->axis_c[t] < 0 || f->axis_c[t] >= f->n_atoms ||
        f->axis_b[t] == f->axis_c[t])
      return set_error(P6_ERR_INVALID_ARG, "a torsion axis names an atom outside the fragment");
    h.axisB[t] = f->axis_b[t];
    h.axisC[t] = f->axis_c[t];
    h.moving[t] = f->moving[t] & (f->n_atoms >= 32 ? 0xffffffffu : ((1u << f->n_atoms) - 1u));
  }
  for (int i = 0; i < 3 * f->n_atoms; ++i) h.ref[i] = (float)f->ref_xyz[i];
  for (int i = 0; i < 9; ++i) h.toFrac[i] = (float)f->to_frac[i];
  h.transStep = (float)f->trans_step;
  h.angleStep = (float)f->angle_step;
  if (!s->dFrag) P6_CUDA(cudaMalloc(&s->dFrag, sizeof(FragDev)));
  if (!s->dFragState) {
    P6_CUDA(cudaMalloc(&s->dFragState, (size_t)s->P.numParticles * kFragParams * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dFragBest, (size_t)s->P.numParticles * kFragParams * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dFragProp, (size_t)s->P.numParticles * kFragParams * sizeof(float)));
    P6_CUDA(cudaMemsetAsync(s->dFragProp, 0, (size_t)s->P.numParticles * kFragParams * sizeof(float), s->stream));
    P6_CUDA(cudaMemsetAsync(s->dFragState, 0, (size_t)s->P.numParticles * kFragParams * sizeof(float), s->stream));
    P6_CUDA(cudaMemsetAsync(s->dFragBest, 0, (size_t)s->P.numParticles * kFragParams * sizeof(float), s->stream));
  }
  P6_CUDA(cudaMemcpyAsync(s->dFrag, &h, sizeof(FragDev), cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->P.frag = s->dFrag;
  s->P.fragState = s->dFragState;
  s->P.fragBest = s->dFragBest;
  s->P.fragProp = s->dFragProp;
  return P6_OK;
}

p6_status p6_wy_write_fragment_state(p6_wy_session *s, const float *current) {
  P6_ENTRY();
  if (!s || !current || !s->dFragState) return set_error(P6_ERR_INVALID_ARG, "no fragment set");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t bytes = (size_t)s->P.numParticles * kFragParams * sizeof(float);
  P6_CUDA(cudaMemcpyAsync(s->dFragState, current, bytes, cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaMemcpyAsync(s->dFragBest, current, bytes, cudaMemcpyHostToDevice, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_read_fragment_state(p6_wy_session *s, float *current, float *best) {
  P6_ENTRY();
  if (!s || !s->dFragState) return set_error(P6_ERR_INVALID_ARG, "no fragment set");
  P6_CUDA(cudaSetDevice(s->device));
  const size_t bytes = (size_t)s->P.numParticles * kFragParams * sizeof(float);
  if (current) P6_CUDA(cudaMemcpyAsync(current, s->dFragState, bytes, cudaMemcpyDeviceToHost, s->stream));
  if (best) P6_CUDA(cudaMemcpyAsync(best, s->dFragBest, bytes, cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_debug_fragment(p6_wy_session *s, const float *params, int n, uint32_t *coords) {
  P6_ENTRY();
  if (!s || !s->dFrag || !params || !coords || n <= 0) return set_error(P6_ERR_INVALID_ARG, "no fragment or bad arguments");
  P6_CUDA(cudaSetDevice(s->device));
  int nAtoms = 0;
  P6_CUDA(cudaMemcpy(&nAtoms, s->dFrag, sizeof(int), cudaMemcpyDeviceToHost));
  float *dp = nullptr;
  uint32_t *dc = nullptr;
  P6_CUDA(cudaMalloc(&dp, (size_t)n * kFragParams * sizeof(float)));
  cudaError_t e = cudaMalloc(&dc, (size_t)n * nAtoms * 3 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, params, (size_t)n * kFragParams * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) {
    wy_fragment_atoms_kernel<<<(n + 7) / 8, 256, 0, s->stream>>>(s->dFrag, dp, n, dc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(coords, dc, (size_t)n * nAtoms * 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(dp);
  if (dc) cudaFree(dc);
  if (e != cudaSuccess) return cuda_error(e, "fragment coordinates");
  return P6_OK;
}

p6_status p6_wy_read_trace_sums(p6_wy_session *s, double *sums) {
  P6_ENTRY();
  if (!s || !s->dTraceSums || !sums) return set_error(P6_ERR_INVALID_ARG, "tracing was not enabled");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaMemcpyAsync(sums, s->dTraceSums, (size_t)s->P.numParticles * 3 * sizeof(double),
                          cudaMemcpyDeviceToHost, s->stream));
  P6_CUDA(cudaStreamSynchronize(s->stream));
  return P6_OK;
}

p6_status p6_wy_debug_expand(p6_wy_session *s, int particle, uint32_t *atoms) {
  P6_ENTRY();
  if (!s || !atoms || particle < 0 || particle >= s->P.numParticles)
    return set_error(P6_ERR_INVALID_ARG, "bad particle or output");
  P6_CUDA(cudaSetDevice(s->device));
  uint32_t *d = nullptr;
  P6_CUDA(cudaMalloc(&d, (size_t)s->P.nTot * 3 * sizeof(uint32_t)));
  wy_expand_one<<<(s->P.nTot + 127) / 128, 128, 0, s->stream>>>(s->P, s->dGenOrig, particle, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(atoms, d, (size_t)s->P.nTot * 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_error(e, "wy_expand_one");
  return P6_OK;
}

p6_status p6_wy_last_kernel_ms(p6_wy_session *s, float *ms) {
  P6_ENTRY();
  if (!s || !ms) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaEventSynchronize(s->ev1));
  P6_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
  return P6_OK;
}

p6_status p6_wy_query(p6_wy_session *s, int *incremental, int *smem_bytes, int *max_grid) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (incremental) *incremental = s->incremental;
  if (smem_bytes) *smem_bytes = s->smemBytes;
  if (max_grid) *max_grid = s->maxGrid;
  return P6_OK;
}

p6_status p6_wy_launch_count(p6_wy_session *s, long long *count) {
  P6_ENTRY();
  if (!s || !count) return set_error(P6_ERR_INVALID_ARG, "null argument");
  *count = s->launches;
  return P6_OK;
}

}  // extern "C"

// ===========================================================================
// Learned search: one generation whose proposals the network pre-ranks.
// ===========================================================================
extern "C" p6_status p6_wy_learned_step(p6_wy_session *s, p6_mlp *net, int K, int gen, int swap_every,
                                        int reeval_first, float *features, float *gains, float *accepted,
                                        float *scores) {
  P6_ENTRY();
  if (!s || K < 1 || (K > 1 && !net)) return set_error(P6_ERR_INVALID_ARG, "bad arguments");
  if (!s->dLadders) return set_error(P6_ERR_INVALID_ARG, "no ladders set (p6_wy_set_ladders)");
  if (!s->dSchedG || gen < 0 || gen >= s->schedLen) return set_error(P6_ERR_INVALID_ARG, "generation outside the schedule");
  if (s->P.frag) return set_error(P6_ERR_INVALID_ARG, "the learned step moves sites, not a fragment");
  if (net && (mlp::input_dim(net) != kFeat || mlp::output_dim(net) < 1))
    return set_error(P6_ERR_INVALID_ARG, "the network must take 64 features");
  if (s->incremental) return set_error(P6_ERR_INVALID_ARG, "the learned search uses the full evaluation");
  P6_CUDA(cudaSetDevice(s->device));
  Params &P = s->P;
  const size_t n = P.numParticles, stride = (size_t)P.maxSites * 3;
  const int dOut = net ? mlp::output_dim(net) : 1;
  if (K > s->learnK || dOut > s->learnOut) {
    for (void **q : {(void **)&s->dCand, (void **)&s->dExt, (void **)&s->dFeat, (void **)&s->dScore,
                     (void **)&s->dChosenFeat, (void **)&s->dChosenScore}) {
      if (*q) cudaFree(*q);
      *q = nullptr;
    }
    s->learnK = 0;
    P6_CUDA(cudaMalloc(&s->dCand, n * K * stride * sizeof(uint32_t)));
    P6_CUDA(cudaMalloc(&s->dExt, n * stride * sizeof(uint32_t)));
    P6_CUDA(cudaMalloc(&s->dFeat, n * K * kFeat * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dScore, n * K * dOut * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dChosenFeat, n * kFeat * sizeof(float)));
    P6_CUDA(cudaMalloc(&s->dChosenScore, n * sizeof(float)));
    s->learnK = K;
    s->learnOut = dOut;
  }
  const long long threads = (long long)n * K;
  wy_candidates_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s->stream>>>(P, gen, K, s->dCand, s->dFeat);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  const float *score = nullptr;
  if (net && K > 1) {
    p6_status st = mlp::predict_device(net, s->dFeat, (int)threads, s->dScore, s->stream);
    if (st != P6_OK) return st;
    score = s->dScore;
  }
  wy_select_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(P, K, score, dOut, s->dCand, s->dFeat, s->dExt,
                                                                      s->dChosenFeat, s->dChosenScore);
  P6_CUDA(cudaGetLastError());
  s->launches++;
  const bool wantTrace = gains || accepted;
  if (wantTrace && !s->dTraceRec) {
    p6_status st = p6_wy_set_trace(s, 1);
    if (st != P6_OK) return st;
    s->trace = false;
  }
  Params saved = P;
  P.ladders = s->dLadders;
  P.rungs = s->rungs;
  P.nLadders = s->nLadders;
  P.schedGroups = s->dSchedG;
  P.schedPen = s->dSchedP;
  P.quenchSd = nullptr;
  P.extProp = s->dExt;
  P.tracePos = nullptr;
  P.traceRec = wantTrace ? s->dTraceRec : nullptr;
  P.traceIc = nullptr;
  cudaError_t e = launch(s, gen, 1, 1, swap_every, reeval_first ? 1 : 0);
  P = saved;
  if (e != cudaSuccess) return cuda_error(e, "wy_kernel launch");
  std::vector<float> rec;
  if (wantTrace) {
    rec.resize(n * 8);
    P6_CUDA(cudaMemcpyAsync(rec.data(), s->dTraceRec, n * 8 * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  }
  if (features)
    P6_CUDA(cudaMemcpyAsync(features, s->dChosenFeat, n * kFeat * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  if (scores) P6_CUDA(cudaMemcpyAsync(scores, s->dChosenScore, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  if (wantTrace || features || scores) {
    P6_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t p = 0; p < n && wantTrace; ++p) {
      if (gains) gains[p] = rec[p * 8] - rec[p * 8 + 5];
      if (accepted) accepted[p] = rec[p * 8 + 4];
    }
  }
  return P6_OK;
}

// The fixed-profile fitness in Gram form for every later evaluation of the
// session: v (n_refl doubles) and the upper band of G by diagonal (band[d *
// n_refl + k] = G[k][k + d], d = 0..bw), sum w y^2 = syy.  v == NULL
// returns to the grouped-intensity fitness.
extern "C" p6_status p6_wy_set_profile(p6_wy_session *s, const double *v, const double *band, int bw, double syy) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  if (!v) {
    s->P.profV = nullptr;
    s->P.profG = nullptr;
    return P6_OK;
  }
  if (!band || bw < 0 || !(syy > 0.0)) return set_error(P6_ERR_INVALID_ARG, "empty profile operands");
  const int K = s->P.nRefl;
  if (bw >= K) bw = K - 1;
  for (double **q : {&s->dProfV, &s->dProfG}) {
    if (*q) cudaFree(*q);
    *q = nullptr;
  }
  p6_status st = upload(&s->dProfV, v, (size_t)K, s->stream);
  if (st != P6_OK) return st;
  st = upload(&s->dProfG, band, (size_t)K * (bw + 1), s->stream);
  if (st != P6_OK) return st;
  P6_CUDA(cudaStreamSynchronize(s->stream));
  s->P.profV = s->dProfV;
  s->P.profG = s->dProfG;
  s->P.profK = K;
  s->P.profBw = bw;
  s->P.profSyy = syy;
  return P6_OK;
}

// A Wyckoff search with the cell and profile fixed: each generation the
// search kernel proposes and evaluates every replica's move with its
// deferred acceptance, writing the proposal's mult |F|^2 row into the
// contraction's intensity buffer; the contraction forms Y = I . P and the
// fitted-scale partials of every replica; wy_profile_accept_kernel reduces
// them to each replica's chi^2 at its best scale and takes the Metropolis
// decisions and the ladder exchange.  Everything is queued on the
// search session's stream.
extern "C" p6_status p6_wy_profile_run(p6_wy_session *s, p6_ct_session *ct, int method, int gen0, int n_gen,
                                       int swap_every, int init, int n_active_points) {
  P6_ENTRY();
  if (!s || !ct) return set_error(P6_ERR_INVALID_ARG, "null session");
  if (!s->dLadders) return set_error(P6_ERR_INVALID_ARG, "no ladders set (p6_wy_set_ladders)");
  if (s->schedPenHost.empty() || gen0 < 0 || n_gen < 0 || gen0 + n_gen > s->schedLen ||
      (n_gen == 0 && !init) || (init && gen0 >= s->schedLen))
    return set_error(P6_ERR_INVALID_ARG, "generation range outside the schedule");
  if (method < P6_CT_SPLIT_BF16 || method > P6_CT_FP32_DENSE) return set_error(P6_ERR_INVALID_ARG, "unknown method");
  const ct::ProfileLink L = ct::link(ct);
  if (L.device != s->device) return set_error(P6_ERR_INVALID_ARG, "the sessions are on different devices");
  if (L.n_refl != s->P.nRefl)
    return set_error(P6_ERR_INVALID_ARG, "the profile's reflections are not the search's reflections");
  if (L.max_replicas < s->P.numParticles)
    return set_error(P6_ERR_CAPACITY, "the contraction holds fewer replicas than the search");
  if (s->dQuench && gen0 + n_gen > s->quenchLen)
    return set_error(P6_ERR_INVALID_ARG, "generation range outside the quench schedule");
  P6_CUDA(cudaSetDevice(s->device));
  if (!s->dTracePos) {
    const bool was = s->trace;
    p6_status st = p6_wy_set_trace(s, 1);
    if (st != P6_OK) return st;
    s->trace = was;
  }
  const int nAct = n_active_points > 0 ? std::min(n_active_points, L.n_points) : L.n_points;
  const double syy = ct::syy(ct, nAct);
  if (!(syy > 0.0)) return set_error(P6_ERR_INVALID_ARG, "no weighted counts in the active points");
  Params &P = s->P;
  const Params saved = P;
  const int savedIncr = s->incremental;
  s->incremental = 0;   // one generation per launch: the full evaluation
  P.ladders = s->dLadders;
  P.rungs = s->rungs;
  P.nLadders = s->nLadders;
  P.schedGroups = nullptr;   // every reflection is evaluated: the pattern needs all of them
  P.schedPen = nullptr;
  P.ngaArg = P.nGroups;
  P.quenchSd = s->dQuench;
  P.extProp = nullptr;
  P.deferAccept = 1;
  P.tracePos = s->dTracePos;
  P.traceRec = s->dTraceRec;
  P.traceIc = L.intensities;
  P.traceSums = nullptr;
  const int n = P.numParticles;
  const int acceptGrid = (P.nLadders + kAcceptWarps - 1) / kAcceptWarps;
  p6_status st = P6_OK;
  cudaError_t e = cudaEventRecord(s->ev0, s->stream);
  auto step = [&](int g, int mcmc, int swapEvery, int first) -> p6_status {
    P.penArg = s->schedPenHost[g];
    cudaError_t le = launch(s, g, 1, mcmc, 0, 0);
    if (le != cudaSuccess) return cuda_error(le, "wy_kernel launch");
    const double2 *part = nullptr;
    int nParts = 0;
    p6_status cs = ct::enqueue_fitted_partials(ct, s->stream, n, method, nAct, &part, &nParts);
    if (cs != P6_OK) return cs;
    wy_profile_accept_kernel<<<acceptGrid, 32 * kAcceptWarps, 0, s->stream>>>(P, part, nParts, syy, g, swapEvery,
                                                                             first);
    le = cudaGetLastError();
    if (le != cudaSuccess) return cuda_error(le, "wy_profile_accept_kernel launch");
    s->launches++;
    return P6_OK;
  };
  if (e != cudaSuccess) st = cuda_error(e, "cudaEventRecord");
  if (st == P6_OK && init) st = step(gen0, 0, 0, 1);
  for (int gi = 0; gi < n_gen && st == P6_OK; ++gi) st = step(gen0 + gi, 1, swap_every, 0);
  if (st == P6_OK) {
    e = cudaEventRecord(s->ev1, s->stream);
    if (e != cudaSuccess) st = cuda_error(e, "cudaEventRecord");
  }
  P = saved;
  s->incremental = savedIncr;
  s->linkedCt = ct;
  return st;
}

// Marks the start (end = 0) or end (end = 1) of a timed span on the session's
// stream; p6_wy_last_kernel_ms then reports the span.
extern "C" p6_status p6_wy_time_mark(p6_wy_session *s, int end) {
  P6_ENTRY();
  if (!s) return set_error(P6_ERR_INVALID_ARG, "null session");
  P6_CUDA(cudaSetDevice(s->device));
  P6_CUDA(cudaEventRecord(end ? s->ev1 : s->ev0, s->stream));
  return P6_OK;
}

// ===========================================================================
// Batched searches: many sessions' ladders in one persistent launch.
// ===========================================================================
struct p6_wy_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<p6_wy_session *> sessions;
  std::vector<cudaEvent_t> evSess;   // one per session: its queued work before the batch
  std::vector<Params> hProbs;
  std::vector<RunArgs> hArgs;
  std::vector<int2> hItems;
  Params *dProbs = nullptr;
  RunArgs *dArgs = nullptr;
  int2 *dItems = nullptr;
  int *dCounter = nullptr;
  int itemsCap = 0, nItems = 0;
  int smemBytes = 0, cosMode = 0, slots = 0, numSMs = 0, maxPerSM = 1;
  int perSM = 0;   // persistent CTAs per SM (0: the occupancy limit)
  int order = 0;   // 0: longest estimated ladder first; 1: problem order
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graphGrid = -1;
  long long launches = 0;
};

namespace {
template <int C, int S>
cudaError_t batch_attr(int smem, int *occ) {
  auto k = wy_batch_kernel<C, S, 0>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, 256, smem);
}
template <int C, int S>
void batch_launch(p6_wy_batch *b, int grid) {
  wy_batch_kernel<C, S, 0><<<grid, 256, b->smemBytes, b->stream>>>(b->dProbs, b->dArgs, b->dItems, b->nItems,
                                                                   b->dCounter);
}
cudaError_t batch_variant_attr(p6_wy_batch *b, int *occ) {
  const int C = b->cosMode, S = b->slots;
  if (S == 0) return C ? batch_attr<1, 0>(b->smemBytes, occ) : batch_attr<0, 0>(b->smemBytes, occ);
  if (S == 64) return C ? batch_attr<1, 64>(b->smemBytes, occ) : batch_attr<0, 64>(b->smemBytes, occ);
  return C ? batch_attr<1, 256>(b->smemBytes, occ) : batch_attr<0, 256>(b->smemBytes, occ);
}
void batch_variant_launch(p6_wy_batch *b, int grid) {
  const int C = b->cosMode, S = b->slots;
  if (S == 0) C ? batch_launch<1, 0>(b, grid) : batch_launch<0, 0>(b, grid);
  else if (S == 64) C ? batch_launch<1, 64>(b, grid) : batch_launch<0, 64>(b, grid);
  else C ? batch_launch<1, 256>(b, grid) : batch_launch<0, 256>(b, grid);
}
void batch_free(p6_wy_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (void *p : {(void *)b->dProbs, (void *)b->dArgs, (void *)b->dItems, (void *)b->dCounter})
    if (p) cudaFree(p);
  for (cudaEvent_t ev : b->evSess)
    if (ev) cudaEventDestroy(ev);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}
}  // namespace

extern "C" {

p6_status p6_wy_batch_create(p6_wy_session *const *sessions, int n_sessions, p6_wy_batch **out) {
  P6_ENTRY();
  if (!sessions || n_sessions <= 0 || !out) return set_error(P6_ERR_INVALID_ARG, "no sessions");
  *out = nullptr;
  for (int i = 0; i < n_sessions; ++i) {
    const p6_wy_session *s = sessions[i];
    if (!s) return set_error(P6_ERR_INVALID_ARG, "null session in the batch");
    if (s->device != sessions[0]->device) return set_error(P6_ERR_INVALID_ARG, "sessions on different devices");
    if (s->cosMode != sessions[0]->cosMode) return set_error(P6_ERR_INVALID_ARG, "sessions with different cos_mode");
    if (s->cosMode == 2)
      return set_error(P6_ERR_INVALID_ARG, "the batched launch takes cos_mode 0 or 1 (the groups of a batch differ)");
    if (s->incremental) return set_error(P6_ERR_INVALID_ARG, "batched searches use the full evaluation (incremental = 0)");
    if (s->P.rungs > 8) return set_error(P6_ERR_CAPACITY, "batched ladders hold at most 8 rungs");
  }
  p6_wy_batch *b = new p6_wy_batch();
  b->device = sessions[0]->device;
  b->sessions.assign(sessions, sessions + n_sessions);
  b->cosMode = sessions[0]->cosMode;
  for (p6_wy_session *s : b->sessions) {
    b->smemBytes = std::max(b->smemBytes, s->smemBytes);
    b->slots = std::max(b->slots, s->slots);
  }
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  b->evSess.assign(n_sessions, nullptr);
  for (int i = 0; i < n_sessions && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&b->evSess[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->dProbs, sizeof(Params) * n_sessions);
  if (e == cudaSuccess) e = cudaMalloc(&b->dArgs, sizeof(RunArgs) * n_sessions);
  if (e == cudaSuccess) e = cudaMalloc(&b->dCounter, sizeof(int));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, b->device);
  int occ = 0;
  if (e == cudaSuccess) e = batch_variant_attr(b, &occ);
  if (e != cudaSuccess) {
    batch_free(b);
    return cuda_error(e, "batch set-up");
  }
  if (occ < 1) {
    batch_free(b);
    return set_error(P6_ERR_CAPACITY, "the largest problem of the batch does not fit one CTA per SM");
  }
  b->maxPerSM = occ;
  *out = b;
  return P6_OK;
}

p6_status p6_wy_batch_destroy(p6_wy_batch *b) {
  P6_ENTRY();
  if (!b) return set_error(P6_ERR_INVALID_ARG, "null batch");
  batch_free(b);
  return P6_OK;
}

p6_status p6_wy_batch_set_launch(p6_wy_batch *b, int ctas_per_sm, int order) {
  P6_ENTRY();
  if (!b || ctas_per_sm < 0 || ctas_per_sm > b->maxPerSM || order < 0 || order > 1)
    return set_error(P6_ERR_INVALID_ARG, "bad launch shape");
  b->perSM = ctas_per_sm;
  b->order = order;
  return P6_OK;
}

p6_status p6_wy_batch_query(p6_wy_batch *b, int *max_ctas_per_sm, int *smem_bytes, int *n_items, long long *launches) {
  P6_ENTRY();
  if (!b) return set_error(P6_ERR_INVALID_ARG, "null batch");
  if (max_ctas_per_sm) *max_ctas_per_sm = b->maxPerSM;
  if (smem_bytes) *smem_bytes = b->smemBytes;
  if (n_items) *n_items = b->nItems;
  if (launches) *launches = b->launches;
  return P6_OK;
}

p6_status p6_wy_batch_run(p6_wy_batch *b, const int32_t *gen0, const int32_t *n_gen, int swap_every, int reeval_first,
                          int use_graph) {
  P6_ENTRY();
  if (!b || !gen0 || !n_gen) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaSetDevice(b->device));
  const int n = (int)b->sessions.size();
  b->hProbs.resize(n);
  b->hArgs.resize(n);
  std::vector<std::pair<double, int2>> items;
  for (int i = 0; i < n; ++i) {
    p6_wy_session *s = b->sessions[i];
    if (!s->dLadders) return set_error(P6_ERR_INVALID_ARG, "a session of the batch has no ladders");
    if (!s->dSchedG || gen0[i] < 0 || n_gen[i] <= 0 || gen0[i] + n_gen[i] > s->schedLen)
      return set_error(P6_ERR_INVALID_ARG, "a generation range lies outside its schedule");
    Params P = s->P;
    P.ladders = s->dLadders;
    P.rungs = s->rungs;
    P.nLadders = s->nLadders;
    P.schedGroups = s->dSchedG;
    P.schedPen = s->dSchedP;
    P.quenchSd = nullptr;
    P.tracePos = nullptr;
    P.traceRec = nullptr;
    P.traceIc = nullptr;
    b->hProbs[i] = P;
    b->hArgs[i] = RunArgs{gen0[i], n_gen[i], 1, swap_every, reeval_first ? 1 : 0, {0, 0, 0}};
    // cost of one ladder: generations x reflections x atoms entering |F|^2 x rungs
    const double cost = (double)n_gen[i] * (double)(P.nRefl + 16) * (double)(P.nTot + 4) * (double)P.rungs;
    for (int L = 0; L < s->nLadders; ++L) items.push_back({cost, make_int2(i, L)});
  }
  if (b->order == 0)
    std::stable_sort(items.begin(), items.end(),
                     [](const std::pair<double, int2> &x, const std::pair<double, int2> &y) { return x.first > y.first; });
  b->hItems.resize(items.size());
  for (size_t k = 0; k < items.size(); ++k) b->hItems[k] = items[k].second;
  if ((int)items.size() > b->itemsCap) {
    if (b->dItems) cudaFree(b->dItems);
    b->dItems = nullptr;
    b->itemsCap = 0;
    P6_CUDA(cudaMalloc(&b->dItems, sizeof(int2) * items.size()));
    b->itemsCap = (int)items.size();
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    b->graphGrid = -1;
  }
  b->nItems = (int)items.size();
  // the batch starts after each session's queued work (state uploads) is done
  for (int i = 0; i < n; ++i) {
    P6_CUDA(cudaEventRecord(b->evSess[i], b->sessions[i]->stream));
    P6_CUDA(cudaStreamWaitEvent(b->stream, b->evSess[i], 0));
  }
  P6_CUDA(cudaMemcpyAsync(b->dProbs, b->hProbs.data(), sizeof(Params) * n, cudaMemcpyHostToDevice, b->stream));
  P6_CUDA(cudaMemcpyAsync(b->dArgs, b->hArgs.data(), sizeof(RunArgs) * n, cudaMemcpyHostToDevice, b->stream));
  P6_CUDA(cudaMemcpyAsync(b->dItems, b->hItems.data(), sizeof(int2) * b->nItems, cudaMemcpyHostToDevice, b->stream));
  const int perSM = b->perSM > 0 ? b->perSM : b->maxPerSM;
  const int grid = std::max(1, std::min(b->nItems, perSM * b->numSMs));
  P6_CUDA(cudaEventRecord(b->ev0, b->stream));
  if (use_graph) {
    if (!b->exec || b->graphGrid != grid) {
      if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
      if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
      P6_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      cudaMemsetAsync(b->dCounter, 0, sizeof(int), b->stream);
      batch_variant_launch(b, grid);
      cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
      if (e != cudaSuccess) return cuda_error(e, "batch graph capture");
      P6_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
      b->graphGrid = grid;
    }
    P6_CUDA(cudaGraphLaunch(b->exec, b->stream));
  } else {
    P6_CUDA(cudaMemsetAsync(b->dCounter, 0, sizeof(int), b->stream));
    batch_variant_launch(b, grid);
    P6_CUDA(cudaGetLastError());
  }
  b->launches++;
  P6_CUDA(cudaEventRecord(b->ev1, b->stream));
  // later work on each session (state reads) waits for the batch
  for (p6_wy_session *s : b->sessions) P6_CUDA(cudaStreamWaitEvent(s->stream, b->ev1, 0));
  return P6_OK;
}

p6_status p6_wy_batch_synchronize(p6_wy_batch *b, double timeout_seconds) {
  P6_ENTRY();
  if (!b) return set_error(P6_ERR_INVALID_ARG, "null batch");
  P6_CUDA(cudaSetDevice(b->device));
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(b->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > timeout_seconds) return set_error(P6_ERR_TIMEOUT, "the batch did not finish within the deadline");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  for (p6_wy_session *s : b->sessions) {
    const p6_status st = check_device_flag(s);
    if (st != P6_OK) return st;
  }
  return P6_OK;
}

p6_status p6_wy_batch_last_ms(p6_wy_batch *b, float *ms) {
  P6_ENTRY();
  if (!b || !ms) return set_error(P6_ERR_INVALID_ARG, "null argument");
  P6_CUDA(cudaEventSynchronize(b->ev1));
  P6_CUDA(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return P6_OK;
}

}  // extern "C"

// ===========================================================================
// Wyckoff-constrained least-squares refinement of coordinates against the
// grouped |F|^2 (refineCoordinatesAgainstWppf, js/coord_refine.js:266-627).
// The device computes, per structure (one CTA each), the group intensities
// Ical_g = sum mult |F|^2 over the group's reflections and their analytic
// derivatives with respect to the site coordinates (the chain rule through
// R^T h, js/coord_refine.js:216-247, projected into each site's Wyckoff
// subspace by P^T), then the closed-form scale, chi^2 and the normal
// equations J'WJ, J'W r in FP64; the host runs the Levenberg-Marquardt
// control of every structure in lock step.
// ===========================================================================
namespace p6 {
namespace wy {

struct RefineArgs {
  int nP;                   // maxSites * 3
  const uint32_t *assign;   // per structure
  const double *coords;     // structures * nP, fractional
  double *ical;             // structures * nGroups
  double *jac;              // structures * nGroups * nP, or null
  double *out;              // structures * (4 + nP + nP * nP): scale, chi2, sum w Io^2, -, J'Wr, J'WJ
};

constexpr int kRefineThreads = 128;
constexpr int kRefineMaxAtoms = 1024;

__global__ void __launch_bounds__(kRefineThreads) wy_refine_eval_kernel(const Params P, const RefineArgs R) {
  __shared__ double ax[kRefineMaxAtoms * 3];
  __shared__ short asite[kRefineMaxAtoms], aop[kRefineMaxAtoms], atype[kRefineMaxAtoms];
  __shared__ int nAt;
  const int st = blockIdx.x, nP = R.nP, ms = P.maxSites;
  const int A = (int)R.assign[st];
  const uint32_t *gen = P.genOrig + (size_t)A * P.nTot;
  const OpFix *ops = P.ops;
  const double *u = R.coords + (size_t)st * nP;
  if (threadIdx.x == 0) {
    int n = 0;
    for (int g = 0; g < P.nTot && n < kRefineMaxAtoms; ++g) {
      const uint32_t w = gen[g];
      if ((w >> 24) & 1u) continue;   // centring translates scale |F|^2 only; the scale absorbs it
      asite[n] = (short)(w & 0xFF);
      aop[n] = (short)((w >> 8) & 0xFFF);
      atype[n] = (short)min((int)((w >> 20) & 0xF), P.nElem - 1);
      ++n;
    }
    nAt = n;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nAt; j += blockDim.x) {
    const OpFix &op = ops[aop[j]];
    const double *x = u + 3 * asite[j];
    for (int i = 0; i < 3; ++i) {
      const double v = op.r[3 * i] * x[0] + op.r[3 * i + 1] * x[1] + op.r[3 * i + 2] * x[2] +
                       (double)op.t[i] * (1.0 / 4294967296.0);
      ax[3 * j + i] = v - floor(v);
    }
  }
  __syncthreads();
  const ReflRec *refl = reinterpret_cast<const ReflRec *>(P.blob + P.offRefl);
  const float *ftab = reinterpret_cast<const float *>(P.blob + P.offF);
  const float4 *groups = reinterpret_cast<const float4 *>(P.blob + P.offGroup);
  const bool jac = R.jac != nullptr;
  for (int gI = threadIdx.x; gI < P.nGroups; gI += blockDim.x) {
    const float4 gm = groups[gI];
    const int r0 = (int)gm.x, cnt = (int)gm.y;
    double acc = 0.0;
    double grow[kMaxSites * 3];
    if (jac)
      for (int p = 0; p < nP; ++p) grow[p] = 0.0;
    for (int r = r0; r < r0 + cnt; ++r) {
      const ReflRec rr = refl[r];
      const double h = rr.h, k = rr.k, l = rr.l;
      double a = 0.0, b = 0.0;
      for (int j = 0; j < nAt; ++j) {
        const double f = ftab[(size_t)r * P.nElem + atype[j]];
        double sn, cs;
        sincospi(2.0 * (h * ax[3 * j] + k * ax[3 * j + 1] + l * ax[3 * j + 2]), &sn, &cs);
        a += f * cs;
        b += f * sn;
      }
      acc += (double)rr.mult * (a * a + b * b);
      if (!jac) continue;
      // d|F|^2/du = 2 (A dA/du + B dB/du), dA/du = -2 pi f (R^T h) sin, dB/du = 2 pi f (R^T h) cos
      for (int j = 0; j < nAt; ++j) {
        const double f = ftab[(size_t)r * P.nElem + atype[j]];
        double sn, cs;
        sincospi(2.0 * (h * ax[3 * j] + k * ax[3 * j + 1] + l * ax[3 * j + 2]), &sn, &cs);
        const double w = (double)rr.mult * 2.0 * 2.0 * 3.14159265358979323846 * f * (b * cs - a * sn);
        const int *Rm = ops[aop[j]].r;
        const int base = 3 * asite[j];
        grow[base] += w * (Rm[0] * h + Rm[3] * k + Rm[6] * l);
        grow[base + 1] += w * (Rm[1] * h + Rm[4] * k + Rm[7] * l);
        grow[base + 2] += w * (Rm[2] * h + Rm[5] * k + Rm[8] * l);
      }
    }
    R.ical[(size_t)st * P.nGroups + gI] = acc;
    if (jac) {
      // into each site's Wyckoff subspace: P^T g
      double *J = R.jac + ((size_t)st * P.nGroups + gI) * nP;
      for (int si = 0; si < ms; ++si) {
        const ProjFix &pf = P.proj[(size_t)A * ms + si];
        const double inv = 1.0 / (double)pf.den;
        const double g0 = grow[3 * si], g1 = grow[3 * si + 1], g2 = grow[3 * si + 2];
        for (int c = 0; c < 3; ++c)
          J[3 * si + c] = (pf.num[c] * g0 + pf.num[3 + c] * g1 + pf.num[6 + c] * g2) * inv;
      }
    }
  }
}

// Scale, chi^2 and (with J) the normal equations of one structure per CTA.
__global__ void __launch_bounds__(kRefineThreads) wy_refine_normal_kernel(const Params P, const RefineArgs R) {
  __shared__ double red[3][kRefineThreads];
  __shared__ double sScale;
  const int st = blockIdx.x, nP = R.nP, nG = P.nGroups, tid = threadIdx.x;
  const float4 *groups = reinterpret_cast<const float4 *>(P.blob + P.offGroup);
  const double *ic = R.ical + (size_t)st * nG;
  double *out = R.out + (size_t)st * (4 + nP + (size_t)nP * nP);
  double num = 0, den = 0, oo = 0;
  for (int g = tid; g < nG; g += blockDim.x) {
    const float4 gm = groups[g];
    const double w = gm.w > 0.f ? (double)gm.w : 0.0, io = gm.z;
    num += w * io * ic[g];
    den += w * ic[g] * ic[g];
    oo += w * io * io;
  }
  red[0][tid] = num; red[1][tid] = den; red[2][tid] = oo;
  __syncthreads();
  if (tid == 0) {
    double a = 0, b = 0, c = 0;
    for (int i = 0; i < blockDim.x; ++i) { a += red[0][i]; b += red[1][i]; c += red[2][i]; }
    sScale = b > 0 ? a / b : 0.0;
    out[0] = sScale;
    out[2] = c;
  }
  __syncthreads();
  const double sc = sScale;
  double chi = 0;
  for (int g = tid; g < nG; g += blockDim.x) {
    const float4 gm = groups[g];
    const double w = gm.w > 0.f ? (double)gm.w : 0.0, d = (double)gm.z - sc * ic[g];
    chi += w * d * d;
  }
  __syncthreads();
  red[0][tid] = chi;
  __syncthreads();
  if (tid == 0) {
    double a = 0;
    for (int i = 0; i < blockDim.x; ++i) a += red[0][i];
    out[1] = a;
  }
  if (!R.jac) return;
  const double *J = R.jac + (size_t)st * nG * nP;
  for (int p = tid; p < nP; p += blockDim.x) {
    double t = 0;
    for (int g = 0; g < nG; ++g) {
      const float4 gm = groups[g];
      const double w = gm.w > 0.f ? (double)gm.w : 0.0;
      t += w * (sc * J[(size_t)g * nP + p]) * ((double)gm.z - sc * ic[g]);
    }
    out[4 + p] = t;
  }
  for (int pq = tid; pq < nP * nP; pq += blockDim.x) {
    const int pp = pq / nP, qq = pq % nP;
    if (qq < pp) continue;
    double t = 0;
    for (int g = 0; g < nG; ++g) {
      const float4 gm = groups[g];
      const double w = gm.w > 0.f ? (double)gm.w : 0.0;
      t += w * (sc * J[(size_t)g * nP + pp]) * (sc * J[(size_t)g * nP + qq]);
    }
    out[4 + nP + (size_t)pp * nP + qq] = t;
    out[4 + nP + (size_t)qq * nP + pp] = t;
  }
}

}  // namespace wy
}  // namespace p6

namespace {
// crSolve (js/coord_refine.js:629-662): Cholesky of the damped normal matrix; false if not positive definite.
bool refine_solve(const std::vector<double> &A, const std::vector<double> &b, int n, std::vector<double> &x) {
  std::vector<double> L((size_t)n * n, 0.0), y(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = A[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      if (i == j) {
        if (!(s > 0)) return false;
        L[(size_t)i * n + i] = std::sqrt(s);
      } else {
        L[(size_t)i * n + j] = s / L[(size_t)j * n + j];
      }
    }
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
    y[i] = s / L[(size_t)i * n + i];
  }
  x.assign(n, 0.0);
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[k];
    x[i] = s / L[(size_t)i * n + i];
  }
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}
}  // namespace

extern "C" p6_status p6_wy_refine(p6_wy_session *s, int n, const uint32_t *assign, double *coords,
                                  const p6_wy_refine_opts *opts, double *r_start, double *r_final, double *chi2,
                                  int *iterations, int *converged) {
  P6_ENTRY();
  if (!s || n <= 0 || !assign || !coords) return set_error(P6_ERR_INVALID_ARG, "null argument or no structures");
  p6_wy_refine_opts o{60, 1e-3, 10.0, 0.4, 1e8, 1e-6, 1e-9, 0.05};
  if (opts) o = *opts;
  if (o.max_iter < 0 || !(o.lambda0 > 0) || !(o.lambda_up > 1) || !(o.lambda_down > 0) ||
      !(o.lambda_max > o.lambda0) || !(o.max_step > 0))
    return set_error(P6_ERR_INVALID_ARG, "refinement options out of range");
  Params &P = s->P;
  const int ms = P.maxSites, nP = ms * 3, nG = P.nGroups;
  for (int i = 0; i < n; ++i)
    if ((int)assign[i] >= P.nAssign) return set_error(P6_ERR_INVALID_ARG, "assignment index out of range");
  if (P.nTot > kRefineMaxAtoms) return set_error(P6_ERR_CAPACITY, "more than 1024 generated atoms for the refinement");
  // free parameters (trace of each projector) against the weighted groups
  int nObs = 0;
  for (const float4 &g : s->groupsHost) nObs += g.w > 0.f ? 1 : 0;
  for (int i = 0; i < n; ++i) {
    int nFree = 0;
    for (int si = 0; si < ms; ++si) {
      const ProjFix &pf = s->projHost[(size_t)assign[i] * ms + si];
      nFree += (int)std::lround((double)(pf.num[0] + pf.num[4] + pf.num[8]) / pf.den);
    }
    if (nObs <= nFree + 1)
      return set_error(P6_ERR_INVALID_ARG, "the refinement is underdetermined: too few weighted groups for the free coordinates");
  }
  P6_CUDA(cudaSetDevice(s->device));
  const size_t outStride = 4 + nP + (size_t)nP * nP;
  uint32_t *dA = nullptr;
  double *dX = nullptr, *dI = nullptr, *dJ = nullptr, *dOut = nullptr;
  auto release = [&]() {
    for (void *q : {(void *)dA, (void *)dX, (void *)dI, (void *)dJ, (void *)dOut})
      if (q) cudaFree(q);
  };
  cudaError_t e = cudaMalloc(&dA, (size_t)n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * nP * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dI, (size_t)n * nG * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dJ, (size_t)n * nG * nP * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dOut, (size_t)n * outStride * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dA, assign, (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) { release(); return cuda_error(e, "refinement buffers"); }

  // projection onto each site's Wyckoff subspace, x mod 1 (js/coord_refine.js:311-327)
  auto project = [&](int i, double *x) {
    for (int si = 0; si < ms; ++si) {
      const ProjFix &pf = s->projHost[(size_t)assign[i] * ms + si];
      double v[3];
      for (int c = 0; c < 3; ++c) {
        v[c] = (pf.num[3 * c] * x[3 * si] + pf.num[3 * c + 1] * x[3 * si + 1] + pf.num[3 * c + 2] * x[3 * si + 2]) /
                   (double)pf.den +
               (double)pf.t[c] * (1.0 / 4294967296.0);
        v[c] -= std::floor(v[c]);
      }
      for (int c = 0; c < 3; ++c) x[3 * si + c] = v[c];
    }
  };
  std::vector<double> outH((size_t)n * outStride);
  auto evaluate = [&](const std::vector<double> &x, bool jac) -> cudaError_t {
    cudaError_t err = cudaMemcpyAsync(dX, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    if (err != cudaSuccess) return err;
    RefineArgs a{nP, dA, dX, dI, jac ? dJ : nullptr, dOut};
    wy_refine_eval_kernel<<<n, kRefineThreads, 0, s->stream>>>(P, a);
    wy_refine_normal_kernel<<<n, kRefineThreads, 0, s->stream>>>(P, a);
    s->launches += 2;
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    // with J, everything; without, only scale, chi^2 and sum w Io^2 of each structure
    err = jac ? cudaMemcpyAsync(outH.data(), dOut, (size_t)n * outStride * sizeof(double), cudaMemcpyDeviceToHost,
                                s->stream)
              : cudaMemcpy2DAsync(outH.data(), outStride * sizeof(double), dOut, outStride * sizeof(double),
                                  4 * sizeof(double), (size_t)n, cudaMemcpyDeviceToHost, s->stream);
    if (err != cudaSuccess) return err;
    return cudaStreamSynchronize(s->stream);
  };
  std::vector<double> cur(coords, coords + (size_t)n * nP), start;
  for (int i = 0; i < n; ++i) project(i, cur.data() + (size_t)i * nP);
  start = cur;
  if ((e = evaluate(cur, false)) != cudaSuccess) { release(); return cuda_error(e, "refinement evaluation"); }
  std::vector<double> scale(n), chi(n), oo(n), lambda(n, o.lambda0);
  std::vector<int> steps(n, 0), conv(n, 0), done(n, 0);
  for (int i = 0; i < n; ++i) {
    scale[i] = outH[(size_t)i * outStride];
    chi[i] = outH[(size_t)i * outStride + 1];
    oo[i] = outH[(size_t)i * outStride + 2];
    if (r_start) r_start[i] = oo[i] > 0 ? std::sqrt(chi[i] / oo[i]) : NAN;
  }
  std::vector<double> JTJ((size_t)n * nP * nP), JTr((size_t)n * nP), trial(cur);
  for (int iter = 0; iter < o.max_iter; ++iter) {
    bool any = false;
    for (int i = 0; i < n; ++i) any |= !done[i];
    if (!any) break;
    if ((e = evaluate(cur, true)) != cudaSuccess) { release(); return cuda_error(e, "refinement normal equations"); }
    std::vector<int> searching(n, 0), stepped(n, 0);
    for (int i = 0; i < n; ++i) {
      if (done[i]) continue;
      const double *oh = outH.data() + (size_t)i * outStride;
      scale[i] = oh[0];
      chi[i] = oh[1];
      std::copy(oh + 4, oh + 4 + nP, JTr.begin() + (size_t)i * nP);
      std::copy(oh + 4 + nP, oh + 4 + nP + (size_t)nP * nP, JTJ.begin() + (size_t)i * nP * nP);
      searching[i] = 1;
    }
    for (;;) {
      std::vector<int> hasTrial(n, 0);
      bool anySearch = false, anyTrial = false;
      for (int i = 0; i < n; ++i) {
        if (!searching[i]) continue;
        if (!(lambda[i] < o.lambda_max)) { searching[i] = 0; continue; }
        anySearch = true;
        std::vector<double> aug(JTJ.begin() + (size_t)i * nP * nP, JTJ.begin() + (size_t)(i + 1) * nP * nP);
        double dmax = 0;
        for (int q = 0; q < nP; ++q) dmax = std::max(dmax, aug[(size_t)q * nP + q]);
        if (!(dmax > 0)) { conv[i] = 1; searching[i] = 0; continue; }
        for (int q = 0; q < nP; ++q) aug[(size_t)q * nP + q] += lambda[i] * std::max(aug[(size_t)q * nP + q], 1e-6 * dmax);
        std::vector<double> rhs(JTr.begin() + (size_t)i * nP, JTr.begin() + (size_t)(i + 1) * nP), dx;
        if (!refine_solve(aug, rhs, nP, dx)) { lambda[i] *= o.lambda_up; continue; }
        // back from the constrained space: the position moves by P du
        for (int si = 0; si < ms; ++si) {
          const ProjFix &pf = s->projHost[(size_t)assign[i] * ms + si];
          const double d0 = dx[3 * si], d1 = dx[3 * si + 1], d2 = dx[3 * si + 2];
          for (int c = 0; c < 3; ++c)
            dx[3 * si + c] = (pf.num[3 * c] * d0 + pf.num[3 * c + 1] * d1 + pf.num[3 * c + 2] * d2) / (double)pf.den;
        }
        double big = 0;
        for (int q = 0; q < nP; ++q) big = std::max(big, std::fabs(dx[q]));
        const double cap = big > o.max_step ? o.max_step / big : 1.0;
        double *t = trial.data() + (size_t)i * nP;
        const double *c0 = cur.data() + (size_t)i * nP;
        for (int q = 0; q < nP; ++q) t[q] = c0[q] + cap * dx[q];
        project(i, t);
        hasTrial[i] = 1;
        anyTrial = true;
      }
      if (!anySearch) break;
      if (!anyTrial) continue;
      for (int i = 0; i < n; ++i)
        if (!hasTrial[i]) std::copy(cur.begin() + (size_t)i * nP, cur.begin() + (size_t)(i + 1) * nP, trial.begin() + (size_t)i * nP);
      if ((e = evaluate(trial, false)) != cudaSuccess) { release(); return cuda_error(e, "refinement trial"); }
      for (int i = 0; i < n; ++i) {
        if (!hasTrial[i]) continue;
        const double sTr = outH[(size_t)i * outStride], chiTr = outH[(size_t)i * outStride + 1];
        if (chiTr < chi[i]) {
          double moved = 0;
          for (int q = 0; q < nP; ++q)
            moved = std::max(moved, std::fabs(trial[(size_t)i * nP + q] - cur[(size_t)i * nP + q]));
          const double rel = (chi[i] - chiTr) / std::max(chi[i], 1e-300);
          std::copy(trial.begin() + (size_t)i * nP, trial.begin() + (size_t)(i + 1) * nP, cur.begin() + (size_t)i * nP);
          scale[i] = sTr;
          chi[i] = chiTr;
          lambda[i] = std::max(lambda[i] * o.lambda_down, 1e-12);
          stepped[i] = 1;
          steps[i]++;
          if (moved < o.tol_step || rel < o.tol_chi) conv[i] = 1;
          searching[i] = 0;
        } else {
          lambda[i] *= o.lambda_up;
        }
      }
    }
    for (int i = 0; i < n; ++i)
      if (!done[i] && (conv[i] || !stepped[i])) done[i] = 1;
  }
  if ((e = evaluate(cur, false)) != cudaSuccess) { release(); return cuda_error(e, "refinement evaluation"); }
  for (int i = 0; i < n; ++i) {
    const double c = outH[(size_t)i * outStride + 1], w = outH[(size_t)i * outStride + 2];
    if (r_final) r_final[i] = w > 0 ? std::sqrt(c / w) : NAN;
    if (chi2) chi2[i] = c;
    if (iterations) iterations[i] = steps[i];
    if (converged) converged[i] = conv[i];
  }
  std::copy(cur.begin(), cur.end(), coords);
  release();
  return P6_OK;
}
