/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 CPU restatement of the reference's Wyckoff-search trial evaluation.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library; the product path never calls it.
 *
 * Parity pinning: the reference's implementation is JavaScript + WGSL and cannot
 * run in this environment (no JS engine, no WebGPU).  These functions restate the
 * reference arithmetic line by line, and tests pin them against the reference's
 * own known-answer tests (js/swarm_wyckoff.js wR2 identity, the centring identity
 * of tests/regressions.test.cjs:1618-1645) and against closed forms.
 *
 *   p6o_wy_fitness      js/swarm_wyckoff.js:679-766 (swFitnessOnCpu): project the
 *                       sites, expand with genPack, group sums, 1 - wR2.
 *   p6o_wy_penalty      swarm_reflection.wgsl:893-1130 (clash floor, nearest-
 *                       neighbour rules, counted shells over the 27-image shell,
 *                       shape cosines, surplus count), times penScale.
 *   p6o_wy_accept       swarm_reflection.wgsl:1156-1268 (incumbent re-scored at
 *                       the current penScale, Metropolis on exp(df/T), step size
 *                       Robbins-Monro update, best-ever cache rule).
 *   p6o_wy_expand_fixed the orbit expansion in 32-bit fixed point (the kernel's
 *                       representation): X_g = R X_s + T mod 2^32, bit-exact.
 *   p6o_wy_generation   one full generation for many particles (proposal,
 *                       projection, fitness, penalty, Metropolis) in FP64 with
 *                       OpenMP over particles: the timed CPU baseline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_PI 6.283185307179586476925286766559
#define NO_NEIGHBOUR 1.0e9
#define NO_PARTNER_CHARGE 5.0
#define COORD_SOFT_A 0.25

/* -------------------------------------------------------------------------- */
/* swFitnessOnCpu                                                              */
/* -------------------------------------------------------------------------- */
static void project_site(const float *sp, double x, double y, double z, double *o)
{
    double ox = sp[0] * x + sp[1] * y + sp[2] * z + sp[9];
    double oy = sp[3] * x + sp[4] * y + sp[5] * z + sp[10];
    double oz = sp[6] * x + sp[7] * y + sp[8] * z + sp[11];
    o[0] = ox - floor(ox);
    o[1] = oy - floor(oy);
    o[2] = oz - floor(oz);
}

/* Expand projected sites into the generated cell (FP64), as the kernel does. */
static void expand(const double *proj, const uint32_t *genPack, int nTot, const float *symPacked, int nElem,
                   double *gx, double *gy, double *gz, int *gT, uint8_t *gSkip)
{
    for (int i = 0; i < nTot; i++) {
        uint32_t pk = genPack[i];
        gSkip[i] = (pk >> 24) & 1u;
        int site = pk & 0xFF, op = (pk >> 8) & 0xFFF, ty = (pk >> 20) & 0xF;
        double px = proj[site * 3], py = proj[site * 3 + 1], pz = proj[site * 3 + 2];
        const float *b = symPacked + op * 12;
        double nx = px * b[0] + py * b[1] + pz * b[2] + b[9];
        double ny = px * b[3] + py * b[4] + pz * b[5] + b[10];
        double nz = px * b[6] + py * b[7] + pz * b[8] + b[11];
        gx[i] = nx - floor(nx);
        gy[i] = ny - floor(ny);
        gz[i] = nz - floor(nz);
        int maxT = (nElem > 1 ? nElem : 1) - 1;
        gT[i] = ty < maxT ? ty : maxT;
    }
}

static double wr2_fitness(double scc, double soo, double sco)
{
    double den = scc * soo;
    if (!(den > 1e-20) || !(sco > 0)) return 0.0;
    double explained = (sco * sco) / den;
    if (explained < 0) explained = 0;
    if (explained > 1) explained = 1;
    double v = 1.0 - sqrt(fmax(0.0, 1.0 - explained));
    if (v < 0) v = 0;
    if (v > 1) v = 1;
    return v;
}

/* Group sums over already-expanded atoms.  sums[0..2] = scc, soo, sco. */
static void group_sums(const double *gx, const double *gy, const double *gz, const int *gT, const uint8_t *gSkip,
                       int nTot, const float *groupMeta, int nGroups, int stride, const uint32_t *reflPack,
                       const float *fTab, int nElem, int centro, double *sums)
{
    double scc = 0, soo = 0, sco = 0;
    for (int g = 0; g < nGroups; g++) {
        const float *gm = groupMeta + (size_t)g * stride;
        int start = (int)gm[0], count = (int)gm[1];
        double iObs = gm[2];
        double wgt = stride >= 4 ? gm[3] : 1.0;
        if (!(wgt > 0)) continue;
        double iCalc = 0;
        for (int m = 0; m < count; m++) {
            int r = start + m;
            uint32_t pk = reflPack[r * 2];
            int h = (int)(pk & 0x3FF) - 512, k = (int)((pk >> 10) & 0x3FF) - 512, l = (int)((pk >> 20) & 0x3FF) - 512;
            double mult = reflPack[r * 2 + 1];
            const float *f = fTab + (size_t)r * nElem;
            double fr = 0, fi = 0;
            for (int a = 0; a < nTot; a++) {
                if (gSkip[a]) continue;
                double q = h * gx[a] + k * gy[a] + l * gz[a];
                double ph = TWO_PI * (q - floor(q));
                fr += f[gT[a]] * cos(ph);
                if (!centro) fi += f[gT[a]] * sin(ph);
            }
            iCalc += mult * (fr * fr + fi * fi);
        }
        scc += wgt * iCalc * iCalc;
        soo += wgt * iObs * iObs;
        sco += wgt * iCalc * iObs;
    }
    sums[0] = scc;
    sums[1] = soo;
    sums[2] = sco;
}

/*
 * swFitnessOnCpu.  coords: nSites*3 raw (unprojected) coordinates.  siteProj:
 * this assignment's row (nSites*12).  Returns 1 - wR2; sums (may be NULL)
 * receives scc, soo, sco.  centro = 1 drops the sine terms (exact for a
 * centrosymmetric cell; the reference always sums both, which is identical).
 */
double p6o_wy_fitness(const double *coords, int nSites, const float *siteProj, const uint32_t *genPack, int nTot,
                      const float *symPacked, const float *groupMeta, int nGroups, int stride,
                      const uint32_t *reflPack, const float *fTab, int nElem, int centro, double *sums)
{
    double *proj = (double *)malloc(sizeof(double) * (size_t)nSites * 3 + 8);
    double *gx = (double *)malloc(sizeof(double) * (size_t)nTot * 3 + 8);
    int *gT = (int *)malloc(sizeof(int) * (size_t)nTot + 8);
    uint8_t *gS = (uint8_t *)malloc((size_t)nTot + 8);
    for (int s = 0; s < nSites; s++) project_site(siteProj + s * 12, coords[s * 3], coords[s * 3 + 1], coords[s * 3 + 2], proj + s * 3);
    expand(proj, genPack, nTot, symPacked, nElem, gx, gx + nTot, gx + 2 * nTot, gT, gS);
    double tmp[3];
    group_sums(gx, gx + nTot, gx + 2 * nTot, gT, gS, nTot, groupMeta, nGroups, stride, reflPack, fTab, nElem, centro, tmp);
    if (sums) { sums[0] = tmp[0]; sums[1] = tmp[1]; sums[2] = tmp[2]; }
    free(proj); free(gx); free(gT); free(gS);
    return wr2_fitness(tmp[0], tmp[1], tmp[2]);
}

/*
 * Same fitness from already-projected coordinates (no projection step): used
 * when the coordinates come from a kernel trace, where they are already on the
 * Wyckoff subspace in fixed point.
 */
double p6o_wy_fitness_projected(const double *proj, const uint32_t *genPack, int nTot, const float *symPacked,
                                const float *groupMeta, int nGroups, int stride, const uint32_t *reflPack,
                                const float *fTab, int nElem, int centro, double *sums)
{
    double *gx = (double *)malloc(sizeof(double) * (size_t)nTot * 3 + 8);
    int *gT = (int *)malloc(sizeof(int) * (size_t)nTot + 8);
    uint8_t *gS = (uint8_t *)malloc((size_t)nTot + 8);
    expand(proj, genPack, nTot, symPacked, nElem, gx, gx + nTot, gx + 2 * nTot, gT, gS);
    double tmp[3];
    group_sums(gx, gx + nTot, gx + 2 * nTot, gT, gS, nTot, groupMeta, nGroups, stride, reflPack, fTab, nElem, centro, tmp);
    if (sums) { sums[0] = tmp[0]; sums[1] = tmp[1]; sums[2] = tmp[2]; }
    free(gx); free(gT); free(gS);
    return wr2_fitness(tmp[0], tmp[1], tmp[2]);
}

/* -------------------------------------------------------------------------- */
/* Fixed-point orbit expansion (the kernel's representation).                  */
/* rint: 9 ints per operator; tfix: 3 u32 per operator (translation * 2^32).   */
/* -------------------------------------------------------------------------- */
void p6o_wy_expand_fixed(const uint32_t *siteX, const uint32_t *genPack, int nTot, const int32_t *rint,
                         const uint32_t *tfix, uint32_t *out)
{
    for (int i = 0; i < nTot; i++) {
        uint32_t pk = genPack[i];
        int site = pk & 0xFF, op = (pk >> 8) & 0xFFF;
        const uint32_t *x = siteX + site * 3;
        const int32_t *r = rint + op * 9;
        for (int c = 0; c < 3; c++) {
            uint32_t v = (uint32_t)r[c * 3] * x[0] + (uint32_t)r[c * 3 + 1] * x[1] + (uint32_t)r[c * 3 + 2] * x[2] + tfix[op * 3 + c];
            out[i * 3 + c] = v;
        }
    }
}

/* -------------------------------------------------------------------------- */
/* Penalties: swarm_reflection.wgsl:893-1130, FP64.                            */
/* -------------------------------------------------------------------------- */
typedef struct {
    double o[9];   /* reduced-basis fractional -> Cartesian, row-major */
    double r[9];   /* original fractional -> reduced fractional, row-major */
    int minImageShell;
    int countShell;
    double penClash, penBond, penCoord, penGeom, penScale;
} p6o_geom;

static void frac_delta(const p6o_geom *G, const double *p1, const double *p2, double *q)
{
    double d[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
    for (int i = 0; i < 3; i++) {
        double v = G->r[i * 3] * d[0] + G->r[i * 3 + 1] * d[1] + G->r[i * 3 + 2] * d[2];
        q[i] = v - floor(v + 0.5); /* WGSL round(): half away from zero; ties do not occur for real data */
    }
}

static void cart_vec(const p6o_geom *G, const double *t, double *c)
{
    for (int i = 0; i < 3; i++) c[i] = G->o[i * 3] * t[0] + G->o[i * 3 + 1] * t[1] + G->o[i * 3 + 2] * t[2];
}

static double cart_len(const p6o_geom *G, const double *t)
{
    double c[3];
    cart_vec(G, t, c);
    return sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

static double cart_dist(const p6o_geom *G, const double *p1, const double *p2)
{
    double q[3];
    frac_delta(G, p1, p2, q);
    double best = 1e30;
    int S = G->minImageShell;
    for (int i = -S; i <= S; i++)
        for (int j = -S; j <= S; j++)
            for (int k = -S; k <= S; k++) {
                double t[3] = {q[0] + i, q[1] + j, q[2] + k}, c[3];
                cart_vec(G, t, c);
                double d2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
                if (d2 < best) best = d2;
            }
    return sqrt(best);
}

static double geom_cos_error(int code, double c)
{
    switch (code) {
    case 1: return c + 1.0;
    case 2: return c + 0.5;
    case 3: return c + 0.3333333;
    case 4:
    case 5: return fmin(fabs(c), fabs(c + 1.0));
    default: return 0.0;
    }
}

/*
 * Penalty of one generated cell.  gx/gy/gz: nTot fractional positions, gT
 * types.  tables: [zByType | rMin | rules], rMinOff/ruleOff offsets into it.
 * maxBondRules, maxCoordSlots: the capacities the kernel was compiled with
 * (rules past them are ignored exactly as the kernel ignores them).
 * Returns pen * penScale.
 */
double p6o_wy_penalty(const double *gx, const double *gy, const double *gz, const int *gT, int nTot, int nElem,
                      const float *tables, int rMinOff, int ruleOff, int nRules, int maxCoordSlots, int geomSlots,
                      const p6o_geom *G)
{
    double ruleMin[32], ruleMax[32], ruleN[32];
    int ruleA[32], ruleB[32], ruleMode[32], ruleGeom[32], slotOff[32], slotN[32];
    if (nRules > 32) nRules = 32;
    for (int k = 0; k < nRules; k++) {
        const float *rb = tables + ruleOff + k * 7;
        ruleA[k] = (int)rb[0];
        ruleB[k] = (int)rb[1];
        ruleMin[k] = rb[2];
        ruleMax[k] = rb[3];
        ruleN[k] = rb[4];
        ruleMode[k] = (int)rb[5];
        ruleGeom[k] = geomSlots >= maxCoordSlots ? (int)rb[6] : 0;
    }
    int acc = 0;
    for (int k = 0; k < nRules; k++) {
        slotOff[k] = acc;
        int nk = 0;
        if (ruleMode[k] != 0) {
            nk = (int)ruleN[k];
            if (nk > maxCoordSlots - acc) nk = maxCoordSlots - acc;
        }
        slotN[k] = nk;
        acc += nk;
    }
    int slotTotal = acc;
    double shellLen[27];
    for (int s = 0; s < 27; s++) {
        double t[3] = {(double)(s / 9 - 1), (double)((s / 3) % 3 - 1), (double)(s % 3 - 1)};
        shellLen[s] = cart_len(G, t);
    }
    double *slot = (double *)malloc(sizeof(double) * (slotTotal > 0 ? slotTotal : 1));
    double (*slotV)[3] = (double (*)[3])malloc(sizeof(double) * 3 * (slotTotal > 0 ? slotTotal : 1));
    double pen = 0;
    for (int i = 0; i < nTot; i++) {
        int ti = gT[i];
        double pi[3] = {gx[i], gy[i], gz[i]};
        uint32_t myRules = 0;
        for (int k = 0; k < nRules; k++) if (ruleA[k] == ti) myRules |= 1u << k;
        double nearest[32], inWindow[32];
        for (int k = 0; k < 32; k++) { nearest[k] = NO_NEIGHBOUR; inWindow[k] = 0; }
        for (int m = 0; m < slotTotal; m++) slot[m] = NO_NEIGHBOUR;
        for (int j = 0; j < nTot; j++) {
            int tj = gT[j];
            double pj[3] = {gx[j], gy[j], gz[j]};
            double d = cart_dist(G, pi, pj);
            if (j != i) {
                double dmin = tables[rMinOff + ti * nElem + tj];
                if (j > i && d < dmin) {
                    double overlap = (dmin - d) / fmax(dmin, 1e-3);
                    pen += G->penClash * (1.0 + 9.0 * overlap);
                }
            }
            if (myRules == 0) continue;
            double qf[3];
            frac_delta(G, pi, pj, qf);
            double dq = cart_len(G, qf);
            for (int k = 0; k < nRules; k++) {
                if (!(myRules & (1u << k))) continue;
                if (ruleB[k] != tj) continue;
                int nk = slotN[k];
                int counted = nk > 0;
                if (j != i) nearest[k] = fmin(nearest[k], d);
                double cutoff = ruleMax[k];
                if (counted) cutoff = fmax(cutoff, slot[slotOff[k] + nk - 1]);
                int S = G->countShell;
                for (int sa = -S; sa <= S; sa++)
                    for (int sb = -S; sb <= S; sb++)
                        for (int sc = -S; sc <= S; sc++) {
                            int si = (sa + 1) * 9 + (sb + 1) * 3 + (sc + 1);
                            if (S == 1 && shellLen[si] - dq > cutoff) continue;
                            double t[3] = {qf[0] + sa, qf[1] + sb, qf[2] + sc}, dv[3];
                            cart_vec(G, t, dv);
                            double dd = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                            if (dd < 1.0e-4 && j == i) continue;
                            if (dd >= ruleMin[k] && dd <= ruleMax[k]) inWindow[k] += 1.0;
                            if (counted) {
                                int lo = slotOff[k], hi = lo + nk;
                                int shaped = ruleGeom[k] != 0;
                                if (dd < slot[hi - 1]) {
                                    int m = hi - 1;
                                    while (m > lo && slot[m - 1] > dd) {
                                        slot[m] = slot[m - 1];
                                        if (shaped) { slotV[m][0] = slotV[m - 1][0]; slotV[m][1] = slotV[m - 1][1]; slotV[m][2] = slotV[m - 1][2]; }
                                        m--;
                                    }
                                    slot[m] = dd;
                                    if (shaped) { slotV[m][0] = dv[0]; slotV[m][1] = dv[1]; slotV[m][2] = dv[2]; }
                                    cutoff = fmax(ruleMax[k], slot[hi - 1]);
                                }
                            }
                        }
            }
        }
        for (int k = 0; k < nRules; k++) {
            if (!(myRules & (1u << k))) continue;
            if (ruleMode[k] == 0) {
                double nk = nearest[k];
                if (nk < NO_NEIGHBOUR && nk > ruleMax[k]) pen += G->penBond * (nk - ruleMax[k]);
            } else {
                int nk = slotN[k];
                double deficit = 0;
                for (int m = 0; m < nk; m++) {
                    double dm = slot[slotOff[k] + m];
                    if (dm >= NO_NEIGHBOUR) deficit += NO_PARTNER_CHARGE;
                    else {
                        double miss = fmax(0.0, dm - ruleMax[k]) + fmax(0.0, ruleMin[k] - dm);
                        deficit += miss * (1.0 + miss / COORD_SOFT_A);
                    }
                }
                pen += G->penBond * deficit;
                if (ruleGeom[k] != 0 && nk >= 2) {
                    int lo = slotOff[k];
                    double g = 0;
                    for (int m = 0; m + 1 < nk; m++) {
                        double dm = slot[lo + m];
                        if (dm >= NO_NEIGHBOUR) continue;
                        for (int n = m + 1; n < nk; n++) {
                            double dn = slot[lo + n];
                            if (dn >= NO_NEIGHBOUR) continue;
                            double c = (slotV[lo + m][0] * slotV[lo + n][0] + slotV[lo + m][1] * slotV[lo + n][1] +
                                        slotV[lo + m][2] * slotV[lo + n][2]) / fmax(dm * dn, 1e-6);
                            double e = geom_cos_error(ruleGeom[k], c);
                            g += e * e;
                        }
                    }
                    pen += G->penBond * G->penGeom * g;
                }
                if (ruleMode[k] == 1) pen += G->penCoord * fmax(0.0, inWindow[k] - ruleN[k]);
            }
        }
    }
    free(slot);
    free(slotV);
    return pen * G->penScale;
}

/* Penalty from projected site coordinates (expands with genPack/symPacked first). */
double p6o_wy_penalty_sites(const double *proj, const uint32_t *genPack, int nTot, const float *symPacked, int nElem,
                            const float *tables, int rMinOff, int ruleOff, int nRules, int maxCoordSlots,
                            int geomSlots, const p6o_geom *G)
{
    double *gx = (double *)malloc(sizeof(double) * (size_t)nTot * 3 + 8);
    int *gT = (int *)malloc(sizeof(int) * (size_t)nTot + 8);
    uint8_t *gS = (uint8_t *)malloc((size_t)nTot + 8);
    expand(proj, genPack, nTot, symPacked, nElem, gx, gx + nTot, gx + 2 * nTot, gT, gS);
    double p = p6o_wy_penalty(gx, gx + nTot, gx + 2 * nTot, gT, nTot, nElem, tables, rMinOff, ruleOff, nRules,
                              maxCoordSlots, geomSlots, G);
    free(gx); free(gT); free(gS);
    return p;
}

/* -------------------------------------------------------------------------- */
/* Acceptance (swarm_reflection.wgsl:1156-1268).                               */
/* st: fit, cc, pen, stepSize, temp, bestFit, bestCC, bestPen (doubles).        */
/* u: the uniform deviate the Metropolis test draws (used only if f_new < f_old)*/
/* Returns 1 if accepted; updates st in place.                                  */
/* -------------------------------------------------------------------------- */
int p6o_wy_accept(double *st, double cc, double pen, double penScale, double u, double stepUp, double stepDown,
                  double stepMin, double stepMax, int *bestUpdated)
{
    double f_new = cc - pen;
    double f_old = st[0];
    if (f_old > -1.0e29) f_old = st[1] - st[2] * penScale;
    int accept = 0;
    if (f_new >= f_old) accept = 1;
    else {
        double prob = exp((f_new - f_old) / fmax(st[4], 1e-9));
        if (u < prob) accept = 1;
    }
    *bestUpdated = 0;
    if (accept) {
        st[0] = f_new;
        st[1] = cc;
        st[2] = pen / fmax(penScale, 1e-9);
        int hasBest = st[5] > -1.0e29;
        double bestRescored = hasBest ? st[6] - st[7] * penScale : -1.0e30;
        if (f_new > bestRescored) {
            st[5] = f_new;
            st[6] = cc;
            st[7] = pen / fmax(penScale, 1e-9);
            *bestUpdated = 1;
        }
    }
    double s = st[3] * (accept ? stepUp : stepDown);
    st[3] = fmin(fmax(s, stepMin), stepMax);
    return accept;
}

/* -------------------------------------------------------------------------- */
/* CPU generation (timed baseline).                                            */
/* -------------------------------------------------------------------------- */
typedef struct {
    const uint32_t *genPack;   /* nAssign * nTot */
    const float *symPacked;
    const float *siteProj;     /* nAssign * maxSites * 12 */
    const uint32_t *reflPack;
    const float *groupMeta;
    const float *fTab;
    const float *tables;
    int nTot, maxSites, nElem, nGroupsActive, stride, rMinOff, ruleOff, nRules, maxCoordSlots, geomSlots, centro;
    double stepUp, stepDown, stepMin, stepMax;
} p6o_problem;

static inline uint32_t mulberry_next(uint32_t *s)
{
    *s += 0x6D2B79F5u;
    uint32_t t = *s;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return t ^ (t >> 14);
}
static inline double uni(uint32_t *s) { return mulberry_next(s) / 4294967296.0; }
static inline double gauss(uint32_t *s)
{
    double u1 = fmax(uni(s), 1e-12), u2 = uni(s);
    return sqrt(-2.0 * log(u1)) * cos(TWO_PI * u2);
}

/*
 * One generation for nParticles particles.  pos: nParticles*maxSites*3
 * (current, projected), assign: per particle, st: 8 doubles per particle
 * (see p6o_wy_accept), seeds: per-particle RNG state.  Returns the number of
 * trials evaluated.  nThreads <= 0 uses all available threads.
 */
long p6o_wy_generation(const p6o_problem *P, const p6o_geom *G, int nParticles, double *pos, const uint32_t *assign,
                       double *st, uint32_t *seeds, int nThreads)
{
#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    long trials = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : trials)
    for (int p = 0; p < nParticles; p++) {
        int A = (int)assign[p];
        const float *sp = P->siteProj + (size_t)A * P->maxSites * 12;
        const uint32_t *gp = P->genPack + (size_t)A * P->nTot;
        double prop[32 * 3];
        double *cur = pos + (size_t)p * P->maxSites * 3;
        uint32_t *rs = seeds + p;
        double sd = st[p * 8 + 3];
        /* proposal: collective with probability 1/4, otherwise one free site */
        int nFree = 0, pick = -1;
        int collective = !(uni(rs) < 0.75);
        for (int s = 0; s < P->maxSites; s++) {
            double norm = 0;
            for (int j = 0; j < 9; j++) norm += fabs(sp[s * 12 + j]);
            if (norm > 1e-6) { nFree++; if (uni(rs) < 1.0 / nFree) pick = s; }
        }
        for (int s = 0; s < P->maxSites; s++) {
            int moving = collective || s == pick;
            double x = cur[s * 3], y = cur[s * 3 + 1], z = cur[s * 3 + 2];
            if (moving) {
                x += gauss(rs) * sd;
                y += gauss(rs) * sd;
                z += gauss(rs) * sd;
                project_site(sp + s * 12, x, y, z, prop + s * 3);
            } else {
                prop[s * 3] = x; prop[s * 3 + 1] = y; prop[s * 3 + 2] = z;
            }
        }
        double *gx = (double *)malloc(sizeof(double) * (size_t)P->nTot * 3 + 8);
        int *gT = (int *)malloc(sizeof(int) * (size_t)P->nTot + 8);
        uint8_t *gS = (uint8_t *)malloc((size_t)P->nTot + 8);
        expand(prop, gp, P->nTot, P->symPacked, P->nElem, gx, gx + P->nTot, gx + 2 * P->nTot, gT, gS);
        double sums[3];
        group_sums(gx, gx + P->nTot, gx + 2 * P->nTot, gT, gS, P->nTot, P->groupMeta, P->nGroupsActive, P->stride,
                   P->reflPack, P->fTab, P->nElem, P->centro, sums);
        double cc = wr2_fitness(sums[0], sums[1], sums[2]);
        double pen = p6o_wy_penalty(gx, gx + P->nTot, gx + 2 * P->nTot, gT, P->nTot, P->nElem, P->tables,
                                    P->rMinOff, P->ruleOff, P->nRules, P->maxCoordSlots, P->geomSlots, G);
        free(gx); free(gT); free(gS);
        int bu;
        double u = uni(rs);
        if (p6o_wy_accept(st + p * 8, cc, pen, G->penScale, u, P->stepUp, P->stepDown, P->stepMin, P->stepMax, &bu))
            memcpy(cur, prop, sizeof(double) * P->maxSites * 3);
        trials++;
    }
    return trials;
}

int p6o_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
