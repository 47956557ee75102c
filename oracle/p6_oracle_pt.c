/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 CPU restatement of the reference's Rietveld cost for parallel
 * tempering, and of its CPU parallel tempering.
 *
 *   p6o_pt_cost      chi^2 = sum_{w>0} w (y - ycalc)^2 of one parameter vector:
 *                    js/rietveld_core.js:1878-1889 (cost), 1152-1165
 *                    (evalDataset), 855-917 (evalPhase, render), 920-931 and
 *                    640-646 (Chebyshev background), 719-747 (geometry),
 *                    749-822 (structure, no anomalous terms), 247-276
 *                    (generateReflections via p6o_generate_reflections),
 *                    238-245 (reflectionDmin); js/profile.js:108-131
 *                    (calculatePeakShift), 149-219 (width floors), 426-550
 *                    (TCH widths, calculateProfileWidths), 552-567
 *                    (getPeakFWHM), 603-760 (prepareVoigt, evalVoigt),
 *                    1013-1090 (buildPeakContributions: all K-alpha-1, then
 *                    all K-alpha-2), 1131-1159 (intensityDerivativeColumn);
 *                    js/constants.js:138-145 (softPositive), 155-201
 *                    (pseudo-Voigt constants, pvMixCoeffs), 248-251 (GSAS
 *                    units); js/crystal.js:480-497 (Lp).
 *   p6o_pt_temper    js/rietveld_core.js:2171-2241 (temper): one xorshift32
 *                    stream, nv single-coordinate proposals per replica per
 *                    sweep, reflecting bounds, Metropolis on chi^2/2, even/odd
 *                    adjacent exchanges.
 *
 * Scope of the restatement: one phase, one dataset, X-rays, TCH profile
 * without Stephens terms or SL/HL asymmetry, no preferred orientation, no
 * displacement or transparency, Chebyshev background -- the model of the
 * parallel-tempering benchmark configuration.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI_ 3.14159265358979323846
#define DEG2RAD (PI_ / 180.0)
#define R2D (180.0 / PI_)

int p6o_generate_reflections(const double *cell, const int *rot, const double *trans, int nOps, double dmin,
                             const int *box, int *oh, int *ok, int *ol, int *om, double *od0, int maxOut);

/* Full parameter vector layout (the values apply() produces). */
enum {
    PT_SCALE = 0, PT_A, PT_B, PT_C, PT_AL, PT_BE, PT_GA, PT_U, PT_V, PT_W, PT_X, PT_Y, PT_ZERO, PT_BISO, PT_BKG0
};

typedef struct {
    /* phase */
    int nOps;
    const int *rot;        /* nOps*9 */
    const double *trans;   /* nOps*3 */
    int nReps;
    const int *repRot;     /* nReps*9 */
    const double *repTrans;/* nReps*3 */
    int nAtoms;
    const double *pos;     /* nAtoms*3 fractional */
    const double *wMult;   /* site multiplicity / nReps, per atom */
    const double *occ;     /* per atom */
    const double *ffA, *ffB, *ffC; /* 5, 5, 1 per atom */
    /* dataset */
    int n;
    const double *tth, *y, *w;
    double lambda1, lambda2, ratio, polK, minFwhm;
    int nBkg;
    double dmin;           /* > 0: use this; <= 0: reflectionDmin of the parameters */
    /* March-Dollase preferred orientation: r = v[PT_BKG0 + nBkg], direction poDir (reciprocal lattice) */
    int hasPo;
    double poDir[3];
    /* SL/HL asymmetry: SL = v[PT_BKG0 + nBkg + hasPo], HL the next entry */
    int hasAsym;
    /* 0 Rietveld; 1 WPPF / Le Bail (js/pt_gpu.js:259-297): every active
     * reflection's height is free and non-negative, solved by NNLS against
     * y - background (atoms unused) */
    int method;
    /* sample displacement and transparency (js/pt_gpu.js:169-171, :355): the
     * two full-vector entries after SL, HL (or 'po', or the background) */
    int hasShift;
} p6o_pt_problem;

static const double GCONV = 0.023548200450309493;   /* sqrt(8 ln 2) / 100 */
static const double LCONV = 0.01;
static const double CG = 2.772588722239781;         /* 4 ln 2 */
static const double WIN_G = 8.0, WIN_L = 25.0, WIN_MAX = 10.0;

static double pv_g0(void) { return 2.0 * sqrt(log(2.0) / PI_); }
static double pv_l0(void) { return 2.0 / PI_; }

static double soft_positive(double x, double f)
{
    if (!isfinite(x)) return f;
    double h = hypot(x, 2 * f);
    return x < 0 ? f * (f / (0.5 * h - 0.5 * x)) : 0.5 * x + 0.5 * h;
}

static double soft_floor(double x, double f)
{
    if (!isfinite(x) || !(x > 0)) return f;
    if (!(f > 0)) return x;
    double r = x / f;
    if (r > 20) return x;
    return f * pow(pow(r, 4) + 1, 0.25);
}

static double peak_fwhm(double gG0, double gL0)
{
    double gG = fmax(1e-9, gG0 != 0 ? gG0 : 1e-9), gL = fmax(1e-9, gL0 != 0 ? gL0 : 1e-9);
    double s = pow(gG, 5) + 2.69269 * pow(gG, 4) * gL + 2.42843 * pow(gG, 3) * pow(gL, 2) +
               4.47163 * pow(gG, 2) * pow(gL, 3) + 0.07842 * gG * pow(gL, 4) + pow(gL, 5);
    if (s < 0 || !isfinite(s)) return fmax(fmax(gG, gL), 1e-6);
    return fmax(1e-6, pow(s, 0.2));
}

typedef struct {
    double x0, inv, cL, cG, pedestal, maxd, area, asym;
} voigt_t;

/* evalVoigt (profile.js:731-759), TCH: the asymmetry stretches one flank. */
static double eval_voigt(double x, const voigt_t *p, double maxd, double pedestal)
{
    double delta = x - p->x0;
    if (delta > maxd || delta < -maxd) return 0.0;
    if (p->asym != 0 && fabs(delta) >= 1e-9) {
        double t = fmax(-0.95, fmin(0.95, p->asym * delta));
        delta /= (1.0 - t);
    }
    double dg = (delta * p->inv) * (delta * p->inv);
    double g = exp(-CG * dg);
    double l = 1.0 / (1.0 + 4.0 * dg);
    double v = p->cL * l + p->cG * g - pedestal;
    return v > 0 ? v : 0.0;
}

/* sharkoErfc (profile.js:791-797): Numerical Recipes' erfcc, fractional error below 1.2e-7. */
static double erfcc(double x)
{
    double z = fabs(x), t = 1 / (1 + 0.5 * z);
    double ans = t * exp(-z * z - 1.26551223 + t * (1.00002368 + t * (0.37409196 + t * (0.09678418 +
                 t * (-0.18628806 + t * (0.27886807 + t * (-1.13520398 + t * (1.48851587 +
                 t * (-0.82215223 + t * 0.17087277)))))))));
    return x >= 0 ? ans : 2 - ans;
}

/* asymmetryAreaCorrection (profile.js:799-826): the area the asymmetry adds to
 * the unit-height peak; H is the TCH fwhm, R the truncation radius. */
static double asym_area_correction(const voigt_t *prep, double H, double R)
{
    static const double X[4] = {0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363};
    static const double W[4] = {0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
    if (!(prep->asym != 0) || !(R > 0)) return 0;
    voigt_t as = *prep, sy = *prep;
    as.x0 = 0; as.pedestal = 0;
    sy.x0 = 0; sy.pedestal = 0; sy.asym = 0;
    const double a = prep->asym, w = fmax(1e-6, fmax(1e-6, H));
    const double clampAt = 0.95 / fabs(a), D = fmax(R, fmin(clampAt, 4096 * w));
    double total = 0;
    for (int sd = 0; sd < 2; sd++) {
        const double side = sd ? 1 : -1;
        double lo = 0, e = 0.25 * w;
        for (;;) {
            double hi = fmin(e, D);
            for (int pass = 0; pass < 2; pass++) {
                double plo = lo, phi = hi;
                if (pass == 0) {
                    if (!(clampAt > lo && clampAt < hi)) continue;
                    phi = clampAt;
                }
                double m = 0.5 * (plo + phi), h = 0.5 * (phi - plo), sum = 0;
                for (int i = 0; i < 4; i++)
                    for (int sg = -1; sg <= 1; sg += 2) {
                        double d = side * (m + sg * h * X[i]);
                        sum += W[i] * (eval_voigt(d, &as, INFINITY, 0) - eval_voigt(d, &sy, INFINITY, 0));
                    }
                total += sum * h;
                if (pass == 0) lo = clampAt;
            }
            lo = hi;
            if (hi >= D) break;
            e *= 2;
        }
        const double k = 1 - fmax(-0.95, fmin(0.95, a * side * D));
        const double xs[2] = {D / k, D};
        double tl[2];
        for (int q = 0; q < 2; q++)
            tl[q] = prep->cL * 0.5 * H * (0.5 * PI_ - atan(2 * xs[q] / H)) +
                    prep->cG * 0.5 * H * sqrt(PI_ / CG) * erfcc(sqrt(CG) * xs[q] / H);
        total += k * tl[0] - tl[1];
    }
    return total;
}

/* prepareVoigt, TCH branch (profile.js:603-722); asymIdx >= 0: v[asymIdx] = SL, v[asymIdx + 1] = HL. */
static void prepare_tch_asym(double tthPeak, double x0, const double *v, double fwhmMin, int asymIdx, voigt_t *p)
{
    double asym = 0;
    if (asymIdx >= 0) {
        double SL = v[asymIdx], HL = v[asymIdx + 1];
        if ((SL != 0 || HL != 0) && tthPeak >= 0.1 && tthPeak < 180) {
            double th = fmax(1e-6, fmin(PI_ / 2.0 - 1e-6, tthPeak * (PI_ / 180) / 2.0)), t = tan(th);
            if (fabs(t) >= 1e-9) asym = SL / t + HL;
        }
    }
    double gG = fwhmMin, gL = fwhmMin;
    double thetaRad = tthPeak * (PI_ / 180) / 2;
    double safe = fmin(thetaRad, PI_ / 2.0 - 1e-6);
    if (!(safe < 1e-6)) {
        double tanT = tan(safe), cosT = cos(safe), cosTs = fmax(cosT, 1e-9);
        double sig2 = v[PT_U] * tanT * tanT + v[PT_V] * tanT + v[PT_W];
        double floorSq = pow(0.25 * fwhmMin / GCONV, 2);
        gG = sqrt(soft_positive(sig2, floorSq)) * GCONV;
        double gLc = v[PT_X] / cosTs + v[PT_Y] * tanT;
        gL = soft_positive(gLc, 0.25 * fwhmMin / LCONV) * LCONV;
    }
    gG = soft_floor(gG, fwhmMin);
    gL = soft_floor(gL, fwhmMin);
    double HG = fmax(1e-9, gG), HL = fmax(1e-9, gL);
    double fwhm = fmax(1e-9, peak_fwhm(HG, HL));
    double eta = 0;
    if (fwhm > 1e-9) {
        double r = HL / fwhm;
        eta = fmax(0, fmin(1, 1.36603 * r - 0.47719 * (r * r) + 0.11116 * pow(r, 3)));
    }
    /* pvMixCoeffs(eta, fwhm, fwhm) */
    double e = fmax(0, fmin(1, eta));
    double wL = e * pv_l0() / fmax(1e-12, fwhm), wG = (1 - e) * pv_g0() / fmax(1e-12, fwhm), s = wL + wG;
    double cL = e, cG = 1 - e;
    if (s > 0 && isfinite(s)) { cL = wL / s; cG = wG / s; }
    p->x0 = x0;
    p->inv = 1 / fwhm;
    p->cL = cL;
    p->cG = cG;
    p->asym = asym;
    p->area = (cL * (1 / pv_l0()) + cG * (1 / pv_g0())) * fwhm;
    double winFwhm = fmax(1e-6, fwhm);
    double etaWin = fmax(0, fmin(1, eta));
    double mult = WIN_G + (WIN_L - WIN_G) * etaWin;
    double R = fmin(WIN_MAX, mult * fmax(0.01, winFwhm) * (asym != 0 ? 2.0 : 1.0));
    p->pedestal = fmax(eval_voigt(x0 + R, p, INFINITY, 0.0), eval_voigt(x0 - R, p, INFINITY, 0.0));
    p->maxd = R;
    p->area += asym_area_correction(p, fwhm, R);
}

static void prepare_tch(double tthPeak, double x0, const double *v, double fwhmMin, voigt_t *p)
{
    prepare_tch_asym(tthPeak, x0, v, fwhmMin, -1, p);
}

static double lp_factor(double tth, double K)
{
    if (!isfinite(tth) || tth <= 0 || tth >= 180) return 1;
    double th = 0.5 * tth * DEG2RAD, s = sin(th), c = cos(th);
    if (s < 1e-6 || c < 1e-6) return 1;
    double L = 1 / (s * s * c);
    double k = (isfinite(K) && K >= 0) ? K : 1;
    double c2 = cos(tth * DEG2RAD);
    double P = (1 + k * c2 * c2) / (1 + k);
    return L * P;
}

static int lower_bound(const double *a, int n, double t)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < t) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static double inv_dsq_cell(const double *c6, double h, double k, double l, int *ok)
{
    double a = c6[0], b = c6[1], c = c6[2];
    double al = c6[3] * DEG2RAD, be = c6[4] * DEG2RAD, ga = c6[5] * DEG2RAD;
    double cA = cos(al), cB = cos(be), cG = cos(ga), sA = sin(al), sB = sin(be), sG = sin(ga);
    double vf = 1 - cA * cA - cB * cB - cG * cG + 2 * cA * cB * cG;
    *ok = 0;
    if (!(a > 0 && b > 0 && c > 0) || vf <= 1e-9 || fabs(sA) < 1e-9 || fabs(sB) < 1e-9 || fabs(sG) < 1e-9) return NAN;
    *ok = 1;
    double V = a * b * c * sqrt(vf);
    double as = b * c * sA / V, bs = a * c * sB / V, cs = a * b * sG / V;
    double cAs = (cB * cG - cA) / (sB * sG), cBs = (cA * cG - cB) / (sA * sG), cGs = (cA * cB - cG) / (sA * sB);
    return h * h * (as * as) + k * k * (bs * bs) + l * l * (cs * cs) + h * k * (2 * as * bs * cGs) +
           k * l * (2 * bs * cs * cAs) + h * l * (2 * as * cs * cBs);
}

#define AIDX(P) ((P)->hasAsym ? PT_BKG0 + (P)->nBkg + ((P)->hasPo ? 1 : 0) : -1)
#define SIDX(P) ((P)->hasShift ? PT_BKG0 + (P)->nBkg + ((P)->hasPo ? 1 : 0) + ((P)->hasAsym ? 2 : 0) : -1)

/* shift(t, disp, transp) of js/pt_gpu.js:355 in degrees: displacement
 * -disp 1e-3 cos(theta), transparency transp sin(2 theta); 0 at theta = 90
 * and wherever it is not finite (profile.js calculatePeakShift) */
static double sample_shift(const p6o_pt_problem *P, const double *v, double t)
{
    if (!P->hasShift) return 0.0;
    const double disp = v[SIDX(P)], transp = v[SIDX(P) + 1];
    const double th = t * DEG2RAD / 2;
    if (fabs(th - PI_ / 2) < 1e-6) return 0.0;
    const double d = (-disp * 0.001 * cos(th) + transp * sin(2 * th)) / DEG2RAD;
    return isfinite(d) ? d : 0.0;
}

/* Coefficients of the 1/d^2 form: aa, bb, cc, ab, bc, ac (the hk, kl, hl terms). */
static void cell_form(const double *c6, double f[6])
{
    int ok;
    f[0] = inv_dsq_cell(c6, 1, 0, 0, &ok);
    f[1] = inv_dsq_cell(c6, 0, 1, 0, &ok);
    f[2] = inv_dsq_cell(c6, 0, 0, 1, &ok);
    f[3] = inv_dsq_cell(c6, 1, 1, 0, &ok) - f[0] - f[1];
    f[4] = inv_dsq_cell(c6, 0, 1, 1, &ok) - f[1] - f[2];
    f[5] = inv_dsq_cell(c6, 1, 0, 1, &ok) - f[0] - f[2];
}

static double form_g(const double f[6], const double *a, const double *b)
{
    return a[0] * b[0] * f[0] + a[1] * b[1] * f[1] + a[2] * b[2] * f[2] + (a[0] * b[1] + a[1] * b[0]) * f[3] / 2 +
           (a[1] * b[2] + a[2] * b[1]) * f[4] / 2 + (a[0] * b[2] + a[2] * b[0]) * f[5] / 2;
}

/*
 * preferredOrientation (js/rietveld_core.js:824-853): the March-Dollase
 * factor of (h, k, l), averaged over its distinct equivalents h R under the
 * phase's operators.
 */
double p6o_po_factor(const p6o_pt_problem *P, const double *c6, double r, int h, int k, int l)
{
    if (!(r > 0) || fabs(r - 1) < 1e-12) return 1;
    double f[6];
    cell_form(c6, f);
    const double *H = P->poDir, HH = form_g(f, H, H), r2 = r * r, ir = 1 / r;
    if (!(HH > 0)) return 1;
    int seen[192 * 3], m = 0;
    double sum = 0;
    for (int o = 0; o < P->nOps && m < 192; o++) {
        const int *R = P->rot + 9 * o;
        int e[3] = {h * R[0] + k * R[3] + l * R[6], h * R[1] + k * R[4] + l * R[7], h * R[2] + k * R[5] + l * R[8]};
        int dup = 0;
        for (int q = 0; q < m && !dup; q++)
            dup = seen[3 * q] == e[0] && seen[3 * q + 1] == e[1] && seen[3 * q + 2] == e[2];
        if (dup) continue;
        seen[3 * m] = e[0]; seen[3 * m + 1] = e[1]; seen[3 * m + 2] = e[2];
        m++;
        double hv[3] = {e[0], e[1], e[2]};
        double hh = form_g(f, hv, hv), c = form_g(f, hv, H) / sqrt(hh * HH), c2 = fmin(1, c * c);
        sum += pow(r2 * c2 + (1 - c2) * ir, -1.5);
    }
    return m ? sum / m : 1;
}

/*
 * chi^2 of the full parameter vector v.  ycalc (may be NULL) receives the
 * calculated pattern; nRefl (may be NULL) the reflection count used.
 */
int p6o_solve_spd(const double *A, const double *b, int n, double *x);

/* Lawson-Hanson active-set NNLS on the normal equations: minimise
 * 1/2 x^T H x - rhs^T x subject to x >= 0 (H symmetric positive semi-definite,
 * m x m, row-major).  It is the exact solution the free-intensity fit of
 * js/pt_gpu.js:259-297 (coordinate descent, then an active-set polish)
 * converges to.  Returns the number of outer iterations, -1 if a passive
 * block could not be factored. */
int p6o_nnls_normal(const double *H, const double *rhs, int m, double *x)
{
    int *passive = calloc(m + 1, sizeof(int)), *blocked = calloc(m + 1, sizeof(int)), *idx = malloc(sizeof(int) * (m + 1));
    double *z = malloc(sizeof(double) * (m + 1)), *Hp = malloc(sizeof(double) * (m * m + 1)),
           *bp = malloc(sizeof(double) * (m + 1)), *zp = malloc(sizeof(double) * (m + 1));
    double mag = 1.0;
    for (int j = 0; j < m; j++) { x[j] = 0.0; mag = fmax(mag, fabs(rhs[j])); }
    const double tol = 1e-12 * mag;
    int outer = 0, status = 0;
    for (; outer < 3 * m + 10; outer++) {
        int enter = -1;
        double best = tol;
        for (int j = 0; j < m; j++) {
            double g = rhs[j];
            for (int k = 0; k < m; k++) g -= H[j * m + k] * x[k];
            if (!passive[j] && !blocked[j] && g > best) { best = g; enter = j; }
        }
        if (enter < 0) break;
        passive[enter] = 1;
        for (int inner = 0; inner < 3 * m + 10; inner++) {
            int np = 0;
            for (int j = 0; j < m; j++)
                if (passive[j]) idx[np++] = j;
            for (int a = 0; a < np; a++) {
                bp[a] = rhs[idx[a]];
                for (int b = 0; b < np; b++) Hp[a * np + b] = H[idx[a] * m + idx[b]];
            }
            if (!p6o_solve_spd(Hp, bp, np, zp)) { status = -1; break; }
            for (int j = 0; j < m; j++) z[j] = 0.0;
            int allpos = 1;
            for (int a = 0; a < np; a++) { z[idx[a]] = zp[a]; if (!(zp[a] > 0)) allpos = 0; }
            if (allpos) { for (int j = 0; j < m; j++) x[j] = z[j]; break; }
            double alpha = INFINITY;
            int hit = -1;
            for (int a = 0; a < np; a++) {
                const int j = idx[a];
                if (z[j] <= 0) {
                    const double t = x[j] / (x[j] - z[j]);
                    if (t < alpha) { alpha = t; hit = j; }
                }
            }
            for (int a = 0; a < np; a++) { const int j = idx[a]; x[j] += alpha * (z[j] - x[j]); }
            x[hit] = 0.0;
            for (int a = 0; a < np; a++) { const int j = idx[a]; if (x[j] <= 0) { x[j] = 0.0; passive[j] = 0; } }
        }
        if (status < 0) break;
        /* an entering column that could not stay positive is not offered again until x moves */
        if (!passive[enter]) blocked[enter] = 1;
        else for (int j = 0; j < m; j++) blocked[j] = 0;
    }
    free(passive); free(blocked); free(idx); free(z); free(Hp); free(bp); free(zp);
    return status < 0 ? -1 : outer;
}

static double chebyshev_background(const p6o_pt_problem *P, const double *v, int i)
{
    const int n = P->n;
    double lo = P->tth[0], hi = P->tth[n - 1];
    double x = hi > lo ? 2 * (P->tth[i] - lo) / (hi - lo) - 1 : 0;
    double Tm2 = 1, Tm1 = x, bk = 0;
    for (int kk = 0; kk < P->nBkg; kk++) {
        double T = kk == 0 ? 1 : kk == 1 ? x : 2 * x * Tm1 - Tm2;
        if (kk >= 2) { Tm2 = Tm1; Tm1 = T; }
        double b = v[PT_BKG0 + kk];
        if (b) bk += b * T;
    }
    return bk;
}

double p6o_pt_cost(const p6o_pt_problem *P, const double *v, double *ycalc, int *nReflOut)
{
    const int n = P->n;
    double c6[6] = {v[PT_A], v[PT_B], v[PT_C], v[PT_AL], v[PT_BE], v[PT_GA]};
    int okc;
    inv_dsq_cell(c6, 1, 0, 0, &okc);
    if (!okc) return INFINITY;
    double dmin = P->dmin;
    if (!(dmin > 0)) {
        double lambda = P->lambda1;
        if (P->ratio > 1e-6 && P->lambda2 > 0) lambda = fmin(lambda, P->lambda2);
        double margin = WIN_MAX + fabs(v[PT_ZERO]) +
                        (P->hasShift ? (fabs(v[SIDX(P)]) * 0.001 + fabs(v[SIDX(P) + 1])) * R2D : 0.0);
        double upper = fmin(179.999999, P->tth[n - 1] + margin + .001);
        dmin = lambda / (2 * sin(upper * DEG2RAD / 2));
    }
    int cap = 200000;
    int *h = malloc(sizeof(int) * cap), *k = malloc(sizeof(int) * cap), *l = malloc(sizeof(int) * cap),
        *m = malloc(sizeof(int) * cap);
    double *d0 = malloc(sizeof(double) * cap);
    int nr = p6o_generate_reflections(c6, P->rot, P->trans, P->nOps, dmin, NULL, h, k, l, m, d0, cap);
    if (nr > cap) nr = cap;
    if (nReflOut) *nReflOut = nr;
    double *tthR = malloc(sizeof(double) * (nr + 1)), *F2 = malloc(sizeof(double) * (nr + 1));
    voigt_t *p1 = malloc(sizeof(voigt_t) * (nr + 1)), *p2 = malloc(sizeof(voigt_t) * (nr + 1));
    int *st1 = malloc(sizeof(int) * (nr + 1) * 4);
    double *w2 = malloc(sizeof(double) * (nr + 1));
    int *has1 = calloc(nr + 1, sizeof(int)), *has2 = calloc(nr + 1, sizeof(int));
    const double lam = P->lambda1;
    const int doublet = P->ratio > 1e-6 && P->lambda2 > 1e-6 && fabs(P->lambda1 - P->lambda2) > 1e-6;
    /* geometry and structure */
    for (int r = 0; r < nr; r++) {
        int okq;
        double q = inv_dsq_cell(c6, h[r], k[r], l[r], &okq), s = sqrt(q), sinT = lam * s / 2, tth = NAN;
        if (q > 0 && sinT < 1) tth = 2 * asin(sinT) * R2D;
        tthR[r] = tth;
        double Ar = 0, Br = 0, s2 = s * s;
        if (isfinite(tth)) {
            for (int j = 0; j < P->nAtoms; j++) {
                double dw = exp(-v[PT_BISO] * s2 / 4);
                const double *a = P->ffA + 5 * j, *b = P->ffB + 5 * j;
                double qq = (s / 2) * (s / 2), f0 = P->ffC[j];
                for (int i = 0; i < 5; i++) f0 += a[i] * exp(-b[i] * qq);
                double wj = P->occ[j] * f0 * dw * P->wMult[j], c = 0, sn = 0;
                const double *pos = P->pos + 3 * j;
                for (int qn = 0; qn < P->nReps; qn++) {
                    const int *R = P->repRot + 9 * qn;
                    const double *t = P->repTrans + 3 * qn;
                    double H0 = h[r] * R[0] + k[r] * R[3] + l[r] * R[6], H1 = h[r] * R[1] + k[r] * R[4] + l[r] * R[7],
                           H2 = h[r] * R[2] + k[r] * R[5] + l[r] * R[8];
                    double ph = 2 * PI_ * (H0 * pos[0] + H1 * pos[1] + H2 * pos[2] + h[r] * t[0] + k[r] * t[1] + l[r] * t[2]);
                    c += cos(ph);
                    sn += sin(ph);
                }
                Ar += wj * c;
                Br += wj * sn;
            }
        }
        F2[r] = Ar * Ar + Br * Br;
        if (P->hasPo && isfinite(tth)) F2[r] *= p6o_po_factor(P, c6, v[PT_BKG0 + P->nBkg], h[r], k[r], l[r]);
    }
    /* contributions: all K-alpha-1, then all K-alpha-2 */
    for (int r = 0; r < nr; r++) {
        double bragg = tthR[r];
        if (!(isfinite(bragg) && bragg > 0 && bragg < 180)) continue;
        double base = bragg + sample_shift(P, v, bragg) + v[PT_ZERO];
        prepare_tch_asym(base, base, v, P->minFwhm, AIDX(P), &p1[r]);
        double lo = base - p1[r].maxd, hi = base + p1[r].maxd;
        int start = lower_bound(P->tth, n, lo), stop = start;
        if (start >= n) continue;
        while (stop < n && P->tth[stop] <= hi) stop++;
        if (stop <= start) continue;
        has1[r] = 1;
        st1[4 * r] = start;
        st1[4 * r + 1] = stop;
    }
    if (doublet) {
        for (int r = 0; r < nr; r++) {
            double bragg = tthR[r];
            if (!(isfinite(bragg) && bragg > 0 && bragg < 180)) continue;
            double sin2 = sin(bragg * DEG2RAD / 2.0) * (P->lambda2 / P->lambda1);
            if (fabs(sin2) >= 1) continue;
            double tth2 = 2 * asin(sin2) / DEG2RAD;
            double base2 = tth2 + sample_shift(P, v, tth2) + v[PT_ZERO];
            prepare_tch_asym(base2, base2, v, P->minFwhm, AIDX(P), &p2[r]);
            /* prep1 of this reflection (built in the first pass even if its window missed the axis) */
            voigt_t ref1;
            const double base1 = bragg + sample_shift(P, v, bragg) + v[PT_ZERO];
            prepare_tch_asym(base1, base1, v, P->minFwhm, AIDX(P), &ref1);
            double lpr = lp_factor(base2, P->polK) / lp_factor(ref1.x0, P->polK);
            w2[r] = P->ratio * ref1.area / p2[r].area * lpr;
            double lo = base2 - p2[r].maxd, hi = base2 + p2[r].maxd;
            int start = lower_bound(P->tth, n, lo), stop = start;
            if (start >= n) continue;
            while (stop < n && P->tth[stop] <= hi) stop++;
            if (stop <= start) continue;
            has2[r] = 1;
            st1[4 * r + 2] = start;
            st1[4 * r + 3] = stop;
        }
    }
    /* heights and the pattern (evalPhase + render): column = Ka1 + w2 Ka2 */
    double *y = calloc(n, sizeof(double));
    double *col = malloc(sizeof(double) * n);
    /* WPPF / Le Bail: the columns are kept, with their windows, for the NNLS */
    int nFree = 0, capFree = 0;
    double *fcol = NULL;
    int *fwin = NULL;
    if (P->method == 1) {
        for (int r = 0; r < nr; r++) capFree += (has1[r] || has2[r]) ? 1 : 0;
        fcol = calloc((size_t)(capFree + 1) * n, sizeof(double));
        fwin = malloc(sizeof(int) * 2 * (capFree + 1));
    }
    for (int r = 0; r < nr; r++) {
        if (!has1[r] && !has2[r]) continue;
        if (!isfinite(tthR[r])) continue;
        double tc = tthR[r] + sample_shift(P, v, tthR[r]) + v[PT_ZERO];
        voigt_t ref1;
        prepare_tch_asym(tc, tc, v, P->minFwhm, AIDX(P), &ref1);
        double K = ref1.area;
        if (!(K > 0)) continue;
        double lp = lp_factor(tc, P->polK);
        double factor = m[r] * lp * 1.0 / K;          /* height per unit S |F|^2 */
        double height = v[PT_SCALE] * (factor * F2[r]);
        int s0 = n, s1 = 0;
        if (has1[r]) { if (st1[4 * r] < s0) s0 = st1[4 * r]; if (st1[4 * r + 1] > s1) s1 = st1[4 * r + 1]; }
        if (has2[r]) { if (st1[4 * r + 2] < s0) s0 = st1[4 * r + 2]; if (st1[4 * r + 3] > s1) s1 = st1[4 * r + 3]; }
        for (int i = s0; i < s1; i++) col[i] = 0;
        if (has1[r])
            for (int i = st1[4 * r]; i < st1[4 * r + 1]; i++) col[i] += 1.0 * eval_voigt(P->tth[i], &p1[r], p1[r].maxd, p1[r].pedestal);
        if (has2[r])
            for (int i = st1[4 * r + 2]; i < st1[4 * r + 3]; i++)
                col[i] += w2[r] * eval_voigt(P->tth[i], &p2[r], p2[r].maxd, p2[r].pedestal);
        if (P->method == 1) {
            for (int i = s0; i < s1; i++) fcol[(size_t)nFree * n + i] = col[i];
            fwin[2 * nFree] = s0;
            fwin[2 * nFree + 1] = s1;
            nFree++;
            continue;
        }
        if (!height) continue;
        for (int i = s0; i < s1; i++) y[i] += height * col[i];
    }
    if (P->method == 1 && nFree > 0) {
        /* scaled normal equations: s_j = |W^1/2 c_j|, H = (C S^-1)^T W (C S^-1), rhs = (C S^-1)^T W (y - bkg) */
        double *sc = calloc(nFree, sizeof(double)), *rhs = calloc(nFree, sizeof(double)),
               *H = calloc((size_t)nFree * nFree, sizeof(double)), *x = calloc(nFree, sizeof(double));
        for (int j = 0; j < nFree; j++) {
            double a = 0, b = 0;
            for (int i = fwin[2 * j]; i < fwin[2 * j + 1]; i++) {
                if (!(P->w[i] > 0)) continue;
                const double c = fcol[(size_t)j * n + i];
                a += P->w[i] * c * c;
                b += P->w[i] * c * (P->y[i] - chebyshev_background(P, v, i));
            }
            sc[j] = sqrt(fmax(0.0, a));
            rhs[j] = sc[j] > 0 ? b / sc[j] : 0.0;
        }
        for (int j = 0; j < nFree; j++)
            for (int k = j; k < nFree; k++) {
                double h = 0;
                if (sc[j] > 0 && sc[k] > 0) {
                    const int lo = fwin[2 * j] > fwin[2 * k] ? fwin[2 * j] : fwin[2 * k];
                    const int hi = fwin[2 * j + 1] < fwin[2 * k + 1] ? fwin[2 * j + 1] : fwin[2 * k + 1];
                    for (int i = lo; i < hi; i++)
                        if (P->w[i] > 0) h += P->w[i] * fcol[(size_t)j * n + i] * fcol[(size_t)k * n + i];
                    h /= sc[j] * sc[k];
                }
                H[j * nFree + k] = H[k * nFree + j] = h;
            }
        /* a column with no weighted points stays at zero height */
        for (int j = 0; j < nFree; j++)
            if (!(sc[j] > 0)) H[j * nFree + j] = 1.0;
        p6o_nnls_normal(H, rhs, nFree, x);
        for (int j = 0; j < nFree; j++) {
            const double height = sc[j] > 0 ? x[j] / sc[j] : 0.0;
            if (!height) continue;
            for (int i = fwin[2 * j]; i < fwin[2 * j + 1]; i++) y[i] += height * fcol[(size_t)j * n + i];
        }
        free(sc); free(rhs); free(H); free(x);
    }
    free(fcol); free(fwin);
    /* background (Chebyshev over the fitted range) and chi^2 */
    double chi2 = 0;
    for (int i = 0; i < n; i++) {
        double yc = chebyshev_background(P, v, i) + y[i];
        if (ycalc) ycalc[i] = yc;
        if (!(P->w[i] > 0)) continue;
        double res = P->y[i] - yc;
        chi2 += P->w[i] * res * res;
    }
    free(h); free(k); free(l); free(m); free(d0); free(tthR); free(F2); free(p1); free(p2); free(st1); free(w2);
    free(has1); free(has2); free(y); free(col);
    return chi2;
}

/* ------------------------------------------------------------------------ */
/* CPU parallel tempering (temper), refined parameters mapped into v.        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nv;
    const int *index;     /* refined parameter j -> full vector index */
    const double *lo, *hi, *scales;
    int cubic;            /* b = c = a, angles fixed */
    int chains, sweeps;
    double maxTemp;
    uint32_t seed;
} p6o_pt_setup;

static void apply_params(const p6o_pt_problem *P, const p6o_pt_setup *S, const double *base, const double *x,
                         double *v, int nFull)
{
    (void)P;
    memcpy(v, base, sizeof(double) * nFull);
    for (int j = 0; j < S->nv; j++) v[S->index[j]] = x[j];
    if (S->cubic) { v[PT_B] = v[PT_A]; v[PT_C] = v[PT_A]; }
}

static double reflect(double value, double low, double high)
{
    if (!isfinite(value)) return NAN;
    if (isfinite(low) && isfinite(high)) {
        double span = high - low;
        if (!(span > 0)) return low;
        double folded = fmod(fmod(value - low, 2 * span) + 2 * span, 2 * span);
        return low + (folded <= span ? folded : 2 * span - folded);
    }
    if (value < low) return low + (low - value);
    if (value > high) return high - (value - high);
    return value;
}

/* temper's random(): xorshift32, (state + 0.5) / 2^32 (rietveld_core.js:2174-2177) */
static double xorshift_uniform(uint32_t *s)
{
    *s ^= *s << 13;
    *s ^= *s >> 17;
    *s ^= *s << 5;
    return ((double)*s + 0.5) / 4294967296.0;
}

/*
 * Runs temper() from x0 (nv refined values).  best (nv) receives the best
 * vector; stats: proposals, accepted, swapAttempts, swaps, bestCost,
 * initialCost.  maxSweeps < sweeps stops early (bounded samples).
 */
double p6o_pt_temper(const p6o_pt_problem *P, const p6o_pt_setup *S, const double *baseFull, int nFull,
                     const double *x0, double *best, double *stats, int maxSweeps)
{
    uint32_t rs = S->seed;
#define RND() xorshift_uniform(&rs)
    const int nv = S->nv, C = S->chains;
    double *v = malloc(sizeof(double) * nFull);
    double *X = malloc(sizeof(double) * nv * C), *cost = malloc(sizeof(double) * C), *T = malloc(sizeof(double) * C);
    double *prop = malloc(sizeof(double) * nv);
    int *order = malloc(sizeof(int) * C);
    apply_params(P, S, baseFull, x0, v, nFull);
    double initial = p6o_pt_cost(P, v, NULL, NULL), bestCost = initial;
    memcpy(best, x0, sizeof(double) * nv);
    for (int r = 0; r < C; r++) {
        T[r] = pow(S->maxTemp, (double)r / (C - 1));
        memcpy(X + r * nv, x0, sizeof(double) * nv);
        cost[r] = initial;
        order[r] = r;
    }
    double proposals = 0, accepted = 0, attempts = 0, swaps = 0;
    int sweeps = maxSweeps > 0 && maxSweeps < S->sweeps ? maxSweeps : S->sweeps;
    for (int sweep = 0; sweep < sweeps; sweep++) {
        for (int r = 0; r < C; r++) {
            int slot = order[r];
            double *x = X + slot * nv;
            for (int move = 0; move < nv; move++) {
                int coord = (int)floor(RND() * nv);
                memcpy(prop, x, sizeof(double) * nv);
                double u1 = RND();                 /* JavaScript evaluates left to right */
                double u2 = RND();
                double g = sqrt(-2 * log(u1)) * cos(2 * PI_ * u2);
                prop[coord] = reflect(prop[coord] + g * S->scales[coord] * sqrt(T[r]), S->lo[coord], S->hi[coord]);
                if (!isfinite(prop[coord])) continue;
                apply_params(P, S, baseFull, prop, v, nFull);
                double c = p6o_pt_cost(P, v, NULL, NULL);
                proposals++;
                if (isfinite(c) && (c <= cost[slot] || log(RND()) < (cost[slot] - c) / (2 * T[r]))) {
                    memcpy(x, prop, sizeof(double) * nv);
                    cost[slot] = c;
                    accepted++;
                    if (c < bestCost) { bestCost = c; memcpy(best, prop, sizeof(double) * nv); }
                }
            }
        }
        for (int r = sweep % 2; r < C - 1; r += 2) {
            int a = order[r], b = order[r + 1];
            double la = 0.5 * (1 / T[r] - 1 / T[r + 1]) * (cost[a] - cost[b]);
            attempts++;
            if (la >= 0 || log(RND()) < la) { order[r] = b; order[r + 1] = a; swaps++; }
        }
    }
#undef RND
    stats[0] = proposals; stats[1] = accepted; stats[2] = attempts; stats[3] = swaps;
    stats[4] = bestCost; stats[5] = initial;
    free(v); free(X); free(cost); free(T); free(prop); free(order);
    return bestCost;
}

/* Test hooks: closed forms of the profile model. */
double p6o_lp(double tth, double K) { return lp_factor(tth, K); }
double p6o_peak_fwhm(double gG, double gL) { return peak_fwhm(gG, gL); }
double p6o_soft_positive(double x, double f) { return soft_positive(x, f); }
double p6o_soft_floor(double x, double f) { return soft_floor(x, f); }
/* prepareVoigt (TCH) of the widths in v at tthPeak: out = x0, 1/fwhm, cL, cG, pedestal, maxd, area */
void p6o_prepare_tch(const double *v, double minFwhm, double tthPeak, double *out)
{
    voigt_t p;
    prepare_tch(tthPeak, tthPeak, v, minFwhm, &p);
    out[0] = p.x0; out[1] = p.inv; out[2] = p.cL; out[3] = p.cG; out[4] = p.pedestal; out[5] = p.maxd; out[6] = p.area;
}
/* prepareVoigt with SL, HL: out = x0, inv, cL, cG, pedestal, maxd, area (with the asymmetry's correction), asym */
void p6o_prepare_tch_asym(const double *v, double minFwhm, double tthPeak, double SL, double HL, double *out)
{
    double vv[16];
    memcpy(vv, v, sizeof(double) * 14);
    vv[14] = SL;
    vv[15] = HL;
    voigt_t p;
    prepare_tch_asym(tthPeak, tthPeak, vv, minFwhm, 14, &p);
    out[0] = p.x0; out[1] = p.inv; out[2] = p.cL; out[3] = p.cG; out[4] = p.pedestal; out[5] = p.maxd; out[6] = p.area;
    out[7] = p.asym;
}
/* evalVoigt without truncation or pedestal, for area checks */
double p6o_voigt_raw(double delta, double inv, double cL, double cG)
{
    voigt_t p = {0, inv, cL, cG, 0, INFINITY, 0};
    return eval_voigt(delta, &p, INFINITY, 0.0);
}

/* ------------------------------------------------------------------------ */
/* Least-squares finish: normal equations and Levenberg-Marquardt            */
/* (js/rietveld_core.js:1953-2140), finite-difference steps and limits       */
/* (fdStep :526-538, defaultLimits :486-508, stepCap :511-524), Cholesky and */
/* solveSPD (:1304-1335).  Parameters are identified by their full index.    */
/* ------------------------------------------------------------------------ */
enum { K_SCALE, K_CELL, K_ANGLE, K_PROFILE, K_LORENTZ, K_ZERO, K_BISO, K_BKG, K_PO, K_SL, K_HL, K_DISP, K_TRANSP };

static int kind_of(const p6o_pt_problem *P, int fi)
{
    if (P->hasPo && fi == PT_BKG0 + P->nBkg) return K_PO;
    if (P->hasShift && fi == SIDX(P)) return K_DISP;
    if (P->hasShift && fi == SIDX(P) + 1) return K_TRANSP;
    if (P->hasAsym && fi == AIDX(P)) return K_SL;
    if (P->hasAsym && fi == AIDX(P) + 1) return K_HL;
    if (fi == PT_SCALE) return K_SCALE;
    if (fi >= PT_A && fi <= PT_C) return K_CELL;
    if (fi >= PT_AL && fi <= PT_GA) return K_ANGLE;
    if (fi >= PT_U && fi <= PT_W) return K_PROFILE;
    if (fi == PT_X || fi == PT_Y) return K_LORENTZ;
    if (fi == PT_ZERO) return K_ZERO;
    if (fi == PT_BISO) return K_BISO;
    return K_BKG;
}

/* fdStep: cell a, b, c max(1e-6|v|, 1e-6); angles, zero 1e-4; others max(1e-4|v|, 1e-5) */
static double fd_step(int kind, double v)
{
    double a = fabs(v);
    switch (kind) {
    case K_CELL: return fmax(1e-6 * a, 1e-6);
    case K_ANGLE: return 1e-4;
    case K_ZERO: return 1e-4;
    case K_PO: return 1e-4;
    case K_DISP: return 1e-2;
    case K_TRANSP: return 1e-6;
    default: return fmax(1e-4 * a, 1e-5);
    }
}

/* defaultLimits: the physical range a finite-difference probe may use */
static void default_limits(int kind, double v, double *lo, double *hi)
{
    switch (kind) {
    case K_SCALE: *lo = 0; *hi = INFINITY; return;
    case K_CELL: *lo = 0.5 * v; *hi = 2 * v; return;
    case K_ANGLE: *lo = 30; *hi = 150; return;
    case K_BISO: *lo = -2; *hi = 30; return;
    case K_ZERO: *lo = -2; *hi = 2; return;
    case K_LORENTZ: *lo = 0; *hi = INFINITY; return;
    case K_PO: *lo = 0.1; *hi = 5; return;
    case K_SL: *lo = 0; *hi = INFINITY; return;
    default: *lo = -INFINITY; *hi = INFINITY; return;
    }
}

/* stepCap: the largest change of one iteration */
static double step_cap(int kind, double v)
{
    switch (kind) {
    case K_CELL: return 0.02 * fabs(v) + 1e-6;
    case K_ANGLE: return 1;
    case K_BISO: return 2;
    case K_ZERO: return 0.1;
    case K_PO: return 0.25;
    case K_SL: case K_HL: return 0.01;
    case K_DISP: return 2;
    case K_TRANSP: return 0.01;
    case K_PROFILE: case K_LORENTZ: return 0.5 * fmax(fabs(v), 5);
    default: return INFINITY;
    }
}

static int cholesky(const double *A, int n, double *L)
{
    memset(L, 0, sizeof(double) * n * n);
    for (int i = 0; i < n; i++)
        for (int j = 0; j <= i; j++) {
            double s = A[i * n + j];
            for (int k = 0; k < j; k++) s -= L[i * n + k] * L[j * n + k];
            if (i == j) {
                if (!(s > 0) || !isfinite(s)) return 0;
                L[i * n + i] = sqrt(s);
            } else
                L[i * n + j] = s / L[j * n + j];
        }
    return 1;
}

static void chol_solve(const double *L, const double *b, int n, double *x)
{
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int k = 0; k < i; k++) s -= L[i * n + k] * x[k];
        x[i] = s / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = i + 1; k < n; k++) s -= L[k * n + i] * x[k];
        x[i] = s / L[i * n + i];
    }
}

/* solveSPD with the growing ridge; returns 0 when it fails */
int p6o_solve_spd(const double *A, const double *b, int n, double *x)
{
    double *L = malloc(sizeof(double) * n * n), *B = malloc(sizeof(double) * n * n);
    int ok = cholesky(A, n, L);
    if (!ok) {
        double tr = 0;
        for (int i = 0; i < n; i++) tr += fabs(A[i * n + i]);
        double ridge = (tr / (n > 1 ? n : 1)) * 1e-12;
        if (!(ridge > 0 || ridge < 0)) ridge = 1e-300;
        for (int a = 0; a < 10 && !ok; a++, ridge *= 100) {
            memcpy(B, A, sizeof(double) * n * n);
            for (int i = 0; i < n; i++) B[i * n + i] += ridge;
            ok = cholesky(B, n, L);
        }
    }
    if (ok) chol_solve(L, b, n, x);
    free(L); free(B);
    return ok;
}

/* Gaussian-variance minimum of U t^2 + V t + W over t = tan(theta) of the fitted range */
static double variance_minimum(const p6o_pt_problem *P, const double *v)
{
    double t0 = tan(P->tth[0] * DEG2RAD / 2), t1 = tan(P->tth[P->n - 1] * DEG2RAD / 2);
    double U = v[PT_U], V = v[PT_V], W = v[PT_W];
    double m = fmin(U * t0 * t0 + V * t0 + W, U * t1 * t1 + V * t1 + W);
    if (U > 0) {
        double ts = -V / (2 * U);
        if (ts > t0 && ts < t1) m = fmin(m, U * ts * ts + V * ts + W);
    }
    return m;
}
static double violation_of(const p6o_pt_problem *P, const double *v)
{
    double m = variance_minimum(P, v);
    return m < 0 ? -m : 0;
}

/*
 * normal(): A = J'WJ, g = J'W r and f = chi^2 at the refined vector x.
 * Scale and background columns are analytic, the others symmetric finite
 * differences of the phase pattern (one-sided at a physical limit).
 */
int p6o_pt_normal(const p6o_pt_problem *P, const p6o_pt_setup *S, const double *baseFull, int nFull, const double *x,
                  double *A, double *g, double *f)
{
    const int n = P->n, nv = S->nv;
    double *v = malloc(sizeof(double) * nFull), *vp = malloc(sizeof(double) * nFull);
    double *y0 = malloc(sizeof(double) * n), *ya = malloc(sizeof(double) * n), *yb = malloc(sizeof(double) * n);
    double *J = calloc((size_t)nv * n, sizeof(double)), *r = calloc(n, sizeof(double));
    apply_params(P, S, baseFull, x, v, nFull);
    double chi = p6o_pt_cost(P, v, y0, NULL);
    if (!isfinite(chi)) { free(v); free(vp); free(y0); free(ya); free(yb); free(J); free(r); return 0; }
    for (int j = 0; j < nv; j++) {
        const int fi = S->index[j], kind = kind_of(P, fi);
        double *col = J + (size_t)j * n;
        if (kind == K_SCALE) {
            memcpy(vp, v, sizeof(double) * nFull);
            vp[PT_SCALE] = 1;
            p6o_pt_cost(P, vp, ya, NULL);
            vp[PT_SCALE] = 0;
            p6o_pt_cost(P, vp, yb, NULL);
            for (int i = 0; i < n; i++) col[i] = ya[i] - yb[i];
        } else if (kind == K_BKG) {
            const int kk = fi - PT_BKG0;
            double lo = P->tth[0], hi = P->tth[n - 1];
            for (int i = 0; i < n; i++) {
                double z = hi > lo ? 2 * (P->tth[i] - lo) / (hi - lo) - 1 : 0, Tm2 = 1, Tm1 = z, T = 1;
                for (int q = 0; q <= kk; q++) {
                    T = q == 0 ? 1 : q == 1 ? z : 2 * z * Tm1 - Tm2;
                    if (q >= 2) { Tm2 = Tm1; Tm1 = T; }
                }
                col[i] = T;
            }
        } else {
            const double val = x[j], h = fd_step(kind, val);
            double llo, lhi;
            default_limits(kind, val, &llo, &lhi);
            /* the March-Dollase column is a forward difference (js/rietveld_core.js:1271-1275) */
            const int plus = kind == K_PO || val + h <= lhi, minus = kind != K_PO && val - h >= llo;
            double xp[64], xm[64];
            memcpy(xp, x, sizeof(double) * nv);
            memcpy(xm, x, sizeof(double) * nv);
            xp[j] = plus ? val + h : val;
            xm[j] = minus ? val - h : val;
            const double d = xp[j] - xm[j];
            if (d != 0) {
                if (plus) {
                    apply_params(P, S, baseFull, xp, vp, nFull);
                    p6o_pt_cost(P, vp, ya, NULL);
                }
                if (minus) {
                    apply_params(P, S, baseFull, xm, vp, nFull);
                    p6o_pt_cost(P, vp, yb, NULL);
                }
                for (int i = 0; i < n; i++) col[i] = ((plus ? ya[i] : y0[i]) - (minus ? yb[i] : y0[i])) / d;
            }
        }
    }
    double ff = 0;
    for (int i = 0; i < n; i++) {
        if (!(P->w[i] > 0)) continue;
        r[i] = P->y[i] - y0[i];
        ff += P->w[i] * r[i] * r[i];
    }
    for (int a = 0; a < nv; a++) {
        const double *Ja = J + (size_t)a * n;
        double ga = 0;
        for (int i = 0; i < n; i++) ga += P->w[i] * Ja[i] * r[i];
        g[a] = ga;
        for (int b = 0; b <= a; b++) {
            const double *Jb = J + (size_t)b * n;
            double s = 0;
            for (int i = 0; i < n; i++) s += P->w[i] * Ja[i] * Jb[i];
            A[a * nv + b] = s;
            A[b * nv + a] = s;
        }
    }
    *f = ff;
    free(v); free(vp); free(y0); free(ya); free(yb); free(J); free(r);
    return 1;
}

static double cost_at(const p6o_pt_problem *P, const p6o_pt_setup *S, const double *baseFull, int nFull, const double *x)
{
    double v[128];
    apply_params(P, S, baseFull, x, v, nFull);
    return p6o_pt_cost(P, v, NULL, NULL);
}

/*
 * lm() of one stage without constraints: x (nv) in/out, bounds S->lo/hi.
 * out[0] = chi^2, out[1] = iterations tried, out[2] = accepted steps,
 * out[3] = exit code (0 iteration limit, 1 chi^2 change below tol,
 * 2 projected gradient below tolerance, 3 singular, 4 stalled,
 * 5 all parameters at limits, 6 stopped at the variance limit).
 * The variance guard cuts a step that would make U tan^2 + V tan + W
 * negative back to the boundary by bisection (the second of the
 * reference's two remedies; its projection onto the face is not restated).
 */
int p6o_pt_lm(const p6o_pt_problem *P, const p6o_pt_setup *S, const double *baseFull, int nFull, double *x,
              int maxIter, double tol, double *out)
{
    const int nv = S->nv, nPts = P->n;
    double *A = malloc(sizeof(double) * nv * nv), *g = malloc(sizeof(double) * nv);
    double *Mx = malloc(sizeof(double) * nv * nv), *bx = malloc(sizeof(double) * nv), *dx = malloc(sizeof(double) * nv);
    double xn[64], step[64], sc[64], v[128], cand[64];
    int F[64];
    double f = cost_at(P, S, baseFull, nFull, x), mu = 1e-3, nu = 2;
    int conv = 0, have = 0, it, code = 0, accepted = 0;
    if (!(tol > 0)) tol = 1e-5;
    apply_params(P, S, baseFull, x, v, nFull);
    double curViolation = violation_of(P, v);
    for (it = 0; it < maxIter; it++) {
        double fNE;
        if (!have) {
            if (!p6o_pt_normal(P, S, baseFull, nFull, x, A, g, &fNE)) { code = 3; break; }
            have = 1;
        }
        int nF = 0;
        for (int j = 0; j < nv; j++) {
            const double lo = S->lo[j], hi = S->hi[j];
            const int atLo = x[j] <= lo + 1e-12 * (1 + fabs(lo)), atHi = x[j] >= hi - 1e-12 * (1 + fabs(hi));
            if (!((atLo && g[j] < 0) || (atHi && g[j] > 0)) && A[j * nv + j] > 0) F[nF++] = j;
        }
        if (!nF) { code = 5; break; }
        double grad = 0, noise = sqrt(fmax(f / fmax(1, nPts - nv), 1e-30));
        for (int a = 0; a < nF; a++) {
            sc[a] = 1 / sqrt(A[F[a] * nv + F[a]]);
            grad = fmax(grad, fabs(g[F[a]]) * sc[a] / noise);
        }
        if (f < 1e-24 || grad < 1e-4) { code = 2; break; }
        for (int a = 0; a < nF; a++) {
            bx[a] = g[F[a]] * sc[a];
            for (int b = 0; b < nF; b++) Mx[a * nF + b] = A[F[a] * nv + F[b]] * sc[a] * sc[b];
            Mx[a * nF + a] += mu;
        }
        if (!p6o_solve_spd(Mx, bx, nF, dx)) {
            mu *= nu; nu *= 2;
            if (mu > 1e30) { code = 3; break; }
            continue;
        }
        memcpy(xn, x, sizeof(double) * nv);
        memset(step, 0, sizeof(double) * nv);
        for (int a = 0; a < nF; a++) {
            const int q = F[a];
            const double cap = step_cap(kind_of(P, S->index[q]), x[q]);
            const double sh = fmax(-cap, fmin(cap, dx[a] * sc[a]));
            xn[q] = fmin(S->hi[q], fmax(S->lo[q], x[q] + sh));
            step[q] = xn[q] - x[q];
        }
        apply_params(P, S, baseFull, xn, v, nFull);
        double violation = violation_of(P, v);
        int blocked = 0;
        if (curViolation == 0 && violation > 0) {
            double loA = 0, hiA = 1;
            for (int bi = 0; bi < 24; bi++) {
                double mid = 0.5 * (loA + hiA);
                for (int a = 0; a < nv; a++) cand[a] = x[a] + mid * step[a];
                apply_params(P, S, baseFull, cand, v, nFull);
                if (violation_of(P, v) == 0) loA = mid; else hiA = mid;
            }
            for (int a = 0; a < nv; a++) { xn[a] = x[a] + loA * step[a]; step[a] = xn[a] - x[a]; }
            apply_params(P, S, baseFull, xn, v, nFull);
            violation = violation_of(P, v);
            blocked = 1;
        }
        double pred = 0, sAs = 0;
        for (int a = 0; a < nv; a++) {
            if (!step[a]) continue;
            pred += 2 * g[a] * step[a];
            double tt = 0;
            for (int b = 0; b < nv; b++) tt += A[a * nv + b] * step[b];
            sAs += step[a] * tt;
        }
        pred -= sAs;
        const double fn = p6o_pt_cost(P, v, NULL, NULL);
        if (fn < f) {
            const double rho = pred > 0 ? (f - fn) / pred : 0.5, rel = (f - fn) / f;
            int small = 1;
            const double s2 = fmax(f, 1e-30) / fmax(1, nPts - nv);
            for (int a = 0; a < nF; a++) {
                const int q = F[a];
                if (fabs(step[q]) * sqrt(A[q * nv + q] / s2) > 0.1) { small = 0; break; }
            }
            memcpy(x, xn, sizeof(double) * nv);
            f = fn;
            have = 0;
            curViolation = violation;
            mu *= fmax(1.0 / 3, 1 - pow(2 * rho - 1, 3));
            nu = 2;
            accepted++;
            if (!blocked && rel < tol && small) {
                if (++conv >= 2) { code = 1; it++; break; }
            } else
                conv = 0;
        } else {
            mu *= nu; nu *= 2;
            if (mu > 1e20) { code = blocked ? 6 : (grad < 1e-3 ? 2 : 4); break; }
        }
    }
    out[0] = f; out[1] = it; out[2] = accepted; out[3] = code;
    free(A); free(g); free(Mx); free(bx); free(dx);
    return 1;
}
