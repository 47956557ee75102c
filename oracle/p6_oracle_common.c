/*
 * ORACLE -- test infrastructure, not product code.
 *
 *   p6o_generate_reflections  js/rietveld_core.js:247-276 (generateReflections)
 *                             with buildInvDsq/invDsq (js/crystal.js:326-377),
 *                             laueRotations (:182-188) and isAllowed (:192-201):
 *                             unique reflections to dmin, canonical Laue-orbit
 *                             member, exact absences, multiplicity, sorted by d
 *                             descending then h, k, l descending.
 *   p6o_philox                Philox4x32-10 (Salmon et al., SC'11), restated from
 *                             the published round function, for known-answer
 *                             checks of the device generator.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEG2RAD (3.14159265358979323846 / 180.0)

typedef struct {
    double aa, bb, cc, ab, bc, ac;
} inv_dsq_form;

static int build_inv_dsq(const double *cell, inv_dsq_form *f)
{
    double a = cell[0], b = cell[1] > 0 ? cell[1] : a, c = cell[2] > 0 ? cell[2] : a;
    if (!(a > 0) || !(b > 0) || !(c > 0)) return 0;
    double al = cell[3] * DEG2RAD, be = cell[4] * DEG2RAD, ga = cell[5] * DEG2RAD;
    double cosA = cos(al), cosB = cos(be), cosG = cos(ga), sinA = sin(al), sinB = sin(be), sinG = sin(ga);
    double vf = 1 - cosA * cosA - cosB * cosB - cosG * cosG + 2 * cosA * cosB * cosG;
    if (vf <= 1e-9 || fabs(sinA) < 1e-9 || fabs(sinB) < 1e-9 || fabs(sinG) < 1e-9) return 0;
    double V = a * b * c * sqrt(vf);
    double as = b * c * sinA / V, bs = a * c * sinB / V, cs = a * b * sinG / V;
    double cosAs = (cosB * cosG - cosA) / (sinB * sinG);
    double cosBs = (cosA * cosG - cosB) / (sinA * sinG);
    double cosGs = (cosA * cosB - cosG) / (sinA * sinB);
    f->aa = as * as;
    f->bb = bs * bs;
    f->cc = cs * cs;
    f->ab = 2 * as * bs * cosGs;
    f->bc = 2 * bs * cs * cosAs;
    f->ac = 2 * as * cs * cosBs;
    return 1;
}

static double inv_dsq(const inv_dsq_form *f, double h, double k, double l)
{
    return h * h * f->aa + k * k * f->bb + l * l * f->cc + h * k * f->ab + k * l * f->bc + h * l * f->ac;
}

typedef struct {
    int h, k, l, m;
    double d0;
} refl_t;

static int cmp_refl(const void *pa, const void *pb)
{
    const refl_t *a = (const refl_t *)pa, *b = (const refl_t *)pb;
    if (b->d0 != a->d0) return b->d0 > a->d0 ? 1 : -1;
    if (b->h != a->h) return b->h - a->h;
    if (b->k != a->k) return b->k - a->k;
    return b->l - a->l;
}

/*
 * cell: a, b, c, alpha, beta, gamma.  rot: nOps*9 ints, trans: nOps*3 doubles.
 * box: NULL, or {hmax, kmax, lmax} (then the metric cutoff is not applied).
 * Outputs at most maxOut rows; returns the total count (may exceed maxOut).
 */
int p6o_generate_reflections(const double *cell, const int *rot, const double *trans, int nOps, double dmin,
                             const int *box, int *oh, int *ok, int *ol, int *om, double *od0, int maxOut)
{
    inv_dsq_form f;
    if (!build_inv_dsq(cell, &f) || !(dmin > 0)) return 0;
    double lim = 1.0 / (dmin * dmin) * (1 + 1e-9);
    /* Laue rotations: R and -R, deduplicated */
    int *rots = (int *)malloc(sizeof(int) * 9 * 2 * (nOps > 0 ? nOps : 1));
    int nr = 0;
    for (int o = 0; o < nOps; o++)
        for (int sgn = 1; sgn >= -1; sgn -= 2) {
            int r[9];
            for (int i = 0; i < 9; i++) r[i] = sgn * rot[o * 9 + i];
            int dup = 0;
            for (int q = 0; q < nr && !dup; q++) dup = memcmp(rots + q * 9, r, sizeof(r)) == 0;
            if (!dup) memcpy(rots + (nr++) * 9, r, sizeof(r));
        }
    int hmax = box ? box[0] : (int)floor(cell[0] / dmin);
    int kmax = box ? box[1] : (int)floor((cell[1] > 0 ? cell[1] : cell[0]) / dmin);
    int lmax = box ? box[2] : (int)floor((cell[2] > 0 ? cell[2] : cell[0]) / dmin);
    size_t cap = 1024, n = 0;
    refl_t *out = (refl_t *)malloc(sizeof(refl_t) * cap);
    int *orbit = (int *)malloc(sizeof(int) * 3 * nr);
    for (int h = -hmax; h <= hmax; h++)
        for (int k = -kmax; k <= kmax; k++)
            for (int l = -lmax; l <= lmax; l++) {
                if (!h && !k && !l) continue;
                double q = inv_dsq(&f, h, k, l);
                if (!(q > 0) || (!box && q > lim)) continue;
                int ch = -1000000000, ck = 0, cl = 0, cp = -1, no = 0;
                for (int i = 0; i < nr; i++) {
                    const int *r = rots + i * 9;
                    int v0 = h * r[0] + k * r[3] + l * r[6];
                    int v1 = h * r[1] + k * r[4] + l * r[7];
                    int v2 = h * r[2] + k * r[5] + l * r[8];
                    int np_ = (v0 >= 0) + (v1 >= 0) + (v2 >= 0);
                    int dup = 0;
                    for (int j = 0; j < no && !dup; j++)
                        dup = orbit[3 * j] == v0 && orbit[3 * j + 1] == v1 && orbit[3 * j + 2] == v2;
                    if (!dup) { orbit[3 * no] = v0; orbit[3 * no + 1] = v1; orbit[3 * no + 2] = v2; no++; }
                    if (np_ > cp || (np_ == cp && (v0 > ch || (v0 == ch && (v1 > ck || (v1 == ck && v2 > cl)))))) {
                        cp = np_; ch = v0; ck = v1; cl = v2;
                    }
                }
                if (ch != h || ck != k || cl != l) continue;
                int allowed = 1;
                for (int o = 0; o < nOps && allowed; o++) {
                    const int *r = rot + o * 9;
                    if (h * r[0] + k * r[3] + l * r[6] != h || h * r[1] + k * r[4] + l * r[7] != k ||
                        h * r[2] + k * r[5] + l * r[8] != l)
                        continue;
                    double p = h * trans[o * 3] + k * trans[o * 3 + 1] + l * trans[o * 3 + 2];
                    if (fabs(p - round(p)) > 1e-6) allowed = 0;
                }
                if (!allowed) continue;
                if (n == cap) { cap *= 2; out = (refl_t *)realloc(out, sizeof(refl_t) * cap); }
                out[n].h = h; out[n].k = k; out[n].l = l; out[n].m = no; out[n].d0 = 1 / sqrt(q);
                n++;
            }
    qsort(out, n, sizeof(refl_t), cmp_refl);
    for (size_t i = 0; i < n && (int)i < maxOut; i++) {
        oh[i] = out[i].h; ok[i] = out[i].k; ol[i] = out[i].l; om[i] = out[i].m; od0[i] = out[i].d0;
    }
    free(out);
    free(orbit);
    free(rots);
    return (int)n;
}

void p6o_philox(const uint32_t *ctr_in, const uint32_t *key_in, uint32_t *out)
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int i = 0; i < 10; i++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
