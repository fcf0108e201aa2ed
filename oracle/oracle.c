/*
 * oracle.c -- CPU restatement of the reference's direct-SCF Fock-build path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file;
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * use it as the reference to compare against.  Each function cites the reference file:line it
 * restates (paths relative to the reference project root).
 *
 * Parity pins (tests/test_oracle.py):
 *   - Boys table + Taylor + asymptotic branch against values produced by the
 *     reference's own src/lookup/boys.cpp compiled unmodified
 *     (tests/golden/boys_ref.json, built by oracle/build_ref.sh);
 *   - converged RHF energies of the reference's regression cases
 *     (tests/golden/regression_cases.json, from tests/regression_cases.json).
 * The Rys roots use the reference's long-double Stieltjes moment construction
 * (src/integrals/rys_roots.cpp:88-235); Eigen's SelfAdjointEigenSolver is
 * replaced by the implicit-shift QL algorithm for symmetric tridiagonal
 * matrices (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math. 11 (1968);
 * the EISPACK tql2 procedure), which agrees with it to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_L 3
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Boys function: src/lookup/boys.cpp:7-15 (table layout), :1592-1618.       */
/* The reference table holds F_n(0.1 k) rounded to 15 decimals, 1571 rows,   */
/* n = 0..65.  The oracle regenerates it from the defining series in long    */
/* double and rounds each value to 15 decimals the same way a literal does.  */
/* ------------------------------------------------------------------------ */
#define BOYS_COLS 66
#define BOYS_ROWS 1571
#define BOYS_STEP 0.1
static double g_boys[BOYS_ROWS][BOYS_COLS];
static int g_boys_ready = 0;

static long double boys_series(int n, long double x)
{
    /* F_n(x) = exp(-x) * sum_k (2x)^k / ((2n+1)(2n+3)...(2n+2k+1)) */
    long double term = 1.0L / (2 * n + 1);
    long double sum = term;
    for (int k = 1; k < 4000; ++k) {
        term *= 2.0L * x / (2 * n + 2 * k + 1);
        sum += term;
        if (term < 1e-24L * sum)
            break;
    }
    return expl(-x) * sum;
}

void orc_boys_init(void)
{
    if (g_boys_ready)
        return;
    char buf[64];
    for (int r = 0; r < BOYS_ROWS; ++r) {
        long double x = (long double)r / 10.0L;
        for (int n = 0; n < BOYS_COLS; ++n) {
            snprintf(buf, sizeof buf, "%.15f", (double)boys_series(n, x));
            g_boys[r][n] = strtod(buf, NULL);
        }
    }
    g_boys_ready = 1;
}

double orc_boys(int n, double x)
{
    static const double kfact[7] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0};
    if (n < 0 || n >= BOYS_COLS)
        return NAN;
    const double x_max = BOYS_ROWS * BOYS_STEP;
    if (x >= x_max)
        return tgamma(n + 0.5) / (2.0 * pow(x, n + 0.5));
    const int xi = (int)(x / BOYS_STEP);
    const double delta = x - xi * BOYS_STEP;
    const int max_k = (6 < BOYS_COLS - 1 - n) ? 6 : BOYS_COLS - 1 - n;
    double result = g_boys[xi][n];
    double delta_k = delta;
    double sign = -1.0;
    for (int k = 1; k <= max_k; ++k, delta_k *= delta, sign = -sign)
        result += sign * g_boys[xi][n + k] / kfact[k] * delta_k;
    return result;
}

/* ------------------------------------------------------------------------ */
/* Basis and AO pairs: src/base/types.h:263-327 (Shell, ContractedView),     */
/* src/basis/basis.cpp:20-37 (Cartesian order lx desc, ly desc),             */
/* src/basis/gaussian.cpp:283-296 (component norm 1/sqrt((2lx-1)!!...)),     */
/* src/base/types.h:606-675 (PrimitivePair / ShellPair ctor),                */
/* src/integrals/shellpair.cpp:7-22 (pair order: i <= j row-major).          */
/* ------------------------------------------------------------------------ */
typedef struct {
    double alpha, beta, zeta, inv_zeta, prefactor, coeff_product;
    double P[3], pA[3], pB[3];
} orc_pp;

typedef struct {
    int i, j;            /* AO indices, i <= j */
    double R[3], R2;
    int npp;
    orc_pp *pp;
} orc_pair;

typedef struct {
    int shell;
    int lx, ly, lz;
    double cnorm;
} orc_ao;

typedef struct {
    int nshell, nbasis;
    int *L, *nprim, *off;     /* off: primitive offset per shell */
    double *center;           /* 3 per shell */
    double *expo, *coef, *norm;
    orc_ao *ao;
    int npairs;
    orc_pair *pairs;
} orc_basis;

static int dfact(int n)
{
    if (n <= 0)
        return 1;
    int r = 1;
    while (n > 0) {
        r *= n;
        n -= 2;
    }
    return r;
}

/* primitive and contracted normalisation: src/basis/basis.cpp:39-75 */
void orc_normalize_shell(int L, int nprim, const double *expo, const double *raw_coef,
                         double *coef_out, double *norm_out)
{
    const double pi = 3.1415926535897932384626433832795;
    const double prefactor = pow(2.0, 2.0 * L + 1.5) / pow(pi, 1.5);
    for (int i = 0; i < nprim; ++i)
        norm_out[i] = sqrt(pow(expo[i], L + 1.5) * prefactor);
    const double pi_factor = pow(pi, 1.5) / pow(2.0, L);
    double sum = 0.0;
    for (int j = 0; j < nprim; ++j)      /* Eigen column-major sum order */
        for (int i = 0; i < nprim; ++i) {
            const double aij = expo[i] + expo[j];
            const double sij = pi_factor / pow(aij, L + 1.5);
            sum += raw_coef[i] * raw_coef[j] * norm_out[i] * norm_out[j] * sij;
        }
    const double Nc = 1.0 / sqrt(sum);
    for (int i = 0; i < nprim; ++i)
        coef_out[i] = raw_coef[i] * Nc;
}

orc_basis *orc_basis_create(int nshell, const int *L, const int *nprim, const double *center,
                            const double *expo, const double *coef, const double *norm)
{
    orc_boys_init();
    orc_basis *b = calloc(1, sizeof *b);
    b->nshell = nshell;
    b->L = malloc(sizeof(int) * nshell);
    b->nprim = malloc(sizeof(int) * nshell);
    b->off = malloc(sizeof(int) * (nshell + 1));
    b->center = malloc(sizeof(double) * 3 * nshell);
    int tot = 0, nb = 0;
    for (int s = 0; s < nshell; ++s) {
        b->L[s] = L[s];
        b->nprim[s] = nprim[s];
        b->off[s] = tot;
        tot += nprim[s];
        nb += (L[s] + 1) * (L[s] + 2) / 2;
        for (int d = 0; d < 3; ++d)
            b->center[3 * s + d] = center[3 * s + d];
    }
    b->off[nshell] = tot;
    b->expo = malloc(sizeof(double) * tot);
    b->coef = malloc(sizeof(double) * tot);
    b->norm = malloc(sizeof(double) * tot);
    memcpy(b->expo, expo, sizeof(double) * tot);
    memcpy(b->coef, coef, sizeof(double) * tot);
    memcpy(b->norm, norm, sizeof(double) * tot);
    b->nbasis = nb;
    b->ao = malloc(sizeof(orc_ao) * nb);
    int k = 0;
    for (int s = 0; s < nshell; ++s)
        for (int lx = L[s]; lx >= 0; --lx)
            for (int ly = L[s] - lx; ly >= 0; --ly) {
                const int lz = L[s] - lx - ly;
                b->ao[k].shell = s;
                b->ao[k].lx = lx;
                b->ao[k].ly = ly;
                b->ao[k].lz = lz;
                b->ao[k].cnorm = 1.0 / sqrt((double)(dfact(2 * lx - 1) * dfact(2 * ly - 1) * dfact(2 * lz - 1)));
                ++k;
            }
    b->npairs = nb * (nb + 1) / 2;
    b->pairs = calloc(b->npairs, sizeof(orc_pair));
    int p = 0;
    for (int i = 0; i < nb; ++i)
        for (int j = i; j < nb; ++j, ++p) {
            orc_pair *sp = &b->pairs[p];
            const int sa = b->ao[i].shell, sb = b->ao[j].shell;
            const double *A = &b->center[3 * sa], *B = &b->center[3 * sb];
            sp->i = i;
            sp->j = j;
            for (int d = 0; d < 3; ++d)
                sp->R[d] = A[d] - B[d];
            sp->R2 = sp->R[0] * sp->R[0] + sp->R[1] * sp->R[1] + sp->R[2] * sp->R[2];
            sp->npp = b->nprim[sa] * b->nprim[sb];
            sp->pp = malloc(sizeof(orc_pp) * sp->npp);
            int q = 0;
            for (int ia = 0; ia < b->nprim[sa]; ++ia)
                for (int ib = 0; ib < b->nprim[sb]; ++ib, ++q) {
                    orc_pp *pp = &sp->pp[q];
                    const double alpha = b->expo[b->off[sa] + ia];
                    const double beta = b->expo[b->off[sb] + ib];
                    const double zeta = alpha + beta;
                    const double inv_zeta = 1.0 / zeta;
                    const double abz = alpha * beta * inv_zeta;
                    pp->alpha = alpha;
                    pp->beta = beta;
                    pp->zeta = zeta;
                    pp->inv_zeta = inv_zeta;
                    pp->coeff_product = b->coef[b->off[sa] + ia] * b->coef[b->off[sb] + ib] *
                                        b->norm[b->off[sa] + ia] * b->norm[b->off[sb] + ib] *
                                        b->ao[i].cnorm * b->ao[j].cnorm;
                    pp->prefactor = pow(ORC_PI * inv_zeta, 1.5) * exp(-abz * sp->R2);
                    for (int d = 0; d < 3; ++d) {
                        pp->P[d] = (alpha * A[d] + beta * B[d]) * inv_zeta;
                        pp->pA[d] = pp->P[d] - A[d];
                        pp->pB[d] = pp->P[d] - B[d];
                    }
                }
        }
    return b;
}

void orc_basis_destroy(orc_basis *b)
{
    if (!b)
        return;
    for (int p = 0; p < b->npairs; ++p)
        free(b->pairs[p].pp);
    free(b->pairs);
    free(b->ao);
    free(b->L);
    free(b->nprim);
    free(b->off);
    free(b->center);
    free(b->expo);
    free(b->coef);
    free(b->norm);
    free(b);
}

int orc_nbasis(const orc_basis *b) { return b->nbasis; }
int orc_npairs(const orc_basis *b) { return b->npairs; }

void orc_ao_info(const orc_basis *b, int *shell, int *lxyz, double *cnorm)
{
    for (int k = 0; k < b->nbasis; ++k) {
        shell[k] = b->ao[k].shell;
        lxyz[3 * k] = b->ao[k].lx;
        lxyz[3 * k + 1] = b->ao[k].ly;
        lxyz[3 * k + 2] = b->ao[k].lz;
        cnorm[k] = b->ao[k].cnorm;
    }
}

/* ------------------------------------------------------------------------ */
/* Obara-Saika ERI for one Cartesian component quartet.                      */
/* VRR: src/integrals/os.cpp:618-828; HRR A->B: os.cpp:837-879;             */
/* C->D via _nuclear_hrr: os.cpp:415-459; primitive: os.cpp:882-924;        */
/* contraction: os.cpp:994-1010.                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
    int d[7];            /* ax, ay, az, cx, cy, cz, m dims */
    size_t cap_v, cap_h;
    double *v, *h;
    /* Rys accumulation buffer */
    size_t cap_r;
    double *r;
} orc_scratch;

static _Thread_local orc_scratch g_scr;

static inline size_t sidx(const orc_scratch *s, int ax, int ay, int az, int cx, int cy, int cz)
{
    size_t i = (size_t)ax;
    i = i * s->d[1] + ay;
    i = i * s->d[2] + az;
    i = i * s->d[3] + cx;
    i = i * s->d[4] + cy;
    i = i * s->d[5] + cz;
    return i;
}
#define V(ax, ay, az, cx, cy, cz, m) s->v[sidx(s, ax, ay, az, cx, cy, cz) * s->d[6] + (m)]
#define Hh(ax, ay, az, cx, cy, cz) s->h[sidx(s, ax, ay, az, cx, cy, cz)]

static void scratch_resize(orc_scratch *s, int lABx, int lABy, int lABz, int lCDx, int lCDy, int lCDz, int mmax)
{
    s->d[0] = lABx + 1;
    s->d[1] = lABy + 1;
    s->d[2] = lABz + 1;
    s->d[3] = lCDx + 1;
    s->d[4] = lCDy + 1;
    s->d[5] = lCDz + 1;
    s->d[6] = mmax + 1;
    size_t spatial = (size_t)s->d[0] * s->d[1] * s->d[2] * s->d[3] * s->d[4] * s->d[5];
    size_t nv = spatial * s->d[6];
    if (nv > s->cap_v) {
        free(s->v);
        s->v = malloc(sizeof(double) * nv);
        s->cap_v = nv;
    }
    memset(s->v, 0, sizeof(double) * nv);
    if (spatial > s->cap_h) {
        free(s->h);
        s->h = malloc(sizeof(double) * spatial);
        s->cap_h = spatial;
    }
}

#define VD 13 /* 2*MAX_L+1 with the reference's MAX_L = 6 */

/* os.cpp:415-459 */
static double nuclear_hrr(double V0[VD][VD][VD], int ax, int ay, int az, int bx, int by, int bz,
                          double ABx, double ABy, double ABz)
{
    if (bx == 0 && by == 0 && bz == 0)
        return V0[ax][ay][az];
    double W[VD][VD][VD];
    for (int ix = 0; ix <= ax + bx; ix++)
        for (int iy = 0; iy <= ay + by; iy++)
            for (int iz = 0; iz <= az + bz; iz++)
                W[ix][iy][iz] = V0[ix][iy][iz];
    for (int kz = 0; kz < bz; kz++)
        for (int ix = 0; ix <= ax + bx; ix++)
            for (int iy = 0; iy <= ay + by; iy++)
                for (int iz = 0; iz <= az + bz - kz - 1; iz++)
                    W[ix][iy][iz] = W[ix][iy][iz + 1] + ABz * W[ix][iy][iz];
    for (int ky = 0; ky < by; ky++)
        for (int ix = 0; ix <= ax + bx; ix++)
            for (int iy = 0; iy <= ay + by - ky - 1; iy++)
                for (int iz = 0; iz <= az; iz++)
                    W[ix][iy][iz] = W[ix][iy + 1][iz] + ABy * W[ix][iy][iz];
    for (int kx = 0; kx < bx; kx++)
        for (int ix = 0; ix <= ax + bx - kx - 1; ix++)
            for (int iy = 0; iy <= ay; iy++)
                for (int iz = 0; iz <= az; iz++)
                    W[ix][iy][iz] = W[ix + 1][iy][iz] + ABx * W[ix][iy][iz];
    return W[ax][ay][az];
}

/* os.cpp:618-828 */
static void eri_vrr(orc_scratch *s, const orc_pp *ab, const orc_pp *cd,
                    int lABx, int lABy, int lABz, int lCDx, int lCDy, int lCDz)
{
    const double zAB = ab->zeta, zCD = cd->zeta;
    const double delta = zAB + zCD;
    const double rho = zAB * zCD / delta;
    const double i2zAB = 0.5 / zAB, i2zCD = 0.5 / zCD, i2d = 0.5 / delta;
    const double rzAB = rho / zAB, rzCD = rho / zCD;
    const double *P = ab->P, *Q = cd->P;
    const double Wx = (zAB * P[0] + zCD * Q[0]) / delta;
    const double Wy = (zAB * P[1] + zCD * Q[1]) / delta;
    const double Wz = (zAB * P[2] + zCD * Q[2]) / delta;
    const double WPx = Wx - P[0], WPy = Wy - P[1], WPz = Wz - P[2];
    const double WQx = Wx - Q[0], WQy = Wy - Q[1], WQz = Wz - Q[2];
    const double PAx = ab->pA[0], PAy = ab->pA[1], PAz = ab->pA[2];
    const double QCx = cd->pA[0], QCy = cd->pA[1], QCz = cd->pA[2];
    const double PQx = P[0] - Q[0], PQy = P[1] - Q[1], PQz = P[2] - Q[2];
    const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
    const int MMAX = lABx + lABy + lABz + lCDx + lCDy + lCDz;
    const double prefac = ab->prefactor * cd->prefactor * 2.0 * sqrt(rho / ORC_PI);

    for (int m = 0; m <= MMAX; ++m)
        V(0, 0, 0, 0, 0, 0, m) = prefac * orc_boys(m, T);
    for (int ax = 1; ax <= lABx; ++ax) {
        const int mlim = MMAX - ax;
        for (int m = 0; m <= mlim; ++m) {
            V(ax, 0, 0, 0, 0, 0, m) = PAx * V(ax - 1, 0, 0, 0, 0, 0, m) + WPx * V(ax - 1, 0, 0, 0, 0, 0, m + 1);
            if (ax > 1)
                V(ax, 0, 0, 0, 0, 0, m) += (ax - 1) * i2zAB *
                    (V(ax - 2, 0, 0, 0, 0, 0, m) - rzAB * V(ax - 2, 0, 0, 0, 0, 0, m + 1));
        }
    }
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 1; ay <= lABy; ++ay) {
            const int mlim = MMAX - ax - ay;
            if (mlim < 0)
                continue;
            for (int m = 0; m <= mlim; ++m) {
                V(ax, ay, 0, 0, 0, 0, m) = PAy * V(ax, ay - 1, 0, 0, 0, 0, m) + WPy * V(ax, ay - 1, 0, 0, 0, 0, m + 1);
                if (ay > 1)
                    V(ax, ay, 0, 0, 0, 0, m) += (ay - 1) * i2zAB *
                        (V(ax, ay - 2, 0, 0, 0, 0, m) - rzAB * V(ax, ay - 2, 0, 0, 0, 0, m + 1));
            }
        }
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 0; ay <= lABy; ++ay)
            for (int az = 1; az <= lABz; ++az) {
                const int mlim = MMAX - ax - ay - az;
                if (mlim < 0)
                    continue;
                for (int m = 0; m <= mlim; ++m) {
                    V(ax, ay, az, 0, 0, 0, m) = PAz * V(ax, ay, az - 1, 0, 0, 0, m) + WPz * V(ax, ay, az - 1, 0, 0, 0, m + 1);
                    if (az > 1)
                        V(ax, ay, az, 0, 0, 0, m) += (az - 1) * i2zAB *
                            (V(ax, ay, az - 2, 0, 0, 0, m) - rzAB * V(ax, ay, az - 2, 0, 0, 0, m + 1));
                }
            }
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 0; ay <= lABy; ++ay)
            for (int az = 0; az <= lABz; ++az)
                for (int cx = 1; cx <= lCDx; ++cx) {
                    const int mlim = MMAX - ax - ay - az - cx;
                    if (mlim < 0)
                        continue;
                    for (int m = 0; m <= mlim; ++m) {
                        V(ax, ay, az, cx, 0, 0, m) = QCx * V(ax, ay, az, cx - 1, 0, 0, m) + WQx * V(ax, ay, az, cx - 1, 0, 0, m + 1);
                        if (cx > 1)
                            V(ax, ay, az, cx, 0, 0, m) += (cx - 1) * i2zCD *
                                (V(ax, ay, az, cx - 2, 0, 0, m) - rzCD * V(ax, ay, az, cx - 2, 0, 0, m + 1));
                        if (ax > 0)
                            V(ax, ay, az, cx, 0, 0, m) += ax * i2d * V(ax - 1, ay, az, cx - 1, 0, 0, m + 1);
                    }
                }
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 0; ay <= lABy; ++ay)
            for (int az = 0; az <= lABz; ++az)
                for (int cx = 0; cx <= lCDx; ++cx)
                    for (int cy = 1; cy <= lCDy; ++cy) {
                        const int mlim = MMAX - ax - ay - az - cx - cy;
                        if (mlim < 0)
                            continue;
                        for (int m = 0; m <= mlim; ++m) {
                            V(ax, ay, az, cx, cy, 0, m) = QCy * V(ax, ay, az, cx, cy - 1, 0, m) + WQy * V(ax, ay, az, cx, cy - 1, 0, m + 1);
                            if (cy > 1)
                                V(ax, ay, az, cx, cy, 0, m) += (cy - 1) * i2zCD *
                                    (V(ax, ay, az, cx, cy - 2, 0, m) - rzCD * V(ax, ay, az, cx, cy - 2, 0, m + 1));
                            if (ay > 0)
                                V(ax, ay, az, cx, cy, 0, m) += ay * i2d * V(ax, ay - 1, az, cx, cy - 1, 0, m + 1);
                        }
                    }
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 0; ay <= lABy; ++ay)
            for (int az = 0; az <= lABz; ++az)
                for (int cx = 0; cx <= lCDx; ++cx)
                    for (int cy = 0; cy <= lCDy; ++cy)
                        for (int cz = 1; cz <= lCDz; ++cz) {
                            const int mlim = MMAX - ax - ay - az - cx - cy - cz;
                            if (mlim < 0)
                                continue;
                            for (int m = 0; m <= mlim; ++m) {
                                V(ax, ay, az, cx, cy, cz, m) = QCz * V(ax, ay, az, cx, cy, cz - 1, m) + WQz * V(ax, ay, az, cx, cy, cz - 1, m + 1);
                                if (cz > 1)
                                    V(ax, ay, az, cx, cy, cz, m) += (cz - 1) * i2zCD *
                                        (V(ax, ay, az, cx, cy, cz - 2, m) - rzCD * V(ax, ay, az, cx, cy, cz - 2, m + 1));
                                if (az > 0)
                                    V(ax, ay, az, cx, cy, cz, m) += az * i2d * V(ax, ay, az - 1, cx, cy, cz - 1, m + 1);
                            }
                        }
}

/* os.cpp:837-879, operating on the h buffer (also used by Rys: rys.cpp:293-325) */
static void hrr_ab(orc_scratch *s, int lAx, int lAy, int lAz, int lBx, int lBy, int lBz,
                   int lCDx, int lCDy, int lCDz, double ABx, double ABy, double ABz)
{
    for (int kz = 0; kz < lBz; ++kz)
        for (int ax = 0; ax <= lAx + lBx; ++ax)
            for (int ay = 0; ay <= lAy + lBy; ++ay)
                for (int az = 0; az <= lAz + lBz - kz - 1; ++az)
                    for (int cx = 0; cx <= lCDx; ++cx)
                        for (int cy = 0; cy <= lCDy; ++cy)
                            for (int cz = 0; cz <= lCDz; ++cz)
                                Hh(ax, ay, az, cx, cy, cz) = Hh(ax, ay, az + 1, cx, cy, cz) + ABz * Hh(ax, ay, az, cx, cy, cz);
    for (int ky = 0; ky < lBy; ++ky)
        for (int ax = 0; ax <= lAx + lBx; ++ax)
            for (int ay = 0; ay <= lAy + lBy - ky - 1; ++ay)
                for (int az = 0; az <= lAz; ++az)
                    for (int cx = 0; cx <= lCDx; ++cx)
                        for (int cy = 0; cy <= lCDy; ++cy)
                            for (int cz = 0; cz <= lCDz; ++cz)
                                Hh(ax, ay, az, cx, cy, cz) = Hh(ax, ay + 1, az, cx, cy, cz) + ABy * Hh(ax, ay, az, cx, cy, cz);
    for (int kx = 0; kx < lBx; ++kx)
        for (int ax = 0; ax <= lAx + lBx - kx - 1; ++ax)
            for (int ay = 0; ay <= lAy; ++ay)
                for (int az = 0; az <= lAz; ++az)
                    for (int cx = 0; cx <= lCDx; ++cx)
                        for (int cy = 0; cy <= lCDy; ++cy)
                            for (int cz = 0; cz <= lCDz; ++cz)
                                Hh(ax, ay, az, cx, cy, cz) = Hh(ax + 1, ay, az, cx, cy, cz) + ABx * Hh(ax, ay, az, cx, cy, cz);
}

typedef struct {
    int a[3], b[3], c[3], d[3];
} orc_comp;

/* os.cpp:882-924 */
static double os_primitive(const orc_pp *ab, const orc_pp *cd, const orc_comp *q,
                           const double *AB, const double *CD)
{
    orc_scratch *s = &g_scr;
    const int lABx = q->a[0] + q->b[0], lABy = q->a[1] + q->b[1], lABz = q->a[2] + q->b[2];
    const int lCDx = q->c[0] + q->d[0], lCDy = q->c[1] + q->d[1], lCDz = q->c[2] + q->d[2];
    const int mmax = lABx + lABy + lABz + lCDx + lCDy + lCDz;
    scratch_resize(s, lABx, lABy, lABz, lCDx, lCDy, lCDz, mmax);
    eri_vrr(s, ab, cd, lABx, lABy, lABz, lCDx, lCDy, lCDz);
    for (int ax = 0; ax <= lABx; ++ax)
        for (int ay = 0; ay <= lABy; ++ay)
            for (int az = 0; az <= lABz; ++az)
                for (int cx = 0; cx <= lCDx; ++cx)
                    for (int cy = 0; cy <= lCDy; ++cy)
                        for (int cz = 0; cz <= lCDz; ++cz)
                            Hh(ax, ay, az, cx, cy, cz) = V(ax, ay, az, cx, cy, cz, 0);
    hrr_ab(s, q->a[0], q->a[1], q->a[2], q->b[0], q->b[1], q->b[2], lCDx, lCDy, lCDz, AB[0], AB[1], AB[2]);
    double V0[VD][VD][VD];
    memset(V0, 0, sizeof V0);
    for (int cx = 0; cx <= lCDx; ++cx)
        for (int cy = 0; cy <= lCDy; ++cy)
            for (int cz = 0; cz <= lCDz; ++cz)
                V0[cx][cy][cz] = Hh(q->a[0], q->a[1], q->a[2], cx, cy, cz);
    return nuclear_hrr(V0, q->c[0], q->c[1], q->c[2], q->d[0], q->d[1], q->d[2], CD[0], CD[1], CD[2]);
}

/* ------------------------------------------------------------------------ */
/* Rys quadrature.  Roots: src/integrals/rys_roots.cpp:88-235 and           */
/* rys_roots.h:28-43.  1D VRR: rys.cpp:250-280.  Primitive: rys.cpp:367-485 */
/* (6D accumulation, prefactor, AB-HRR, CD-HRR rys.cpp:329-363).            */
/* ------------------------------------------------------------------------ */
#define RYS_MAX 11

static long double boys_moment(int m, long double T)
{
    if (T < 1.0e-14L)
        return 1.0L / (long double)(2 * m + 1);
    if (T < 1.0L) {
        long double sum = 0.0L, coeff = 1.0L;
        for (int n = 0; n < 256; ++n) {
            const long double term = coeff / (long double)(2 * m + 2 * n + 1);
            sum += term;
            if (fabsl(term) < 1.0e-28L * fabsl(sum))
                break;
            coeff *= -T / (long double)(n + 1);
        }
        return sum;
    }
    const long double sqrtT = sqrtl(T);
    long double F = 0.5L * sqrtl(3.141592653589793238462643383279502884L / T) * erfl(sqrtT);
    if (m == 0)
        return F;
    const long double eT = expl(-T);
    for (int k = 1; k <= m; ++k)
        F = ((2 * k - 1) * F - eT) / (2.0L * T);
    return F;
}

static long double poly_inner(const long double *a, int da, const long double *b, int db, const long double *mom)
{
    long double s = 0.0L;
    for (int i = 0; i <= da; ++i)
        for (int j = 0; j <= db; ++j)
            s += a[i] * b[j] * mom[i + j];
    return s;
}

/* Symmetric tridiagonal eigenproblem by implicit-shift QL (EISPACK tql2).
 * d: diagonal (n), e: subdiagonal in e[0..n-2]; z: n x n, row-major,
 * initialised to identity; on return d holds eigenvalues (ascending) and
 * column k of z the k-th eigenvector.  Returns 0 on success. */
static int tql2(int n, double *d, double *e, double *z)
{
    double ee[RYS_MAX + 1];
    for (int i = 0; i < n - 1; ++i)
        ee[i] = e[i];
    ee[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        double h = fabs(d[l]) + fabs(ee[l]);
        if (tst1 < h)
            tst1 = h;
        int m = l;
        while (m < n) {
            if (tst1 + fabs(ee[m]) == tst1)
                break;
            ++m;
        }
        if (m == n)
            m = n - 1;
        if (m > l) {
            do {
                if (++iter > 60)
                    return 1;
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * ee[l]);
                double r = hypot(p, 1.0);
                d[l] = ee[l] / (p + (p >= 0 ? r : -r));
                d[l + 1] = ee[l] * (p + (p >= 0 ? r : -r));
                double dl1 = d[l + 1];
                h = g - d[l];
                for (int i = l + 2; i < n; ++i)
                    d[i] -= h;
                f += h;
                p = d[m];
                double c = 1.0, c2 = 1.0, c3 = 1.0, el1 = ee[l + 1], s = 0.0, s2 = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * ee[i];
                    h = c * p;
                    r = hypot(p, ee[i]);
                    ee[i + 1] = s * r;
                    s = ee[i] / r;
                    c = p / r;
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; ++k) {
                        h = z[k * n + i + 1];
                        z[k * n + i + 1] = s * z[k * n + i] + c * h;
                        z[k * n + i] = c * z[k * n + i] - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * ee[l] / dl1;
                ee[l] = s * p;
                d[l] = c * p;
            } while (tst1 + fabs(ee[l]) > tst1);
        }
        d[l] = d[l] + f;
        ee[l] = 0.0;
    }
    /* sort ascending */
    for (int i = 0; i < n - 1; ++i) {
        int k = i;
        double p = d[i];
        for (int j = i + 1; j < n; ++j)
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int j = 0; j < n; ++j) {
                double t = z[j * n + i];
                z[j * n + i] = z[j * n + k];
                z[j * n + k] = t;
            }
        }
    }
    return 0;
}

/* Gauss-Legendre fallback on [0,1] (rys_roots.cpp:17-86): used by the
 * reference only when the Jacobi build breaks down.  Computed here from the
 * Legendre recurrence by Newton iteration instead of being tabulated. */
static void rys_gl_fallback(int n, double *roots, double *weights)
{
    for (int i = 0; i < n; ++i) {
        double x = cos(ORC_PI * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double pn = (n == 1) ? x : p1;
            double pm = (n == 1) ? 1.0 : p0;
            dp = n * (x * pn - pm) / (x * x - 1.0);
            double dx = pn / dp;
            x -= dx;
            if (fabs(dx) < 1e-16)
                break;
        }
        roots[n - 1 - i] = 0.5 * (1.0 - x);
        weights[n - 1 - i] = 1.0 / ((1.0 - x * x) * dp * dp);
    }
}

void orc_rys_roots(int n, double T, double *roots, double *weights)
{
    if (n == 1) { /* rys_roots.h:28-43 */
        if (T < 1.0e-14) {
            roots[0] = 1.0 / 3.0;
            weights[0] = 1.0;
        } else {
            const double sqrtT = sqrt(T);
            const double F0 = 0.5 * sqrt(ORC_PI / T) * erf(sqrtT);
            const double F1 = (F0 - exp(-T)) / (2.0 * T);
            roots[0] = F1 / F0;
            weights[0] = F0;
        }
        return;
    }
    /* rys_roots.cpp:135-219 */
    long double mom[2 * RYS_MAX + 1];
    for (int k = 0; k <= 2 * n; ++k)
        mom[k] = boys_moment(k, (long double)T);
    long double polys[RYS_MAX + 1][RYS_MAX + 1];
    long double alphas[RYS_MAX], betas[RYS_MAX];
    memset(polys, 0, sizeof polys);
    memset(alphas, 0, sizeof alphas);
    memset(betas, 0, sizeof betas);
    polys[0][0] = 1.0L / sqrtl(mom[0]);
    for (int k = 0; k < n; ++k) {
        long double xpk[RYS_MAX + 1];
        memset(xpk, 0, sizeof xpk);
        for (int i = 0; i <= k; ++i)
            xpk[i + 1] = polys[k][i];
        alphas[k] = poly_inner(xpk, k + 1, polys[k], k, mom);
        if (k == n - 1)
            break;
        long double q[RYS_MAX + 1];
        memset(q, 0, sizeof q);
        for (int i = 0; i <= k + 1; ++i)
            q[i] += xpk[i];
        for (int i = 0; i <= k; ++i)
            q[i] -= alphas[k] * polys[k][i];
        if (k > 0)
            for (int i = 0; i <= k - 1; ++i)
                q[i] -= betas[k - 1] * polys[k - 1][i];
        long double norm2 = poly_inner(q, k + 1, q, k + 1, mom);
        if (norm2 < 0.0L && fabsl(norm2) < 1.0e-24L)
            norm2 = 0.0L;
        betas[k] = sqrtl(norm2);
        if (!(betas[k] > 0.0L)) {
            rys_gl_fallback(n, roots, weights);
            return;
        }
        for (int i = 0; i <= k + 1; ++i)
            polys[k + 1][i] = q[i] / betas[k];
    }
    double d[RYS_MAX], e[RYS_MAX], z[RYS_MAX * RYS_MAX];
    for (int i = 0; i < n; ++i) {
        d[i] = (double)alphas[i];
        e[i] = (i + 1 < n) ? (double)betas[i] : 0.0;
        for (int j = 0; j < n; ++j)
            z[i * n + j] = (i == j) ? 1.0 : 0.0;
    }
    if (tql2(n, d, e, z) != 0) {
        rys_gl_fallback(n, roots, weights);
        return;
    }
    const double m0 = (double)mom[0];
    for (int i = 0; i < n; ++i) {
        double r = d[i];
        roots[i] = r < 0.0 ? 0.0 : (r > 1.0 ? 1.0 : r);
        double w = m0 * z[i] * z[i];
        weights[i] = w > 0.0 ? w : 0.0;
    }
}

/* rys.cpp:250-280 */
static void rys_vrr_1d(double vrr[VD][VD], int lAB, int lCD, double C00, double D00,
                       double B00, double B10, double B01)
{
    vrr[0][0] = 1.0;
    for (int a = 1; a <= lAB; ++a) {
        vrr[a][0] = C00 * vrr[a - 1][0];
        if (a >= 2)
            vrr[a][0] += (a - 1) * B10 * vrr[a - 2][0];
    }
    for (int c = 1; c <= lCD; ++c) {
        vrr[0][c] = D00 * vrr[0][c - 1];
        if (c >= 2)
            vrr[0][c] += (c - 1) * B01 * vrr[0][c - 2];
        for (int a = 1; a <= lAB; ++a) {
            vrr[a][c] = D00 * vrr[a][c - 1] + a * B00 * vrr[a - 1][c - 1];
            if (c >= 2)
                vrr[a][c] += (c - 1) * B01 * vrr[a][c - 2];
        }
    }
}

/* rys.cpp:329-363 */
static double rys_hrr_cd(double V0[VD][VD][VD], int lCx, int lCy, int lCz, int lDx, int lDy, int lDz,
                         double CDx, double CDy, double CDz)
{
    double W[VD][VD][VD];
    for (int cx = 0; cx <= lCx + lDx; ++cx)
        for (int cy = 0; cy <= lCy + lDy; ++cy)
            for (int cz = 0; cz <= lCz + lDz; ++cz)
                W[cx][cy][cz] = V0[cx][cy][cz];
    for (int kx = 0; kx < lDx; ++kx)
        for (int cx = 0; cx <= lCx + lDx - kx - 1; ++cx)
            for (int cy = 0; cy <= lCy + lDy; ++cy)
                for (int cz = 0; cz <= lCz + lDz; ++cz)
                    W[cx][cy][cz] = W[cx + 1][cy][cz] + CDx * W[cx][cy][cz];
    for (int ky = 0; ky < lDy; ++ky)
        for (int cy = 0; cy <= lCy + lDy - ky - 1; ++cy)
            for (int cz = 0; cz <= lCz + lDz; ++cz)
                W[lCx][cy][cz] = W[lCx][cy + 1][cz] + CDy * W[lCx][cy][cz];
    for (int kz = 0; kz < lDz; ++kz)
        for (int cz = 0; cz <= lCz + lDz - kz - 1; ++cz)
            W[lCx][lCy][cz] = W[lCx][lCy][cz + 1] + CDz * W[lCx][lCy][cz];
    return W[lCx][lCy][lCz];
}

/* rys.cpp:367-485 */
static double rys_primitive(const orc_pp *ab, const orc_pp *cd, const orc_comp *q,
                            const double *AB, const double *CD)
{
    orc_scratch *s = &g_scr;
    const double zeta = ab->zeta, eta = cd->zeta;
    const double delta = zeta + eta;
    const double inv_delta = 1.0 / delta;
    const double rho = zeta * eta * inv_delta;
    const double roz = rho * ab->inv_zeta, roe = rho * cd->inv_zeta;
    const double Px = ab->P[0], Py = ab->P[1], Pz = ab->P[2];
    const double Qx = cd->P[0], Qy = cd->P[1], Qz = cd->P[2];
    const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
    const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
    const double PAx = ab->pA[0], PAy = ab->pA[1], PAz = ab->pA[2];
    const double QCx = cd->pA[0], QCy = cd->pA[1], QCz = cd->pA[2];
    const double Wx = (zeta * Px + eta * Qx) * inv_delta;
    const double Wy = (zeta * Py + eta * Qy) * inv_delta;
    const double Wz = (zeta * Pz + eta * Qz) * inv_delta;
    const double WPx = Wx - Px, WPy = Wy - Py, WPz = Wz - Pz;
    const double WQx = Wx - Qx, WQy = Wy - Qy, WQz = Wz - Qz;
    const double prefac = ab->prefactor * cd->prefactor * 2.0 * sqrt(rho / ORC_PI);
    const int lABx = q->a[0] + q->b[0], lABy = q->a[1] + q->b[1], lABz = q->a[2] + q->b[2];
    const int lCDx = q->c[0] + q->d[0], lCDy = q->c[1] + q->d[1], lCDz = q->c[2] + q->d[2];
    const int L = lABx + lABy + lABz + lCDx + lCDy + lCDz;
    const int n = L / 2 + 1;
    double t2[RYS_MAX], w[RYS_MAX];
    orc_rys_roots(n, T, t2, w);

    /* the 6D buffer lives in the h slot; size it like the OS scratch */
    s->d[0] = lABx + 1; s->d[1] = lABy + 1; s->d[2] = lABz + 1;
    s->d[3] = lCDx + 1; s->d[4] = lCDy + 1; s->d[5] = lCDz + 1; s->d[6] = 1;
    size_t spatial = (size_t)s->d[0] * s->d[1] * s->d[2] * s->d[3] * s->d[4] * s->d[5];
    if (spatial > s->cap_h) {
        free(s->h);
        s->h = malloc(sizeof(double) * spatial);
        s->cap_h = spatial;
    }
    memset(s->h, 0, sizeof(double) * spatial);
    for (int r = 0; r < n; ++r) {
        const double u = t2[r], wr = w[r];
        const double B00 = 0.5 * inv_delta * u;
        const double B10 = 0.5 * ab->inv_zeta * (1.0 - roz * u);
        const double B01 = 0.5 * cd->inv_zeta * (1.0 - roe * u);
        double Ix[VD][VD], Iy[VD][VD], Iz[VD][VD];
        rys_vrr_1d(Ix, lABx, lCDx, PAx + u * WPx, QCx + u * WQx, B00, B10, B01);
        rys_vrr_1d(Iy, lABy, lCDy, PAy + u * WPy, QCy + u * WQy, B00, B10, B01);
        rys_vrr_1d(Iz, lABz, lCDz, PAz + u * WPz, QCz + u * WQz, B00, B10, B01);
        for (int ax = 0; ax <= lABx; ++ax)
            for (int ay = 0; ay <= lABy; ++ay)
                for (int az = 0; az <= lABz; ++az)
                    for (int cx = 0; cx <= lCDx; ++cx)
                        for (int cy = 0; cy <= lCDy; ++cy)
                            for (int cz = 0; cz <= lCDz; ++cz)
                                Hh(ax, ay, az, cx, cy, cz) += wr * Ix[ax][cx] * Iy[ay][cy] * Iz[az][cz];
    }
    for (size_t i = 0; i < spatial; ++i)
        s->h[i] *= prefac;
    hrr_ab(s, q->a[0], q->a[1], q->a[2], q->b[0], q->b[1], q->b[2], lCDx, lCDy, lCDz, AB[0], AB[1], AB[2]);
    double V0[VD][VD][VD];
    for (int cx = 0; cx <= lCDx; ++cx)
        for (int cy = 0; cy <= lCDy; ++cy)
            for (int cz = 0; cz <= lCDz; ++cz)
                V0[cx][cy][cz] = Hh(q->a[0], q->a[1], q->a[2], cx, cy, cz);
    return rys_hrr_cd(V0, q->c[0], q->c[1], q->c[2], q->d[0], q->d[1], q->d[2], CD[0], CD[1], CD[2]);
}

/* rys.cpp:195-220 */
static int auto_prefers_rys(const orc_comp *q)
{
    const int lABx = q->a[0] + q->b[0], lABy = q->a[1] + q->b[1], lABz = q->a[2] + q->b[2];
    const int lCDx = q->c[0] + q->d[0], lCDy = q->c[1] + q->d[1], lCDz = q->c[2] + q->d[2];
    const int L = lABx + lABy + lABz + lCDx + lCDy + lCDz;
    const int nroots = L / 2 + 1;
    const double six_d = (double)(lABx + 1) * (double)(lABy + 1) * (double)(lABz + 1) *
                         (double)(lCDx + 1) * (double)(lCDy + 1) * (double)(lCDz + 1);
    const int lbd = q->b[0] + q->b[1] + q->b[2] + q->d[0] + q->d[1] + q->d[2];
    const double os_work = six_d * (double)(L + 1) + (double)(lbd + 1) * six_d * 0.25;
    const double rys_work = six_d * (double)nroots + (double)(lbd + 1) * six_d * 0.20 + 24.0 * (double)nroots;
    return rys_work < os_work;
}

enum { ORC_OS = 0, ORC_RYS = 1, ORC_AUTO = 2 };

static void make_comp(const orc_basis *b, const orc_pair *ab, const orc_pair *cd, orc_comp *q)
{
    const orc_ao *A = &b->ao[ab->i], *B = &b->ao[ab->j], *C = &b->ao[cd->i], *D = &b->ao[cd->j];
    q->a[0] = A->lx; q->a[1] = A->ly; q->a[2] = A->lz;
    q->b[0] = B->lx; q->b[1] = B->ly; q->b[2] = B->lz;
    q->c[0] = C->lx; q->c[1] = C->ly; q->c[2] = C->lz;
    q->d[0] = D->lx; q->d[1] = D->ly; q->d[2] = D->lz;
}

/* contracted ERI over AO pairs (os.cpp:994-1010, rys.cpp:489-505, rys.cpp:222-236) */
static double contracted(const orc_basis *b, const orc_pair *ab, const orc_pair *cd, int engine)
{
    orc_comp q;
    make_comp(b, ab, cd, &q);
    int use_rys = engine == ORC_RYS || (engine == ORC_AUTO && auto_prefers_rys(&q));
    double eri = 0.0;
    for (int i = 0; i < ab->npp; ++i)
        for (int j = 0; j < cd->npp; ++j)
            eri += ab->pp[i].coeff_product * cd->pp[j].coeff_product *
                   (use_rys ? rys_primitive(&ab->pp[i], &cd->pp[j], &q, ab->R, cd->R)
                            : os_primitive(&ab->pp[i], &cd->pp[j], &q, ab->R, cd->R));
    return eri;
}

double orc_eri_pair(const orc_basis *b, int p, int q, int engine)
{
    return contracted(b, &b->pairs[p], &b->pairs[q], engine);
}

/* Schwarz table: os.cpp:1703-1752 for the OS engine; the Rys and auto
 * engines both use the all-Rys table of rys.cpp:509-556 (rys.cpp:569, 640).
 * Q is nb x nb, row-major here (symmetric). */
void orc_schwarz(const orc_basis *b, int engine, double *Q)
{
    const int nb = b->nbasis;
    memset(Q, 0, sizeof(double) * nb * nb);
    /* The reference runs this loop serially; every element is computed on
     * its own, so the threads change the time, not the values. */
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < b->npairs; ++p) {
        const orc_pair *sp = &b->pairs[p];
        const double diag = contracted(b, sp, sp, engine == ORC_OS ? ORC_OS : ORC_RYS);
        const double q = sqrt(fabs(diag));
        Q[sp->i * nb + sp->j] = q;
        Q[sp->j * nb + sp->i] = q;
    }
}

/* ------------------------------------------------------------------------ */
/* Tensor build with 8-fold scatter (os.cpp:137-163, 1755-1829) and its     */
/* digestion (os.cpp:1831-1876).  Row-major i*nb^3 + j*nb^2 + k*nb + l.     */
/* ------------------------------------------------------------------------ */
static void write_perm(double *eri, size_t nb, int i, int j, int k, int l, double v)
{
    const size_t nb2 = nb * nb, nb3 = nb2 * nb;
    eri[i * nb3 + j * nb2 + k * nb + l] = v;
    eri[j * nb3 + i * nb2 + k * nb + l] = v;
    eri[i * nb3 + j * nb2 + l * nb + k] = v;
    eri[j * nb3 + i * nb2 + l * nb + k] = v;
    eri[k * nb3 + l * nb2 + i * nb + j] = v;
    eri[l * nb3 + k * nb2 + i * nb + j] = v;
    eri[k * nb3 + l * nb2 + j * nb + i] = v;
    eri[l * nb3 + k * nb2 + j * nb + i] = v;
}

/* Fills the dense tensor; returns the number of screened-in AO quartets. */
long long orc_eri_tensor(const orc_basis *b, double tol, int engine, const double *Q, double *eri)
{
    const size_t nb = b->nbasis;
    memset(eri, 0, sizeof(double) * nb * nb * nb * nb);
    long long count = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : count)
    for (int p = 0; p < b->npairs; ++p) {
        const orc_pair *ab = &b->pairs[p];
        for (int q = p; q < b->npairs; ++q) {
            const orc_pair *cd = &b->pairs[q];
            if (Q[ab->i * nb + ab->j] * Q[cd->i * nb + cd->j] < tol)
                continue;
            ++count;
            write_perm(eri, nb, ab->i, ab->j, cd->i, cd->j, contracted(b, ab, cd, engine));
        }
    }
    return count;
}

/* G = J - K/2 from the dense tensor: os.cpp:1831-1847 (P, G row-major; the
 * reference's Eigen matrices are column-major but P and G are symmetric). */
void orc_fock_rhf_from_tensor(size_t nb, const double *eri, const double *P, double *G)
{
    const size_t nb2 = nb * nb, nb3 = nb2 * nb;
#pragma omp parallel for schedule(static)
    for (size_t mu = 0; mu < nb; ++mu)
        for (size_t nu = 0; nu < nb; ++nu) {
            double g = 0.0;
            for (size_t lam = 0; lam < nb; ++lam)
                for (size_t sig = 0; sig < nb; ++sig)
                    g += P[lam * nb + sig] *
                         (eri[mu * nb3 + nu * nb2 + lam * nb + sig] - 0.5 * eri[mu * nb3 + lam * nb2 + nu * nb + sig]);
            G[mu * nb + nu] = g;
        }
}

/* os.cpp:1849-1876 */
void orc_fock_uhf_from_tensor(size_t nb, const double *eri, const double *Pa, const double *Pb,
                              double *Ga, double *Gb)
{
    const size_t nb2 = nb * nb, nb3 = nb2 * nb;
#pragma omp parallel for schedule(static)
    for (size_t mu = 0; mu < nb; ++mu)
        for (size_t nu = 0; nu < nb; ++nu) {
            double ga = 0.0, gb = 0.0;
            for (size_t lam = 0; lam < nb; ++lam)
                for (size_t sig = 0; sig < nb; ++sig) {
                    const double c = eri[mu * nb3 + nu * nb2 + lam * nb + sig];
                    const double x = eri[mu * nb3 + lam * nb2 + nu * nb + sig];
                    const double pt = Pa[lam * nb + sig] + Pb[lam * nb + sig];
                    ga += pt * c - Pa[lam * nb + sig] * x;
                    gb += pt * c - Pb[lam * nb + sig] * x;
                }
            Ga[mu * nb + nu] = ga;
            Gb[mu * nb + nu] = gb;
        }
}

/* ------------------------------------------------------------------------ */
/* Streaming direct build (no nb^4 tensor): the same screened canonical AO   */
/* quartets and the same contracted integrals as os.cpp:1458-1507, digested  */
/* by visiting each DISTINCT permutation of the quartet once, which is what  */
/* the tensor scatter + O(nb^4) contraction (os.cpp:1512-1520) sums.  Used   */
/* for systems whose tensor does not fit and as the timed CPU baseline.      */
/* pair_begin/pair_end restrict the outer pair loop (a bounded sample).      */
/* J and K are accumulated separately: G_rhf = J - K/2; for UHF with         */
/* Pa, Pb: Ga = J(Pa+Pb) - K(Pa), Gb = J(Pa+Pb) - K(Pb).                    */
/* ------------------------------------------------------------------------ */
static long long jk_rows(const orc_basis *b, double tol, int engine, const double *Q, int nmat, const double *Pj,
                         const double *Pk, double *J, double *K, const int *rows, int nrows, int row_begin)
{
    const int nb = b->nbasis;
    const size_t nb2 = (size_t)nb * nb;
    long long count = 0;
    memset(J, 0, sizeof(double) * nb2);
    memset(K, 0, sizeof(double) * nb2 * nmat);
#pragma omp parallel reduction(+ : count)
    {
        double *Jl = calloc(nb2, sizeof(double));
        double *Kl = calloc(nb2 * nmat, sizeof(double));
#pragma omp for schedule(dynamic)
        for (int r = 0; r < nrows; ++r) {
            const int p = rows ? rows[r] : row_begin + r;
            const orc_pair *ab = &b->pairs[p];
            for (int q = p; q < b->npairs; ++q) {
                const orc_pair *cd = &b->pairs[q];
                if (Q[ab->i * nb + ab->j] * Q[cd->i * nb + cd->j] < tol)
                    continue;
                ++count;
                const double v = contracted(b, ab, cd, engine);
                const int i = ab->i, j = ab->j, k = cd->i, l = cd->j;
                int perm[8][4] = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                                  {k, l, i, j}, {l, k, i, j}, {k, l, j, i}, {l, k, j, i}};
                for (int a = 0; a < 8; ++a) {
                    int dup = 0;
                    for (int c = 0; c < a && !dup; ++c)
                        dup = perm[c][0] == perm[a][0] && perm[c][1] == perm[a][1] &&
                              perm[c][2] == perm[a][2] && perm[c][3] == perm[a][3];
                    if (dup)
                        continue;
                    const int m = perm[a][0], n = perm[a][1], rr = perm[a][2], s = perm[a][3];
                    /* (mn|rs): J(m,n) += P(r,s) v ; K(m,r) += P(n,s) v */
                    Jl[(size_t)m * nb + n] += Pj[(size_t)rr * nb + s] * v;
                    for (int t = 0; t < nmat; ++t)
                        Kl[t * nb2 + (size_t)m * nb + rr] += Pk[t * nb2 + (size_t)n * nb + s] * v;
                }
            }
        }
#pragma omp critical
        {
            for (size_t x = 0; x < nb2; ++x)
                J[x] += Jl[x];
            for (size_t x = 0; x < nb2 * nmat; ++x)
                K[x] += Kl[x];
        }
        free(Jl);
        free(Kl);
    }
    return count;
}

long long orc_jk_direct(const orc_basis *b, double tol, int engine, const double *Q,
                        int nmat, const double *Pj, const double *Pk, double *J, double *K,
                        int pair_begin, int pair_end)
{
    if (pair_end < 0 || pair_end > b->npairs)
        pair_end = b->npairs;
    if (pair_begin < 0)
        pair_begin = 0;
    return jk_rows(b, tol, engine, Q, nmat, Pj, Pk, J, K, NULL,
                   pair_end > pair_begin ? pair_end - pair_begin : 0, pair_begin);
}

/* The same over an explicit list of bra AO-pair rows (a bounded sample). */
long long orc_jk_direct_rows(const orc_basis *b, double tol, int engine, const double *Q,
                             int nmat, const double *Pj, const double *Pk, double *J, double *K,
                             const int *rows, int nrows)
{
    return jk_rows(b, tol, engine, Q, nmat, Pj, Pk, J, K, rows, nrows, 0);
}

/* Index of AO pair (i, j) in the upper-triangle row-major pair order. */
static inline int pair_index(int nb, int i, int j)
{
    if (i > j) {
        const int t = i;
        i = j;
        j = t;
    }
    return i * (2 * nb - i + 1) / 2 + (j - i);
}

/* Selected elements G(m, n) of the RHF two-electron matrix, straight from
 * its definition over the full index range, G = J - K/2 with
 * J(m,n) = sum_{r,s} (mn|rs) P(r,s) and K(m,n) = sum_{r,s} (mr|ns) P(r,s)
 * (the contraction of os.cpp:1512-1520), each integral dropped when its
 * canonical quartet fails the Schwarz test (os.cpp:1475; the test is
 * invariant under the 8-fold permutations).  Costs O(nb^2) integrals per
 * element, so it checks single elements of systems whose full build is far
 * too slow for the oracle.  elems holds (m, n) pairs. */
void orc_fock_elements(const orc_basis *b, double tol, int engine, const double *Q, const double *P,
                       const int *elems, int nelem, double *out)
{
    const int nb = b->nbasis;
    for (int e = 0; e < nelem; ++e) {
        const int m = elems[2 * e], n = elems[2 * e + 1];
        const orc_pair *mn = &b->pairs[pair_index(nb, m, n)];
        const double qmn = Q[m * nb + n];
        double J = 0.0, K = 0.0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : J, K)
        for (int r = 0; r < nb; ++r) {
            /* J: (mn|rs) = (mn|sr) and P is symmetric, so s >= r with weight 2 off the diagonal */
            for (int s = r; s < nb; ++s) {
                if (qmn * Q[r * nb + s] < tol)
                    continue;
                const double v = contracted(b, mn, &b->pairs[pair_index(nb, r, s)], engine);
                J += (s == r ? 1.0 : 2.0) * v * P[r * nb + s];
            }
            /* K: (mr|ns) for every s */
            const double qmr = Q[m * nb + r];
            const orc_pair *mr = &b->pairs[pair_index(nb, m, r)];
            for (int s = 0; s < nb; ++s) {
                if (qmr * Q[n * nb + s] < tol)
                    continue;
                K += contracted(b, mr, &b->pairs[pair_index(nb, n, s)], engine) * P[r * nb + s];
            }
        }
        out[e] = J - 0.5 * K;
    }
}

/* The contracted Cartesian block of one shell quartet (sa sb|sc sd) without
 * screening: out[((ia*NB + ib)*NC + ic)*ND + id] = (i j|k l) for the AOs of the
 * four shells in the reference's component order, each from the per-component
 * contraction of os.cpp:994-1010 / rys.cpp:489-505. */
void orc_shell_block(const orc_basis *b, int sa, int sb, int sc, int sd, int engine, double *out)
{
    const int nb = b->nbasis;
    const int sh[4] = {sa, sb, sc, sd};
    int first[4], n[4];
    for (int q = 0; q < 4; ++q) {
        first[q] = -1;
        for (int k = 0; k < nb && first[q] < 0; ++k)
            if (b->ao[k].shell == sh[q])
                first[q] = k;
        n[q] = (b->L[sh[q]] + 1) * (b->L[sh[q]] + 2) / 2;
    }
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int ia = 0; ia < n[0]; ++ia)
        for (int ib = 0; ib < n[1]; ++ib) {
            const orc_pair *ab = &b->pairs[pair_index(nb, first[0] + ia, first[1] + ib)];
            for (int ic = 0; ic < n[2]; ++ic)
                for (int id = 0; id < n[3]; ++id) {
                    const orc_pair *cd = &b->pairs[pair_index(nb, first[2] + ic, first[3] + id)];
                    out[((ia * n[1] + ib) * n[2] + ic) * n[3] + id] = contracted(b, ab, cd, engine);
                }
        }
}

/* Number of screened canonical AO quartets in bra row p (q >= p). */
long long orc_row_count(const orc_basis *b, double tol, const double *Q, int p)
{
    const int nb = b->nbasis;
    const orc_pair *ab = &b->pairs[p];
    const double qa = Q[ab->i * nb + ab->j];
    long long c = 0;
    for (int q = p; q < b->npairs; ++q) {
        const orc_pair *cd = &b->pairs[q];
        c += !(qa * Q[cd->i * nb + cd->j] < tol);
    }
    return c;
}

/* ------------------------------------------------------------------------ */
/* Screened canonical AO quartet list (os.cpp:1458-1476): count, an order-   */
/* independent 64-bit digest of the set, and (optionally) the list itself.   */
/* ------------------------------------------------------------------------ */
static inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

uint64_t orc_quartet_code(int i, int j, int k, int l)
{
    return ((uint64_t)i << 48) | ((uint64_t)j << 32) | ((uint64_t)k << 16) | (uint64_t)l;
}

long long orc_quartet_list(const orc_basis *b, double tol, const double *Q, uint64_t *digest,
                           int *out, long long out_cap)
{
    const int nb = b->nbasis;
    long long count = 0;
    uint64_t h = 0;
    if (!out) {
        /* count and digest only: the digest is a sum of per-quartet hashes,
         * so threads over the bra pairs give the serial loop's exact result;
         * the pairs' Q values and codes are gathered into arrays first */
        const int np = b->npairs;
        double *qv = (double *)malloc(sizeof(double) * (size_t)(np > 0 ? np : 1));
        uint64_t *code = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(np > 0 ? np : 1));
        for (int p = 0; p < np; ++p) {
            qv[p] = Q[b->pairs[p].i * nb + b->pairs[p].j];
            code[p] = orc_quartet_code(b->pairs[p].i, b->pairs[p].j, 0, 0);
        }
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : count, h)
        for (int p = 0; p < np; ++p) {
            const double qab = qv[p];
            const uint64_t cab = code[p];
            for (int q = p; q < np; ++q) {
                if (qab * qv[q] < tol)
                    continue;
                h += mix64(cab | (code[q] >> 32));
                ++count;
            }
        }
        free(qv);
        free(code);
        *digest = h;
        return count;
    }
    for (int p = 0; p < b->npairs; ++p) {
        const orc_pair *ab = &b->pairs[p];
        for (int q = p; q < b->npairs; ++q) {
            const orc_pair *cd = &b->pairs[q];
            if (Q[ab->i * nb + ab->j] * Q[cd->i * nb + cd->j] < tol)
                continue;
            h += mix64(orc_quartet_code(ab->i, ab->j, cd->i, cd->j));
            if (out && count < out_cap) {
                out[4 * count] = ab->i;
                out[4 * count + 1] = ab->j;
                out[4 * count + 2] = cd->i;
                out[4 * count + 3] = cd->j;
            }
            ++count;
        }
    }
    *digest = h;
    return count;
}

/* ------------------------------------------------------------------------ */
/* One-electron integrals (host-side in the reference and here; used by the  */
/* oracle SCF only): os.cpp:253-292 (_os_1d), 294-393 (S, T), 460-602 (V).   */
/* ------------------------------------------------------------------------ */
static double os_1d(double gamma, double PA, double PB, int lA, int lB)
{
    double S[9][9];
    memset(S, 0, sizeof S);
    S[0][0] = 1.0;
    for (int i = 1; i <= lA; i++) {
        S[i][0] = PA * S[i - 1][0];
        if (i > 1)
            S[i][0] = (i - 1) * gamma * S[i - 2][0] + S[i][0];
    }
    for (int j = 1; j <= lB; j++) {
        S[0][j] = PB * S[0][j - 1];
        if (j > 1)
            S[0][j] = (j - 1) * gamma * S[0][j - 2] + S[0][j];
    }
    for (int i = 1; i <= lA; i++)
        for (int j = 1; j <= lB; j++) {
            S[i][j] = PA * S[i - 1][j] + j * gamma * S[i - 1][j - 1];
            if (i > 1)
                S[i][j] += (i - 1) * gamma * S[i - 2][j];
        }
    return S[lA][lB];
}

static double nuclear_primitive(const orc_pp *pp, const orc_ao *A, const orc_ao *B,
                                const double *AB, const double *C)
{
    const int L = A->lx + A->ly + A->lz + B->lx + B->ly + B->lz;
    const double pCx = pp->P[0] - C[0], pCy = pp->P[1] - C[1], pCz = pp->P[2] - C[2];
    const double T = pp->zeta * (pCx * pCx + pCy * pCy + pCz * pCz);
    const double nuc_pref = pp->prefactor * 2.0 * sqrt(pp->zeta / ORC_PI);
    enum { MM = 2 * 6 + 2 };
    static _Thread_local double Vn[VD][VD][VD][MM];
    memset(Vn, 0, sizeof Vn);
    for (int m = 0; m <= L; m++)
        Vn[0][0][0][m] = nuc_pref * orc_boys(m, T);
    const double pAx = pp->pA[0], pAy = pp->pA[1], pAz = pp->pA[2];
    const double hiz = pp->inv_zeta * 0.5;
    const int lxm = A->lx + B->lx, lym = A->ly + B->ly, lzm = A->lz + B->lz;
    for (int ix = 1; ix <= lxm; ix++)
        for (int m = 0; m <= L - ix; m++) {
            Vn[ix][0][0][m] = pAx * Vn[ix - 1][0][0][m] - pCx * Vn[ix - 1][0][0][m + 1];
            if (ix > 1)
                Vn[ix][0][0][m] += (ix - 1) * hiz * (Vn[ix - 2][0][0][m] - Vn[ix - 2][0][0][m + 1]);
        }
    for (int ix = 0; ix <= lxm; ix++)
        for (int iy = 1; iy <= lym; iy++) {
            const int mm = L - ix - iy;
            if (mm < 0)
                continue;
            for (int m = 0; m <= mm; m++) {
                Vn[ix][iy][0][m] = pAy * Vn[ix][iy - 1][0][m] - pCy * Vn[ix][iy - 1][0][m + 1];
                if (iy > 1)
                    Vn[ix][iy][0][m] += (iy - 1) * hiz * (Vn[ix][iy - 2][0][m] - Vn[ix][iy - 2][0][m + 1]);
            }
        }
    for (int ix = 0; ix <= lxm; ix++)
        for (int iy = 0; iy <= lym; iy++)
            for (int iz = 1; iz <= lzm; iz++) {
                const int mm = L - ix - iy - iz;
                if (mm < 0)
                    continue;
                for (int m = 0; m <= mm; m++) {
                    Vn[ix][iy][iz][m] = pAz * Vn[ix][iy][iz - 1][m] - pCz * Vn[ix][iy][iz - 1][m + 1];
                    if (iz > 1)
                        Vn[ix][iy][iz][m] += (iz - 1) * hiz * (Vn[ix][iy][iz - 2][m] - Vn[ix][iy][iz - 2][m + 1]);
                }
            }
    double V0[VD][VD][VD];
    memset(V0, 0, sizeof V0);
    for (int ix = 0; ix <= lxm; ix++)
        for (int iy = 0; iy <= lym; iy++)
            for (int iz = 0; iz <= lzm; iz++)
                V0[ix][iy][iz] = Vn[ix][iy][iz][0];
    return nuclear_hrr(V0, A->lx, A->ly, A->lz, B->lx, B->ly, B->lz, AB[0], AB[1], AB[2]);
}

/* S, T, V (row-major nb x nb).  charges: natom x (x, y, z, Z) in Bohr. */
void orc_one_electron(const orc_basis *b, int natom, const double *charges, double *S, double *T, double *Vm)
{
    const int nb = b->nbasis;
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < b->npairs; ++p) {
        const orc_pair *sp = &b->pairs[p];
        const orc_ao *A = &b->ao[sp->i], *B = &b->ao[sp->j];
        const int ca[3] = {A->lx, A->ly, A->lz}, cb[3] = {B->lx, B->ly, B->lz};
        double s = 0.0, t = 0.0;
        for (int k = 0; k < sp->npp; ++k) {
            const orc_pp *pp = &sp->pp[k];
            const double hiz = pp->inv_zeta * 0.5;
            const double beta = pp->beta, beta2 = beta * beta;
            const double scale = pp->prefactor * pp->coeff_product;
            double Sd[3], Sp[3], Sm[3], Td[3];
            for (int d = 0; d < 3; ++d) {
                Sd[d] = os_1d(hiz, pp->pA[d], pp->pB[d], ca[d], cb[d]);
                Sp[d] = os_1d(hiz, pp->pA[d], pp->pB[d], ca[d], cb[d] + 2);
                Sm[d] = cb[d] >= 2 ? os_1d(hiz, pp->pA[d], pp->pB[d], ca[d], cb[d] - 2) : 0.0;
                Td[d] = -0.5 * cb[d] * (cb[d] - 1) * Sm[d] + beta * (2 * cb[d] + 1) * Sd[d] - 2.0 * beta2 * Sp[d];
            }
            s += Sd[0] * Sd[1] * Sd[2] * scale;
            t += (Td[0] * Sd[1] * Sd[2] + Sd[0] * Td[1] * Sd[2] + Sd[0] * Sd[1] * Td[2]) * scale;
        }
        double v = 0.0;
        for (int c = 0; c < natom; ++c) {
            double vp = 0.0;
            for (int k = 0; k < sp->npp; ++k)
                vp += nuclear_primitive(&sp->pp[k], A, B, sp->R, &charges[4 * c]) * sp->pp[k].coeff_product;
            v -= charges[4 * c + 3] * vp;
        }
        S[sp->i * nb + sp->j] = S[sp->j * nb + sp->i] = s;
        T[sp->i * nb + sp->j] = T[sp->j * nb + sp->i] = t;
        Vm[sp->i * nb + sp->j] = Vm[sp->j * nb + sp->i] = v;
    }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
