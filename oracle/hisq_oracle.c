/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — plain-C restatement of the KuQCD HISQ even-odd dslash and multishift CG.
 * Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker; never by the product.
 *
 * Each function names the reference lines it restates.  The dslash keeps the reference's order of floating-point
 * operations (spinor scaled first, row sums from column 0, forward hops then backward hops, fat before Naik), so
 * with FMA contraction off it reproduces the reference's double- and single-precision results bit for bit; the
 * tests check that against oracle/_ref/libkuqcd_ref.so.
 */
#include "hisq_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- geometry (index_utils.cpp:17-33,91-111) */
typedef struct {
    int n[4];  /* nx ny nz nt */
    int hx;    /* nx / 2 */
    long vh;   /* V / 2 */
} geom_t;

static geom_t mkgeom(const int d[4])
{
    geom_t g;
    for (int i = 0; i < 4; ++i) g.n[i] = d[i];
    g.hx = d[0] / 2;
    g.vh = (long)d[0] * d[1] * d[2] * d[3] / 2;
    return g;
}

/* checkerboard index -> full coordinates for the given parity (GetPosition + GetPosFromCBPos) */
static void cb_coords(const geom_t *g, long i, int parity, int c[4])
{
    long r = i / g->hx;
    int xcb = (int)(i - r * g->hx);
    c[1] = (int)(r % g->n[1]);
    r /= g->n[1];
    c[2] = (int)(r % g->n[2]);
    c[3] = (int)(r / g->n[2]);
    c[0] = 2 * xcb + ((c[1] + c[2] + c[3] + parity) & 1);
}

/* checkerboard index of full coordinates (GetCBPos + Position::Index over latSubBulkCB) */
static long cb_index(const geom_t *g, const int c[4])
{
    return (long)(c[0] >> 1) + (long)g->hx * (c[1] + (long)g->n[1] * (c[2] + (long)g->n[2] * c[3]));
}

/* periodic wrap, Position::Normalize (space_time.cpp:187-197) */
static int wrap(int v, int n)
{
    v %= n;
    if (v < 0) v += n;
    return v;
}

static long nbr(const geom_t *g, const int c[4], int dir, int hop)
{
    int d[4] = {c[0], c[1], c[2], c[3]};
    d[dir] = wrap(d[dir] + hop, g->n[dir]);
    return cb_index(g, d);
}

/* ---------------------------------------------------------------- dslash (dirac_hisq.cpp:409-502) */
/* U v and U^dag v with the accumulation order of kuqcd_math.cpp:20-35 and :91-106; the result is added to
 * (sign = +1) or subtracted from (sign = -1) acc, as ColorSpinor::operator+= / -= do. */
#define KQO_DSLASH_BODY(T)                                                                                       \
    {                                                                                                            \
        const geom_t g = mkgeom(dims);                                                                           \
        const int q = 1 - dst_parity;                                                                            \
        const long fwd_off = dst_parity == 0 ? 0 : g.vh; /* gauge row of the output site */                   \
        const long bwd_off = dst_parity == 0 ? g.vh : 0; /* gauge row of a neighbour on the other parity */     \
        const T half = (T)0.5;                                                                                   \
        const T c3 = (T)(-1.0 / 48.0);                                                                           \
        for (long i = 0; i < g.vh; ++i) {                                                                        \
            int c[4];                                                                                            \
            cb_coords(&g, i, dst_parity, c);                                                                     \
            T acc[6] = {0, 0, 0, 0, 0, 0};                                                                       \
            for (int pass = 0; pass < 2; ++pass) {                                                               \
                for (int dir = 0; dir < 4; ++dir) {                                                              \
                    for (int naik = 0; naik < 2; ++naik) {                                                       \
                        const int hop = (naik ? 3 : 1) * (pass == 0 ? 1 : -1);                                   \
                        const long ni = nbr(&g, c, dir, hop);                                                    \
                        const T *u = (naik ? lng : fat) +                                                        \
                                     18 * (dir + 4 * (pass == 0 ? (fwd_off + i) : (bwd_off + ni)));              \
                        const T s = naik ? c3 : half;                                                            \
                        T v[6];                                                                                  \
                        for (int k = 0; k < 6; ++k) v[k] = src[6 * ni + k] * s;                                  \
                        (void)q;                                                                                 \
                        for (int r = 0; r < 3; ++r) {                                                            \
                            T re = 0, im = 0;                                                                    \
                            for (int col = 0; col < 3; ++col) {                                                  \
                                const int l = pass == 0 ? (col + 3 * r) : (r + 3 * col);                         \
                                const T ur = u[2 * l], ui = u[2 * l + 1];                                        \
                                const T vr = v[2 * col], vi = v[2 * col + 1];                                    \
                                if (pass == 0) {                                                                 \
                                    re += ur * vr - ui * vi;                                                     \
                                    im += ur * vi + ui * vr;                                                     \
                                } else {                                                                         \
                                    re += ur * vr + ui * vi;                                                     \
                                    im += ur * vi - ui * vr;                                                     \
                                }                                                                                \
                            }                                                                                    \
                            if (pass == 0) {                                                                     \
                                acc[2 * r] += re;                                                                \
                                acc[2 * r + 1] += im;                                                            \
                            } else {                                                                             \
                                acc[2 * r] -= re;                                                                \
                                acc[2 * r + 1] -= im;                                                            \
                            }                                                                                    \
                        }                                                                                        \
                    }                                                                                            \
                }                                                                                                \
            }                                                                                                    \
            for (int k = 0; k < 6; ++k) dst[6 * i + k] = acc[k];                                                 \
        }                                                                                                        \
    }

void kqo_dslash_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst,
                  int dst_parity) KQO_DSLASH_BODY(double)

void kqo_dslash_f(const int dims[4], const float *fat, const float *lng, const float *src, float *dst,
                  int dst_parity) KQO_DSLASH_BODY(float)

/* The non-PC operator of dirac_hisq.cpp:409-455 with diracType KUQCD_HISQ_DIRAC on KUQCD_ALL fields: offseti =
 * offsetg = 0 and the neighbour tables of dirac_hisq.cpp:128-136 point even sites at the odd half (index + Vh) and
 * odd sites at the even half, so each half of dst is the even-odd dslash of the other half of src. */
void kqo_dslash_full_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst)
{
    const long n = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2 * 6;
    kqo_dslash_d(dims, fat, lng, src + n, dst, 0);
    kqo_dslash_d(dims, fat, lng, src, dst + n, 1);
}

void kqo_mdaggm_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst,
                  double *tmp, int parity)
{
    kqo_dslash_d(dims, fat, lng, src, tmp, 1 - parity);
    kqo_dslash_d(dims, fat, lng, tmp, dst, parity);
}

static void mdaggm_f(const int dims[4], const float *fat, const float *lng, const float *src, float *dst, float *tmp,
                     int parity)
{
    kqo_dslash_f(dims, fat, lng, src, tmp, 1 - parity);
    kqo_dslash_f(dims, fat, lng, tmp, dst, parity);
}

/* ---------------------------------------------------------------- multishift CG (inverter_cgm.cpp:17-87) */
/* BLAS-1 of spinor_field.cpp:130-252, sequential sums */
#define KQO_CGM_BODY(T, MDAGGM)                                                                                  \
    {                                                                                                            \
        const geom_t g = mkgeom(dims);                                                                           \
        const long n = g.vh * 6;                                                                                 \
        const int ns = num_shift;                                                                                \
        T *a = (T *)malloc(sizeof(T) * ns), *B = (T *)malloc(sizeof(T) * ns);                                    \
        T *Z = (T *)malloc(sizeof(T) * ns), *Zm1 = (T *)malloc(sizeof(T) * ns);                                  \
        T **p = (T **)malloc(sizeof(T *) * ns);                                                                  \
        T *s = (T *)malloc(sizeof(T) * n), *r = (T *)malloc(sizeof(T) * n), *tmp = (T *)malloc(sizeof(T) * n);   \
        for (int k = 0; k < ns; ++k) {                                                                           \
            p[k] = (T *)malloc(sizeof(T) * n);                                                                   \
            memcpy(p[k], b, sizeof(T) * n);                                                                      \
            a[k] = 0;                                                                                            \
            B[k] = 1;                                                                                            \
            Z[k] = 1;                                                                                            \
            Zm1[k] = 1;                                                                                          \
            memset(x[k], 0, sizeof(T) * n);                                                                      \
        }                                                                                                        \
        memcpy(r, b, sizeof(T) * n);                                                                             \
        T rNorm2 = 0;                                                                                            \
        for (long e = 0; e < n; ++e) rNorm2 += r[e] * r[e];                                                      \
        T pAp, lambda, lambda2, rr1, Bm1 = 1;                                                                    \
        int maxTerm = ns, iter = 0;                                                                              \
        do {                                                                                                     \
            iter++;                                                                                              \
            MDAGGM(dims, fat, lng, p[0], s, tmp, parity);                                                        \
            for (long e = 0; e < n; ++e) s[e] = shifts[0] * p[0][e] - s[e];                                      \
            pAp = 0;                                                                                             \
            for (long e = 0; e < n; ++e) pAp += p[0][e] * s[e];                                                  \
            B[0] = -rNorm2 / pAp;                                                                                \
            for (long e = 0; e < n; ++e) r[e] += B[0] * s[e];                                                    \
            for (int j = 1; j < maxTerm; ++j) {                                                                  \
                rr1 = Bm1 * Zm1[j] /                                                                             \
                      (B[0] * a[0] * (Zm1[j] - Z[j]) + Zm1[j] * Bm1 * (1.0 - shifts[j] * B[0]));                 \
                Zm1[j] = Z[j];                                                                                   \
                Z[j] = Z[j] * rr1;                                                                               \
                B[j] = B[0] * rr1;                                                                               \
            }                                                                                                    \
            Bm1 = B[0];                                                                                          \
            lambda2 = 0;                                                                                         \
            for (long e = 0; e < n; ++e) lambda2 += r[e] * r[e];                                                 \
            a[0] = lambda2 / rNorm2;                                                                             \
            rNorm2 = lambda2;                                                                                    \
            for (int k = 0; k < maxTerm; ++k)                                                                    \
                for (long e = 0; e < n; ++e) x[k][e] -= B[k] * p[k][e];                                          \
            for (int j = 1; j < maxTerm; ++j) a[j] = a[0] * Z[j] * B[j] / (Zm1[j] * B[0]);                       \
            for (int k = 0; k < maxTerm; ++k)                                                                    \
                for (long e = 0; e < n; ++e) p[k][e] = Z[k] * r[e] + a[k] * p[k][e];                             \
            do {                                                                                                 \
                lambda = Z[maxTerm - 1] * Z[maxTerm - 1] * lambda2;                                              \
                if (lambda < tol) maxTerm--;                                                                     \
            } while ((maxTerm > 0) && (lambda < tol));                                                           \
        } while ((maxTerm > 0) && (iter < max_iter));                                                            \
        for (int k = 0; k < ns; ++k) free(p[k]);                                                                 \
        free(p);                                                                                                 \
        free(s);                                                                                                 \
        free(r);                                                                                                 \
        free(tmp);                                                                                               \
        free(a);                                                                                                 \
        free(B);                                                                                                 \
        free(Z);                                                                                                 \
        free(Zm1);                                                                                               \
        return iter;                                                                                             \
    }

int kqo_cgm_d(const int dims[4], const double *fat, const double *lng, int parity, int num_shift,
              const double *shifts, const double *b, double **x, double tol, int max_iter)
    KQO_CGM_BODY(double, kqo_mdaggm_d)

int kqo_cgm_f(const int dims[4], const float *fat, const float *lng, int parity, int num_shift,
              const float *shifts, const float *b, float **x, double tol, int max_iter)
    KQO_CGM_BODY(float, mdaggm_f)

double kqo_true_residual_d(const int dims[4], const double *fat, const double *lng, int parity, double sigma,
                           const double *b, const double *x)
{
    const geom_t g = mkgeom(dims);
    const long n = g.vh * 6;
    double *s = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
    kqo_mdaggm_d(dims, fat, lng, x, s, t, parity);
    double rr = 0, bb = 0;
    for (long e = 0; e < n; ++e) {
        const double res = b[e] - (sigma * x[e] - s[e]);
        rr += res * res;
        bb += b[e] * b[e];
    }
    free(s);
    free(t);
    return sqrt(rr / bb);
}

/* ---------------------------------------------------------------- field construction */
/* counter-based generator: a splitmix64-style finaliser applied to seed and counter */
uint64_t kqo_hash(uint64_t seed, uint64_t counter)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (counter + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    z += seed ^ 0xD1B54A32D192ED03ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* uniform in (0, 1] */
static double unif(uint64_t seed, uint64_t counter)
{
    return (double)((kqo_hash(seed, counter) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

/* Box-Muller pair of standard normals from counters (2k, 2k+1) */
static void gauss2(uint64_t seed, uint64_t k, double *n0, double *n1)
{
    const double u1 = unif(seed, 2 * k), u2 = unif(seed, 2 * k + 1);
    const double rad = sqrt(-2.0 * log(u1));
    const double th = 6.283185307179586476925 * u2;
    *n0 = rad * cos(th);
    *n1 = rad * sin(th);
}

/* complex 3x3 helpers, interleaved re/im, row-major l = col + 3*row */
static void cmul33(const double *A, const double *B, double *C)
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double re = 0, im = 0;
            for (int k = 0; k < 3; ++k) {
                const double ar = A[2 * (k + 3 * r)], ai = A[2 * (k + 3 * r) + 1];
                const double br = B[2 * (c + 3 * k)], bi = B[2 * (c + 3 * k) + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            C[2 * (c + 3 * r)] = re;
            C[2 * (c + 3 * r) + 1] = im;
        }
}

/* U = exp(i eps H) by scaling and squaring of a degree-16 Taylor series (H Hermitian, so U is unitary). */
void kqo_su3_exp_iH(const double *H, double eps, double *U)
{
    double X[18];
    double nrm = 0;
    for (int l = 0; l < 9; ++l) { /* X = i eps H */
        X[2 * l] = -eps * H[2 * l + 1];
        X[2 * l + 1] = eps * H[2 * l];
        nrm += X[2 * l] * X[2 * l] + X[2 * l + 1] * X[2 * l + 1];
    }
    nrm = sqrt(nrm);
    int sq = 0;
    while (nrm > 0.25) {
        nrm *= 0.5;
        ++sq;
    }
    const double scale = ldexp(1.0, -sq);
    for (int l = 0; l < 18; ++l) X[l] *= scale;
    /* Horner: U = I + X(I + X/2(I + X/3(... (I + X/16)))) */
    double P[18], T[18];
    memset(P, 0, sizeof(P));
    P[0] = P[8] = P[16] = 1.0;
    for (int k = 16; k >= 1; --k) {
        cmul33(X, P, T);
        for (int l = 0; l < 18; ++l) P[l] = T[l] / (double)k;
        P[0] += 1.0;
        P[8] += 1.0;
        P[16] += 1.0;
    }
    for (int s = 0; s < sq; ++s) {
        cmul33(P, P, T);
        memcpy(P, T, sizeof(P));
    }
    memcpy(U, P, sizeof(P));
}

/* traceless Hermitian H = (A + A^dag)/2 - tr/3, A with N(0,1) re and im parts; 9 Gaussian pairs per link */
static void make_H(uint64_t seed, uint64_t link, double *H)
{
    double A[18];
    for (int k = 0; k < 9; ++k) gauss2(seed, 9 * link + k, &A[2 * k], &A[2 * k + 1]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            H[2 * (c + 3 * r)] = 0.5 * (A[2 * (c + 3 * r)] + A[2 * (r + 3 * c)]);
            H[2 * (c + 3 * r) + 1] = 0.5 * (A[2 * (c + 3 * r) + 1] - A[2 * (r + 3 * c) + 1]);
        }
    const double tr = (H[0] + H[8] + H[16]) / 3.0;
    H[0] -= tr;
    H[8] -= tr;
    H[16] -= tr;
}

/* even-odd site index of full coordinates: even sites first (kuqcd.cpp:103-127 with myIdx of latt_base.cpp) */
static long eo_index(const geom_t *g, const int c[4])
{
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    return cb_index(g, c) + (par ? g->vh : 0);
}

/* link counter: lexicographic site x + nx*(y + ny*(z + nz*t)), times 4, plus mu */
static uint64_t link_id(const geom_t *g, const int c[4], int mu)
{
    const uint64_t lex = (uint64_t)c[0] + (uint64_t)g->n[0] * (c[1] + (uint64_t)g->n[1] * (c[2] + (uint64_t)g->n[2] * c[3]));
    return 4 * lex + (uint64_t)mu;
}

static void thin_link(const geom_t *g, double eps, uint64_t seed, const int c[4], int mu, double *U)
{
    double H[18];
    make_H(seed, link_id(g, c, mu), H);
    kqo_su3_exp_iH(H, eps, U);
}

static int eta(const int c[4], int mu)
{
    int s = 0;
    for (int k = 0; k < mu; ++k) s += c[k];
    return (s & 1) ? -1 : 1;
}

void kqo_make_links(const int dims[4], double eps, uint64_t seed, double *fat, double *lng, double *thin)
{
    const geom_t g = mkgeom(dims);
    const long V = 2 * g.vh;
#pragma omp parallel for schedule(static)
    for (long lex = 0; lex < V; ++lex) {
        int c[4];
        long r = lex;
        c[0] = (int)(r % g.n[0]);
        r /= g.n[0];
        c[1] = (int)(r % g.n[1]);
        r /= g.n[1];
        c[2] = (int)(r % g.n[2]);
        c[3] = (int)(r / g.n[2]);
        const long site = eo_index(&g, c);
        for (int mu = 0; mu < 4; ++mu) {
            double U0[18], U1[18], U2[18], T[18], L[18];
            thin_link(&g, eps, seed, c, mu, U0);
            int c1[4] = {c[0], c[1], c[2], c[3]}, c2[4] = {c[0], c[1], c[2], c[3]};
            c1[mu] = wrap(c[mu] + 1, g.n[mu]);
            c2[mu] = wrap(c[mu] + 2, g.n[mu]);
            thin_link(&g, eps, seed, c1, mu, U1);
            thin_link(&g, eps, seed, c2, mu, U2);
            cmul33(U0, U1, T);
            cmul33(T, U2, L);
            const double e = (double)eta(c, mu);
            double *F = fat + 18 * (mu + 4 * site);
            double *N = lng + 18 * (mu + 4 * site);
            for (int l = 0; l < 18; ++l) {
                F[l] = (9.0 / 8.0) * e * U0[l];
                N[l] = (-1.0 / 24.0) * e * L[l];
            }
            if (thin) memcpy(thin + 18 * (mu + 4 * site), U0, sizeof(U0));
        }
    }
}

void kqo_make_source(const int dims[4], int parity, uint64_t seed, double *b)
{
    const geom_t g = mkgeom(dims);
    const uint64_t sseed = seed ^ 0x50C3A1E5D00DF00Dull;
    for (long i = 0; i < g.vh; ++i) {
        int c[4];
        cb_coords(&g, i, parity, c);
        const uint64_t lex =
            (uint64_t)c[0] + (uint64_t)g.n[0] * (c[1] + (uint64_t)g.n[1] * (c[2] + (uint64_t)g.n[2] * c[3]));
        for (int k = 0; k < 3; ++k) gauss2(sseed, 3 * lex + k, &b[6 * i + 2 * k], &b[6 * i + 2 * k + 1]);
    }
}
