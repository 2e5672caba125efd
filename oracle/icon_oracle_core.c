/*
 * icon_oracle_core.c -- CPU restatement of the ICON-GPU NUFFT and solver.
 *
 * TEST INFRASTRUCTURE ONLY (see icon_oracle.h).  Compiled twice:
 *   -DREAL=double -DSFX=_f64   FP64 oracle
 *   -DREAL=float  -DSFX=_f32   float oracle, rounding like the reference
 *                              (products rounded to float, fused multiply-adds
 *                              where nvcc contracts them), except that the FFT
 *                              is this file's radix-2 FFT instead of cuFFT.
 * Reference paths below are relative to
 * tomography/ICON_GPU_v1.2.9/sourceCode/ICON-GPU/ (NU = nufft_gpu_v8.cu).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "icon_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#define SFX _f64
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

#define IS_F32 (sizeof(REAL) == sizeof(float))
#define REF_PI 3.1415926535898

/* Multiply-add as the reference's device code computes it: nvcc contracts
 * "acc += a*b" into one fused multiply-add in float. */
static inline REAL madd(REAL a, REAL b, REAL acc)
{
    if (IS_F32) return (REAL)fmaf((float)a, (float)b, (float)acc);
    return a * b + acc;
}

typedef struct {
    int nx, nz, N0, N1, n0, n1, M;
    float th0, th1, b0, bf0, b1, bf1;
    int window;         /* ORA_WINDOW_GAUSS6 (the reference's) or ORA_WINDOW_KB4 */
    double kb0, kb1;    /* Kaiser-Bessel shape b = pi (2 - 1/theta) per dimension */
    float *xy;          /* [M][2] node coordinates (px2D)          */
    float *w;           /* [M] density weights (Weight)            */
    REAL *phix, *phiy;  /* [M][14] window values per tap           */
    int *ix, *iy;       /* [M][14] wrapped grid indices per tap    */
    REAL *cx, *cy;      /* [N0], [N1] deapodisation factors        */
    REAL *phi1;         /* [nx][14] 1-D row-transform window       */
    int *i1;            /* [nx][14]                                */
    REAL *tw0, *tw1;    /* FFT twiddles for n0 and n1              */
    int *br0, *br1;     /* bit reversal tables                     */
} ora_plan;

/* ---------------------------------------------------------------- FFT ---- */
/* Iterative radix-2 complex FFT, unnormalised, sign -1 forward (e^{-2 pi i}).
 * Twiddles are evaluated in double and rounded to REAL once. */
static REAL *make_twiddles(int n)
{
    REAL *t = (REAL *)malloc(sizeof(REAL) * (size_t)n);   /* n/2 complex */
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        t[2 * k] = (REAL)cos(a);
        t[2 * k + 1] = (REAL)sin(a);
    }
    return t;
}

static int *make_bitrev(int n)
{
    int *r = (int *)malloc(sizeof(int) * (size_t)n);
    int lg = 0;
    while ((1 << lg) < n) lg++;
    for (int i = 0; i < n; i++) {
        int v = 0;
        for (int b = 0; b < lg; b++)
            if (i & (1 << b)) v |= 1 << (lg - 1 - b);
        r[i] = v;
    }
    return r;
}

/* In-place FFT of n complex values at a (contiguous, interleaved). */
static void fft1(REAL *a, int n, const REAL *tw, const int *br, int inverse)
{
    for (int i = 0; i < n; i++) {
        int j = br[i];
        if (j > i) {
            REAL t0 = a[2 * i], t1 = a[2 * i + 1];
            a[2 * i] = a[2 * j];
            a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = t0;
            a[2 * j + 1] = t1;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; k++) {
                REAL wr = tw[2 * (k * step)];
                REAL wi = tw[2 * (k * step) + 1];
                if (inverse) wi = -wi;
                REAL *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
                REAL vr = v[0] * wr - v[1] * wi;
                REAL vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr;
                v[1] = u[1] - vi;
                u[0] = u[0] + vr;
                u[1] = u[1] + vi;
            }
        }
    }
}

/* 2-D FFT of an n0 x n1 grid, row-major with the n1 index fastest (the layout
 * of the reference's grid, NU:763-764), as cufftPlan2d(n0, n1) computes. */
static void fft2(const ora_plan *p, REAL *g, int inverse, REAL *col)
{
    for (int x = 0; x < p->n0; x++)
        fft1(g + 2 * (size_t)x * p->n1, p->n1, p->tw1, p->br1, inverse);
    for (int y = 0; y < p->n1; y++) {
        for (int x = 0; x < p->n0; x++) {
            col[2 * x] = g[2 * ((size_t)x * p->n1 + y)];
            col[2 * x + 1] = g[2 * ((size_t)x * p->n1 + y) + 1];
        }
        fft1(col, p->n0, p->tw0, p->br0, inverse);
        for (int x = 0; x < p->n0; x++) {
            g[2 * ((size_t)x * p->n1 + y)] = col[2 * x];
            g[2 * ((size_t)x * p->n1 + y) + 1] = col[2 * x + 1];
        }
    }
}

/* ------------------------------------------------------------ windows ---- */
/* Modified Bessel function I0 by its power series sum_k ((x/2)^k / k!)^2, in
 * double (all terms positive; 60 terms are far more than x <= 40 needs). */
static double bessel_i0(double x)
{
    double term = 1.0, sum = 1.0, q = 0.25 * x * x;
    for (int k = 1; k < 60; k++) {
        term *= q / ((double)k * (double)k);
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}

/* NU:221-235 (nufft_Phi2d_1dCU) and NU:1242-1256 (nufft_Phi1dCU):
 * l = floor(n*x) - m + t, x1 = x - l/n, phi = bf*exp(-(n*x1)^2/b),
 * index (l+n) % n.  The float build repeats the float expression with expf.
 *
 * ORA_WINDOW_KB4 (no counterpart in the reference): the Kaiser-Bessel window
 * of half-width K = 4 grid points in the same 14-tap layout, u = n*x1,
 *   phi(u) = sinh(kb sqrt(K^2 - u^2)) / (pi sqrt(K^2 - u^2)) / I0(kb K)  for |u| < K,
 * 0 otherwise (so only taps 3..10 can be non-zero), kb = pi (2 - 1/theta)
 * (Kaiser 1974; Jackson et al., IEEE TMI 10 (1991); the shape parameter of
 * Potts, Steidl and Tasche's NFFT).  Its Fourier transform, the
 * deapodisation below, is I0(K sqrt(kb^2 - (2 pi k / n)^2)) / I0(kb K). */
static void window_taps(float x, int n, float b, float bf, int kind, double kb, REAL *phi, int *idx)
{
    float nf = (float)n * x;
    int l0 = (int)(floorf(nf) - ORA_M);
    const double inv = 1.0 / (REF_PI * bessel_i0(kb * ORA_KB_M));
    for (int t = 0; t < ORA_T; t++) {
        int l = l0 + t;
        if (kind == ORA_WINDOW_KB4) {
            /* u = n*x1 is exact in float (n is a power of two); the window
             * itself is evaluated in double in both builds and rounded once,
             * since sinh of arguments up to kb*K ~ 19 would amplify float
             * rounding of its argument ~19-fold. */
            float x1f = x - (float)l / (float)n;
            double u = IS_F32 ? (double)((float)n * x1f) : (double)n * ((double)x - (double)l / (double)n);
            double q = (double)(ORA_KB_M * ORA_KB_M) - u * u;
            double v = q > 0.0 ? sinh(kb * sqrt(q)) / sqrt(q) * inv : 0.0;
            phi[t] = IS_F32 ? (REAL)(float)v : (REAL)v;
        } else if (IS_F32) {
            float x1 = x - (float)l / (float)n;
            float q = ((float)n * x1) * ((float)n * x1) / b;
            phi[t] = (REAL)(bf * expf(-q));
        } else {
            double x1 = (double)x - (double)l / (double)n;
            double q = ((double)n * x1) * ((double)n * x1) / (double)b;
            phi[t] = (REAL)((double)bf * exp(-q));
        }
        idx[t] = (l + n) % n;
    }
}

/* NU:22-42 (nufft_ck2d2) and NU:1258-1271 (nufft_ck1d): per-dimension
 * deapodisation exp(-b (pi k / n)^2), k = X - N/2, evaluated in double; the
 * reference stores each factor as float and multiplies the two in float.
 * Kaiser-Bessel: I0(K sqrt(kb^2 - (2 pi k/n)^2)) / I0(kb K) (kb >= pi/theta
 * >= 2 pi |k|/n for theta >= 1, so the root is real). */
static void deapod(int N, int n, float b, int kind, double kb, REAL *c)
{
    const double i0m = bessel_i0(kb * ORA_KB_M);
    for (int X = 0; X < N; X++) {
        int k = X - N / 2;
        double v;
        if (kind == ORA_WINDOW_KB4) {
            double w = 2.0 * REF_PI * k / (double)n;
            v = bessel_i0(ORA_KB_M * sqrt(kb * kb - w * w)) / i0m;
        } else {
            v = exp(-(double)b * ((REF_PI * k / (double)n) * (REF_PI * k / (double)n)));
        }
        c[X] = IS_F32 ? (REAL)(float)v : (REAL)v;
    }
}

/* -------------------------------------------------------------- plans ---- */
/* Builds what Lib_2D2 builds for one tilt series (MainCode.cu:38-109):
 * negated angles, nodes, weights, grid sizes, window tables, deapodisation. */
int FN(ora_plan_create_w)(int nx, int thickness, int nz, const float *tlt, int window, void **out)
{
    if (nx < 8 || thickness < 8 || nz < 2 || !tlt || !out) return 1;
    if (window != ORA_WINDOW_GAUSS6 && window != ORA_WINDOW_KB4) return 1;
    ora_plan *p = (ora_plan *)calloc(1, sizeof(ora_plan));
    p->window = window;
    p->nx = nx;
    p->nz = nz;
    p->N0 = nx;
    p->N1 = thickness;
    p->M = nx * nz;
    ora_grid_params(p->N0, &p->th0, &p->n0, &p->b0, &p->bf0);
    ora_grid_params(p->N1, &p->th1, &p->n1, &p->b1, &p->bf1);
    p->kb0 = REF_PI * (2.0 - 1.0 / (double)p->th0);
    p->kb1 = REF_PI * (2.0 - 1.0 / (double)p->th1);
    float *th = (float *)malloc(sizeof(float) * (size_t)nz);
    for (int i = 0; i < nz; i++) th[i] = -tlt[i];       /* MainCode.cu:42 */
    p->xy = (float *)malloc(sizeof(float) * 2 * (size_t)p->M);
    p->w = (float *)malloc(sizeof(float) * (size_t)p->M);
    ora_px2d(nx, nz, th, p->xy);
    ora_weight(nx, nz, th, p->w);
    free(th);
    size_t MT = (size_t)p->M * ORA_T;
    p->phix = (REAL *)malloc(sizeof(REAL) * MT);
    p->phiy = (REAL *)malloc(sizeof(REAL) * MT);
    p->ix = (int *)malloc(sizeof(int) * MT);
    p->iy = (int *)malloc(sizeof(int) * MT);
    for (int j = 0; j < p->M; j++) {
        window_taps(p->xy[2 * j], p->n0, p->b0, p->bf0, window, p->kb0, p->phix + (size_t)j * ORA_T,
                    p->ix + (size_t)j * ORA_T);
        window_taps(p->xy[2 * j + 1], p->n1, p->b1, p->bf1, window, p->kb1, p->phiy + (size_t)j * ORA_T,
                    p->iy + (size_t)j * ORA_T);
    }
    p->cx = (REAL *)malloc(sizeof(REAL) * (size_t)p->N0);
    p->cy = (REAL *)malloc(sizeof(REAL) * (size_t)p->N1);
    deapod(p->N0, p->n0, p->b0, window, p->kb0, p->cx);
    deapod(p->N1, p->n1, p->b1, window, p->kb1, p->cy);
    /* 1-D row transform: nodes (k - nx/2)/nx on the n0 grid (MainCode.cu:72-80). */
    p->phi1 = (REAL *)malloc(sizeof(REAL) * (size_t)nx * ORA_T);
    p->i1 = (int *)malloc(sizeof(int) * (size_t)nx * ORA_T);
    for (int k = 0; k < nx; k++) {
        float x = (float)(((double)(float)k - (double)(float)nx / 2.0) / (double)(float)nx);
        window_taps(x, p->n0, p->b0, p->bf0, window, p->kb0, p->phi1 + (size_t)k * ORA_T, p->i1 + (size_t)k * ORA_T);
    }
    p->tw0 = make_twiddles(p->n0);
    p->tw1 = make_twiddles(p->n1);
    p->br0 = make_bitrev(p->n0);
    p->br1 = make_bitrev(p->n1);
    *out = p;
    return 0;
}

/* A plan whose nodes are one line at a single angle (the reprojection plan of
 * MainCode.cu:101-109), sharing grid parameters with a series of width nx. */
int FN(ora_plan_create)(int nx, int thickness, int nz, const float *tlt, void **out)
{
    return FN(ora_plan_create_w)(nx, thickness, nz, tlt, ORA_WINDOW_GAUSS6, out);
}

int FN(ora_plan_create_line_w)(int nx, int thickness, float angle_neg, int window, void **out)
{
    float t2[2] = {-angle_neg, -angle_neg};
    void *pp;
    int rc = FN(ora_plan_create_w)(nx, thickness, 2, t2, window, &pp);
    if (rc) return rc;
    ora_plan *p = (ora_plan *)pp;
    p->nz = 1;
    p->M = nx;
    *out = p;
    return 0;
}

int FN(ora_plan_create_line)(int nx, int thickness, float angle_neg, void **out)
{
    return FN(ora_plan_create_line_w)(nx, thickness, angle_neg, ORA_WINDOW_GAUSS6, out);
}

void FN(ora_plan_destroy)(void *pp)
{
    ora_plan *p = (ora_plan *)pp;
    if (!p) return;
    free(p->xy); free(p->w); free(p->phix); free(p->phiy); free(p->ix); free(p->iy);
    free(p->cx); free(p->cy); free(p->phi1); free(p->i1);
    free(p->tw0); free(p->tw1); free(p->br0); free(p->br1);
    free(p);
}

void FN(ora_plan_dims)(const void *pp, int *d)
{
    const ora_plan *p = (const ora_plan *)pp;
    d[0] = p->N0; d[1] = p->N1; d[2] = p->n0; d[3] = p->n1; d[4] = p->M; d[5] = p->nz;
}

void FN(ora_plan_geometry)(const void *pp, float *xy, float *w, float *params)
{
    const ora_plan *p = (const ora_plan *)pp;
    if (xy) memcpy(xy, p->xy, sizeof(float) * 2 * (size_t)p->M);
    if (w) memcpy(w, p->w, sizeof(float) * (size_t)p->M);
    if (params) {
        params[0] = p->th0; params[1] = p->th1; params[2] = p->b0;
        params[3] = p->bf0; params[4] = p->b1; params[5] = p->bf1;
    }
}

void FN(ora_plan_windows)(const void *pp, REAL *phix, int *ix, REAL *phiy, int *iy, REAL *cx, REAL *cy)
{
    const ora_plan *p = (const ora_plan *)pp;
    size_t MT = (size_t)p->M * ORA_T;
    if (phix) memcpy(phix, p->phix, sizeof(REAL) * MT);
    if (phiy) memcpy(phiy, p->phiy, sizeof(REAL) * MT);
    if (ix) memcpy(ix, p->ix, sizeof(int) * MT);
    if (iy) memcpy(iy, p->iy, sizeof(int) * MT);
    if (cx) memcpy(cx, p->cx, sizeof(REAL) * (size_t)p->N0);
    if (cy) memcpy(cy, p->cy, sizeof(REAL) * (size_t)p->N1);
}

/* ------------------------------------------------------------- NUFFTs ---- */
static REAL ckv(const ora_plan *p, int X, int Y)
{
    return IS_F32 ? (REAL)((float)p->cx[X] * (float)p->cy[Y]) : p->cx[X] * p->cy[Y];
}

/* Forward 2-D NUFFT, image (N0 x N1, Y fastest) -> M node values.
 * NU:984-1076 (cunfft_trafo_2d_R2C2) when img_is_real, NU:844-949
 * (cunfft_trafo_2d2) otherwise:
 *   pre-pass NU:784-809 / NU:754-781: g[x][y] = img[X][Y]/ck(X,Y) with
 *     X = (x+N0/2)%n0, Y = (y+N1/2)%n1, zero elsewhere;
 *   forward FFT (NU:1030);
 *   interpolation NU:669-727: f = sum_{t1} sum_{t0} g[ix][iy]*(phix*phiy),
 *     the t0 sum inside (f1 of nufft_GPhi_p1CU_noPreCompute) and the t1 sum
 *     outside (nufft_GPhi_p2CU). */
void FN(ora_forward)(const void *pp, const REAL *img, int img_is_real, REAL *f, REAL *grid, REAL *col)
{
    const ora_plan *p = (const ora_plan *)pp;
    int N0 = p->N0, N1 = p->N1, n0 = p->n0, n1 = p->n1;
    memset(grid, 0, sizeof(REAL) * 2 * (size_t)n0 * n1);
    for (int X = 0; X < N0; X++) {
        int x = (X - N0 / 2 + n0) % n0;
        for (int Y = 0; Y < N1; Y++) {
            int y = (Y - N1 / 2 + n1) % n1;
            REAL c = ckv(p, X, Y);
            size_t gi = 2 * ((size_t)x * n1 + y), ii = (size_t)X * N1 + Y;
            if (img_is_real) {
                grid[gi] = img[ii] / c;
                grid[gi + 1] = 0;
            } else {
                grid[gi] = img[2 * ii] / c;
                grid[gi + 1] = img[2 * ii + 1] / c;
            }
        }
    }
    fft2(p, grid, 0, col);
    for (int j = 0; j < p->M; j++) {
        const REAL *px = p->phix + (size_t)j * ORA_T, *py = p->phiy + (size_t)j * ORA_T;
        const int *ix = p->ix + (size_t)j * ORA_T, *iy = p->iy + (size_t)j * ORA_T;
        REAL fr = 0, fi = 0;
        for (int t1 = 0; t1 < ORA_T; t1++) {
            REAL ar = 0, ai = 0;
            for (int t0 = 0; t0 < ORA_T; t0++) {
                REAL phi = px[t0] * py[t1];
                const REAL *g = grid + 2 * ((size_t)ix[t0] * n1 + iy[t1]);
                ar = madd(g[0], phi, ar);
                ai = madd(g[1], phi, ai);
            }
            fr += ar;
            fi += ai;
        }
        f[2 * j] = fr;
        f[2 * j + 1] = fi;
    }
}

/* Adjoint 2-D NUFFT, M node values -> image (N0 x N1, Y fastest).
 * NU:1167-1238 (cunfft_adjoint_2d2): the CSR gather of NU:1078-1102 sums, per
 * grid point, f_j * (phix*phiy) in the order the host builder appended the
 * entries (NU:137-145: node j ascending, then y tap, then x tap); the scatter
 * below visits the same terms in the same order per grid point.  Then the
 * inverse FFT (NU:1203) and crop/deapodisation (NU:1104-1121):
 *   fhat[X][Y] = g[(X+n0-N0/2)%n0][(Y+n1-N1/2)%n1] / ck(X,Y). */
void FN(ora_adjoint)(const void *pp, const REAL *f, REAL *fhat, REAL *grid, REAL *col)
{
    const ora_plan *p = (const ora_plan *)pp;
    int N0 = p->N0, N1 = p->N1, n0 = p->n0, n1 = p->n1;
    memset(grid, 0, sizeof(REAL) * 2 * (size_t)n0 * n1);
    for (int j = 0; j < p->M; j++) {
        const REAL *px = p->phix + (size_t)j * ORA_T, *py = p->phiy + (size_t)j * ORA_T;
        const int *ix = p->ix + (size_t)j * ORA_T, *iy = p->iy + (size_t)j * ORA_T;
        REAL fr = f[2 * j], fi = f[2 * j + 1];
        for (int t1 = 0; t1 < ORA_T; t1++) {
            for (int t0 = 0; t0 < ORA_T; t0++) {
                REAL phi = px[t0] * py[t1];
                REAL *g = grid + 2 * ((size_t)ix[t0] * n1 + iy[t1]);
                g[0] = madd(fr, phi, g[0]);
                g[1] = madd(fi, phi, g[1]);
            }
        }
    }
    fft2(p, grid, 1, col);
    for (int X = 0; X < N0; X++) {
        int x = (X + n0 - N0 / 2) % n0;
        for (int Y = 0; Y < N1; Y++) {
            int y = (Y + n1 - N1 / 2) % n1;
            REAL c = ckv(p, X, Y);
            size_t gi = 2 * ((size_t)x * n1 + y), oi = 2 * ((size_t)X * N1 + Y);
            fhat[oi] = grid[gi] / c;
            fhat[oi + 1] = grid[gi + 1] / c;
        }
    }
}

/* 1-D forward NUFFT of one real projection row of length nx evaluated at the
 * nodes (k - nx/2)/nx: NU:1479-1516 (cunfft_trafo_1d) with the pre-pass of
 * NU:1432-1452 and the interpolation of NU:1454-1477 (taps in order). */
static void row_forward(const ora_plan *p, const float *row, REAL *out, REAL *g1)
{
    int N = p->nx, n = p->n0;
    memset(g1, 0, sizeof(REAL) * 2 * (size_t)n);
    for (int x = 0; x < n; x++) {
        int X = (x + N / 2) % n;
        if (X < N) g1[2 * x] = (REAL)row[X] / p->cx[X];
    }
    fft1(g1, n, p->tw0, p->br0, 0);
    for (int k = 0; k < N; k++) {
        const REAL *ph = p->phi1 + (size_t)k * ORA_T;
        const int *ii = p->i1 + (size_t)k * ORA_T;
        REAL fr = 0, fi = 0;
        for (int t = 0; t < ORA_T; t++) {
            fr = madd(g1[2 * ii[t]], ph[t], fr);
            fi = madd(g1[2 * ii[t] + 1], ph[t], fi);
        }
        out[2 * k] = fr;
        out[2 * k + 1] = fi;
    }
}

/* 1-D adjoint NUFFT (NU:1518-1536): spread, inverse FFT, crop and divide by
 * the 1-D deapodisation (NU:1123-1135). */
static void row_adjoint(const ora_plan *p, const REAL *f, REAL *out, REAL *g1)
{
    int N = p->nx, n = p->n0;
    memset(g1, 0, sizeof(REAL) * 2 * (size_t)n);
    for (int k = 0; k < N; k++) {
        const REAL *ph = p->phi1 + (size_t)k * ORA_T;
        const int *ii = p->i1 + (size_t)k * ORA_T;
        for (int t = 0; t < ORA_T; t++) {
            g1[2 * ii[t]] = madd(f[2 * k], ph[t], g1[2 * ii[t]]);
            g1[2 * ii[t] + 1] = madd(f[2 * k + 1], ph[t], g1[2 * ii[t] + 1]);
        }
    }
    fft1(g1, n, p->tw0, p->br0, 1);
    for (int X = 0; X < N; X++) {
        int x = (X + n - N / 2) % n;
        out[2 * X] = g1[2 * x] / p->cx[X];
        out[2 * X + 1] = g1[2 * x + 1] / p->cx[X];
    }
}

/* ------------------------------------------------------------ drivers ---- */
typedef struct {
    REAL *grid, *col, *g1, *f, *fhat, *rhat, *r;
} ora_work;

static void work_alloc(const ora_plan *p, ora_work *w)
{
    size_t nn = (size_t)p->n0 * p->n1, NN = (size_t)p->N0 * p->N1;
    w->grid = (REAL *)malloc(sizeof(REAL) * 2 * nn);
    w->col = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->n0);
    w->g1 = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->n0);
    w->f = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->M);
    w->r = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->M);
    w->fhat = (REAL *)malloc(sizeof(REAL) * 2 * NN);
    w->rhat = w->fhat;   /* aliased as in initGICONPara2 (NU:1755) */
}

static void work_free(ora_work *w)
{
    free(w->grid); free(w->col); free(w->g1); free(w->f); free(w->r); free(w->fhat);
}

void FN(ora_nufft_forward)(const void *pp, const REAL *img, int img_is_real, REAL *f)
{
    ora_work w;
    work_alloc((const ora_plan *)pp, &w);
    FN(ora_forward)(pp, img, img_is_real, f, w.grid, w.col);
    work_free(&w);
}

void FN(ora_nufft_adjoint)(const void *pp, const REAL *f, REAL *fhat)
{
    ora_work w;
    work_alloc((const ora_plan *)pp, &w);
    FN(ora_adjoint)(pp, f, fhat, w.grid, w.col);
    work_free(&w);
}

/* Projection rows of one slice (nz x nx floats, readSlicePart.cu:13-22) ->
 * b (M complex), one 1-D NUFFT per tilt row. */
void FN(ora_rows_forward)(const void *pp, const float *rows, REAL *b)
{
    const ora_plan *p = (const ora_plan *)pp;
    REAL *g1 = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->n0);
    for (int i = 0; i < p->nz; i++)
        row_forward(p, rows + (size_t)i * p->nx, b + 2 * (size_t)i * p->nx, g1);
    free(g1);
}

void FN(ora_row_adjoint)(const void *pp, const REAL *f, REAL *out)
{
    const ora_plan *p = (const ora_plan *)pp;
    REAL *g1 = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)p->n0);
    row_adjoint(p, f, out, g1);
    free(g1);
}

/* Right-hand side A^H W b (MainCode.cu:115-134): rows -> b, b *= w
 * (complexMulDoubleCU, NU:1539-1549), adjoint. */
void FN(ora_rhs)(const void *pp, const float *rows, REAL *Ahwb)
{
    const ora_plan *p = (const ora_plan *)pp;
    ora_work w;
    work_alloc(p, &w);
    FN(ora_rows_forward)(pp, rows, w.f);
    for (int j = 0; j < p->M; j++) {
        w.f[2 * j] = w.f[2 * j] * (REAL)p->w[j];
        w.f[2 * j + 1] = w.f[2 * j + 1] * (REAL)p->w[j];
    }
    FN(ora_adjoint)(pp, w.f, Ahwb, w.grid, w.col);
    work_free(&w);
}

/* Iteration3 (Iteration2.cu:3-150) with Alpha2 (alpha_new2.cu:3-119).
 * m (N0*N1 real) is the start value on entry (the reference zeroes it,
 * Iteration2.cu:33) and the result on exit.  Schedule: the clamped ICON update
 * (NU:1597-1616) for a <= i < a+b, the plain INFR update (NU:1630-1639)
 * otherwise.  alphas/rtrs, when given, receive alpha and ||rhat||^2 per
 * iteration. */
void FN(ora_solve)(const void *pp, const REAL *Ahwb, int a, int bmid, int c, int dataType,
                   float threshold, REAL *m, double *alphas, double *rtrs)
{
    const ora_plan *p = (const ora_plan *)pp;
    int iters = a + bmid + c;
    size_t NN = (size_t)p->N0 * p->N1;
    ora_work w;
    work_alloc(p, &w);
    for (int it = 0; it < iters; it++) {
        FN(ora_forward)(pp, m, 1, w.f, w.grid, w.col);                 /* Iteration2.cu:53 */
        for (int j = 0; j < p->M; j++) {                                /* :69 */
            w.f[2 * j] = w.f[2 * j] * (REAL)p->w[j];
            w.f[2 * j + 1] = w.f[2 * j + 1] * (REAL)p->w[j];
        }
        FN(ora_adjoint)(pp, w.f, w.fhat, w.grid, w.col);               /* :80 */
        for (size_t i = 0; i < 2 * NN; i++) w.rhat[i] = w.fhat[i] - Ahwb[i];   /* :96 */
        double rtr = 0;                                                 /* alpha0, NU:1641-1650 */
        for (size_t i = 0; i < NN; i++)
            rtr += (double)w.rhat[2 * i] * (double)w.rhat[2 * i] + (double)w.rhat[2 * i + 1] * (double)w.rhat[2 * i + 1];
        FN(ora_forward)(pp, w.rhat, 0, w.r, w.grid, w.col);            /* alpha_new2.cu:77 */
        double rtar = 0;                                                /* alpha1, NU:1652-1661 */
        for (int j = 0; j < p->M; j++) {
            double wj = (double)p->w[j];
            rtar += (double)w.r[2 * j] * (double)w.r[2 * j] * wj + (double)w.r[2 * j + 1] * (double)w.r[2 * j + 1] * wj;
        }
        double al = rtar != 0 ? rtr / rtar : 0;                          /* alpha2, NU:1663-1673 */
        if (alphas) alphas[it] = al;
        if (rtrs) rtrs[it] = rtr;
        int icon = (a <= it && it < iters - c);                         /* Iteration2.cu:129 */
        for (size_t i = 0; i < NN; i++) {
            REAL v = (REAL)((double)m[i] - al * (double)w.rhat[2 * i]);
            if (icon) {
                if (dataType == 1) {
                    if (v > (REAL)threshold) v = (REAL)threshold;
                } else {
                    if (v < (REAL)threshold) v = (REAL)threshold;
                }
            }
            m[i] = v;
        }
    }
    work_free(&w);
}

/* reProject_NFFT2 (reProject_NFFT.cu:25-42): forward 2-D NUFFT of m at the
 * nodes of the line plan, then the 1-D adjoint; the real part is returned. */
void FN(ora_reproject)(const void *line_plan, const void *series_plan, const REAL *m, REAL *out)
{
    const ora_plan *lp = (const ora_plan *)line_plan;
    ora_work w;
    work_alloc(lp, &w);
    REAL *tmp = (REAL *)malloc(sizeof(REAL) * 2 * (size_t)lp->nx);
    FN(ora_forward)(line_plan, m, 1, w.f, w.grid, w.col);
    FN(ora_row_adjoint)(series_plan, w.f, tmp);
    for (int X = 0; X < lp->nx; X++) out[X] = tmp[2 * X];
    free(tmp);
    work_free(&w);
}

/* One slice of Lib_2D2 (MainCode.cu:113-142): rows -> A^H W b -> Iteration3
 * from m = 0 -> m.  Batch form: S slices, OpenMP over slices when built with
 * -fopenmp; returns the number of threads used. */
int FN(ora_reconstruct)(const void *pp, const float *rows, int S, int a, int bmid, int c,
                        int dataType, float threshold, REAL *m, int nthreads)
{
    const ora_plan *p = (const ora_plan *)pp;
    size_t NN = (size_t)p->N0 * p->N1, R = (size_t)p->nz * p->nx;
    int used = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
#pragma omp single
        used = omp_get_num_threads();
#pragma omp for schedule(dynamic, 1)
        for (int s = 0; s < S; s++) {
            REAL *Ahwb = (REAL *)malloc(sizeof(REAL) * 2 * NN);
            FN(ora_rhs)(pp, rows + (size_t)s * R, Ahwb);
            memset(m + (size_t)s * NN, 0, sizeof(REAL) * NN);
            FN(ora_solve)(pp, Ahwb, a, bmid, c, dataType, threshold, m + (size_t)s * NN, NULL, NULL);
            free(Ahwb);
        }
    }
#else
    (void)nthreads;
    for (int s = 0; s < S; s++) {
        REAL *Ahwb = (REAL *)malloc(sizeof(REAL) * 2 * NN);
        FN(ora_rhs)(pp, rows + (size_t)s * R, Ahwb);
        memset(m + (size_t)s * NN, 0, sizeof(REAL) * NN);
        FN(ora_solve)(pp, Ahwb, a, bmid, c, dataType, threshold, m + (size_t)s * NN, NULL, NULL);
        free(Ahwb);
    }
#endif
    return used;
}

/* Direct NDFT in double (known-answer check, no reference counterpart):
 * f_j = sum_{X,Y} img[X][Y] exp(-2 pi i ((X-N0/2) x0_j + (Y-N1/2) x1_j)). */
/* Batched input stage and solve for timing the CPU path in pieces: S slices,
 * OpenMP over slices.  ora_rhs_batch: Ahwb[s] = A^H W b of rows[s] (the input
 * stage of Lib_2D2, MainCode.cu:115-134).  ora_solve_batch: ora_solve on every
 * slice, m[s] holding its start value on entry, so that consecutive calls
 * with consecutive pieces of the schedule (a, bmid, c counted within each
 * piece) run the whole schedule: the iteration carries no state but m.
 * Return the number of threads used. */
int FN(ora_rhs_batch)(const void *pp, const float *rows, int S, REAL *Ahwb, int nthreads)
{
    const ora_plan *p = (const ora_plan *)pp;
    size_t NN = (size_t)p->N0 * p->N1, R = (size_t)p->nz * p->nx;
    int used = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
#pragma omp single
        used = omp_get_num_threads();
#pragma omp for schedule(dynamic, 1)
        for (int s = 0; s < S; s++) FN(ora_rhs)(pp, rows + (size_t)s * R, Ahwb + (size_t)s * 2 * NN);
    }
#else
    (void)nthreads;
    for (int s = 0; s < S; s++) FN(ora_rhs)(pp, rows + (size_t)s * R, Ahwb + (size_t)s * 2 * NN);
#endif
    return used;
}

int FN(ora_solve_batch)(const void *pp, const REAL *Ahwb, int S, int a, int bmid, int c, int dataType,
                        float threshold, REAL *m, int nthreads)
{
    const ora_plan *p = (const ora_plan *)pp;
    size_t NN = (size_t)p->N0 * p->N1;
    int used = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
#pragma omp single
        used = omp_get_num_threads();
#pragma omp for schedule(dynamic, 1)
        for (int s = 0; s < S; s++)
            FN(ora_solve)(pp, Ahwb + (size_t)s * 2 * NN, a, bmid, c, dataType, threshold, m + (size_t)s * NN, NULL, NULL);
    }
#else
    (void)nthreads;
    for (int s = 0; s < S; s++)
        FN(ora_solve)(pp, Ahwb + (size_t)s * 2 * NN, a, bmid, c, dataType, threshold, m + (size_t)s * NN, NULL, NULL);
#endif
    return used;
}

void FN(ora_ndft_forward)(const void *pp, const double *img, int img_is_real, double *f)
{
    const ora_plan *p = (const ora_plan *)pp;
    for (int j = 0; j < p->M; j++) {
        double x0 = p->xy[2 * j], x1 = p->xy[2 * j + 1];
        double fr = 0, fi = 0;
        for (int X = 0; X < p->N0; X++) {
            for (int Y = 0; Y < p->N1; Y++) {
                double ph = -2.0 * M_PI * ((double)(X - p->N0 / 2) * x0 + (double)(Y - p->N1 / 2) * x1);
                double c = cos(ph), s = sin(ph);
                size_t ii = (size_t)X * p->N1 + Y;
                double vr = img_is_real ? img[ii] : img[2 * ii];
                double vi = img_is_real ? 0 : img[2 * ii + 1];
                fr += vr * c - vi * s;
                fi += vr * s + vi * c;
            }
        }
        f[2 * j] = fr;
        f[2 * j + 1] = fi;
    }
}

/* Direct adjoint NDFT in double: img[X][Y] = sum_j f_j exp(+2 pi i (...)). */
void FN(ora_ndft_adjoint)(const void *pp, const double *f, double *img)
{
    const ora_plan *p = (const ora_plan *)pp;
    for (int X = 0; X < p->N0; X++) {
        for (int Y = 0; Y < p->N1; Y++) {
            double ar = 0, ai = 0;
            for (int j = 0; j < p->M; j++) {
                double ph = 2.0 * M_PI * ((double)(X - p->N0 / 2) * p->xy[2 * j] + (double)(Y - p->N1 / 2) * p->xy[2 * j + 1]);
                double c = cos(ph), s = sin(ph);
                ar += f[2 * j] * c - f[2 * j + 1] * s;
                ai += f[2 * j] * s + f[2 * j + 1] * c;
            }
            img[2 * ((size_t)X * p->N1 + Y)] = ar;
            img[2 * ((size_t)X * p->N1 + Y) + 1] = ai;
        }
    }
}
