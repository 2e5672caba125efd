// icon_kernels.cuh -- the sm_100a kernels of the ICON hot path.
//
// The reference (ICON-GPU v1.2.9, NU = nufft_gpu_v8.cu) computes a NUFFT as
// pre-pass -> full 2-D cuFFT of the n0 x n1 grid -> interpolation (forward), or
// CSR gather onto the grid -> 2-D cuFFT -> crop (adjoint), one slice at a time.
// Here a batch of B slices moves through two FFT passes whose far ends are
// fused with the non-uniform step, so the oversampled grid is never stored:
//
//   forward   K1  xpass_fwd   per (column Y, group): deapodise + pad + shift
//                             the image column, FFT along x (length n0)
//                             -> G1[x][Y][b]                 (N1 of n1 columns)
//             K2  ypass_fwd   per (row x, group): pad row x of G1, FFT along y
//                             (length n1) in shared memory, then for every
//                             (node j, x-tap t0) whose x-tap lands on row x
//                             the y-interpolation sum_t1 phiy*G -> P[j][t0][b]
//             K3  interp_fin  per node: f_j = sum_t0 phix * P[j][t0]
//                             (+ weighting / step-length partial sums)
//   adjoint   K2T ypass_adj   per (row x, group): gather every node's
//                             contribution on row x into shared memory (no
//                             atomics), inverse FFT along y, keep the N1 rows
//                             the crop keeps -> G1[x][Y][b]
//             K1T xpass_adj   per (column Y, group): inverse FFT along x,
//                             crop, divide by the deapodisation
//                             (+ r = fhat - Ahwb and ||r||^2 partial sums)
#pragma once
#include "icon_device.cuh"

namespace icon {

// Device view of one tilt-series geometry (all pointers are device memory).
struct Geo {
    int N0, N1, n0, n1, lg0, lg1, M, nx, nz, B;
    const float *w;        // [M] density weights (Weight, weight.cu:8-41)
    const float *phix;     // [M][14] window values, x taps   (NU:221-235)
    const float *phiy;     // [M][14] window values, y taps
    const int *ix0;        // [M] first x tap, unwrapped: floor(n0*x0) - 6
    const int *iy0;        // [M] first y tap, unwrapped
    const float *cx;       // [N0] deapodisation factor along x (NU:22-42)
    const float *cy;       // [N1] deapodisation factor along y
    const int *row_off;    // [n0+1] entry range of every grid row x
    const int *ent_jt;     // [M*14] entry: node*16 + x tap, sorted by (row, iy0, node)
    const int *ent_iy0;    // [M*14] iy0 of the entry's node (sort key within a row)
    const float2 *tw0;     // [n0] exp(-2 pi i q / n0)
    const float2 *tw1;     // [n1] exp(-2 pi i q / n1)
};

// 1-D row-transform tables (cunfft_initPlan_1d, NU:1298-1391).
struct Geo1 {
    const float *phi1;     // [nx][14]
    const int *i10;        // [nx] first tap, unwrapped, nondecreasing in k
};

// ------------------------------------------------------------- tables ----
// Window taps exactly as nufft_Phi2d_1dCU (NU:221-235) computes them, in float:
// l = floor(n*x) - m + t, x1 = x - l/n, phi = bf*exp(-(n*x1)^2/b).
__global__ void k_window(const float *__restrict__ x, int stride, int M, int n, float b, float bf,
                         float *__restrict__ phi, int *__restrict__ l0out)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    float xv = x[(size_t)j * stride];
    int l0 = (int)(floorf(n * xv) - kHalf);
    l0out[j] = l0;
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
        int l = l0 + t;
        float x1 = xv - (float)l / (float)n;
        phi[(size_t)j * kTaps + t] = bf * expf(-((n * x1) * (n * x1) / b));
    }
}

// --------------------------------------------------------------- K1 ----
// Forward x-pass.  in: [G][N1][N0][B] real (m) or complex; out G1 [G][n0][N1][B].
// Pre-pass of NU:784-809 / NU:754-781: grid x holds img[X]/ck(X,Y) with
// X = (x + N0/2) % n0 when X < N0, else 0; ck = cx[X]*cy[Y] in float.
template <bool REAL_IN>
__global__ void __launch_bounds__(1024) k_xpass_fwd(Geo g, const void *__restrict__ in, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    const int Y = blockIdx.x, grp = blockIdx.y, B = g.B, n = g.n0, N0 = g.N0;
    const float cyY = g.cy[Y];
    const size_t ibase = ((size_t)grp * g.N1 + Y) * N0 * B;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        int b = idx % B, x = idx / B;
        int X = (x + N0 / 2) % n;
        float2 v = make_float2(0.f, 0.f);
        if (X < N0) {
            float ck = g.cx[X] * cyY;
            if (REAL_IN) {
                v.x = ((const float *)in)[ibase + (size_t)X * B + b] / ck;
            } else {
                float2 t = ((const float2 *)in)[ibase + (size_t)X * B + b];
                v.x = t.x / ck;
                v.y = t.y / ck;
            }
        }
        s[idx] = v;
    }
    __syncthreads();
    fft_smem(s, n, g.lg0, B, g.tw0, -1.f);
    const size_t obase = (size_t)grp * n * g.N1 * B;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        int b = idx % B, x = idx / B;
        G1[obase + ((size_t)x * g.N1 + Y) * B + b] = s[idx];
    }
}

// --------------------------------------------------------------- K2 ----
// Forward y-pass fused with the y-direction interpolation.  Row x of G1 holds
// the N1 nonzero columns; column Y sits at y with (y + N1/2) % n1 == Y.
// P[G][M][14][B]: P[j][t0] = sum_t1 phiy[j][t1] * G[x][(iy0_j + t1) mod n1],
// x = (ix0_j + t0) mod n0.  (NU:669-727 sum the same 196 products per node.)
__global__ void __launch_bounds__(1024) k_ypass_fwd(Geo g, const float2 *__restrict__ G1, float2 *__restrict__ P)
{
    extern __shared__ float2 s[];
    const int x = blockIdx.x, grp = blockIdx.y, B = g.B, n = g.n1, N1 = g.N1;
    const size_t rbase = ((size_t)grp * g.n0 + x) * N1 * B;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        int b = idx % B, y = idx / B;
        int Y = (y + N1 / 2) % n;
        s[idx] = (Y < N1) ? G1[rbase + (size_t)Y * B + b] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_smem(s, n, g.lg1, B, g.tw1, -1.f);
    const int e0 = g.row_off[x], ne = g.row_off[x + 1] - e0;
    const size_t pbase = (size_t)grp * g.M * kTaps * B;
    for (int idx = threadIdx.x; idx < ne * B; idx += blockDim.x) {
        int b = idx % B, e = e0 + idx / B;
        int jt = __ldg(&g.ent_jt[e]);
        int j = jt >> 4, t0 = jt & 15;
        int iy = __ldg(&g.ent_iy0[e]);
        const float *py = g.phiy + (size_t)j * kTaps;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t1 = 0; t1 < kTaps; ++t1) {
            int y = iy + t1;
            y += (y < 0) ? n : 0;
            y -= (y >= n) ? n : 0;
            float2 v = s[y * B + b];
            float p = __ldg(&py[t1]);
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        P[pbase + ((size_t)j * kTaps + t0) * B + b] = acc;
    }
}

// --------------------------------------------------------------- K3 ----
// f_j = sum_t0 phix[j][t0] * P[j][t0].  MODE 0: store f.  MODE 1: store
// f*w (complexMulDoubleCU, NU:1539-1549).  MODE 2: store nothing; per-slice
// partial sums of w*|f|^2 in double (alpha1, NU:1652-1661) into
// part[G][gridDim.x][B].
template <int MODE>
__global__ void k_interp_fin(Geo g, const float2 *__restrict__ P, float2 *__restrict__ f, double *__restrict__ part)
{
    __shared__ double red[256];
    const int grp = blockIdx.y, B = g.B;
    const int item = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = item / B, b = item % B;
    double acc2 = 0.0;
    if (j < g.M) {
        const float *px = g.phix + (size_t)j * kTaps;
        const float2 *pp = P + ((size_t)grp * g.M + j) * kTaps * B + b;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t0 = 0; t0 < kTaps; ++t0) {
            float2 v = pp[(size_t)t0 * B];
            float p = __ldg(&px[t0]);
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        if (MODE == 0) {
            f[((size_t)grp * g.M + j) * B + b] = acc;
        } else if (MODE == 1) {
            float w = __ldg(&g.w[j]);
            f[((size_t)grp * g.M + j) * B + b] = make_float2(acc.x * w, acc.y * w);
        } else {
            double w = (double)__ldg(&g.w[j]);
            acc2 = (double)acc.x * (double)acc.x * w + (double)acc.y * (double)acc.y * w;
        }
    }
    if (MODE == 2) {
        double r = block_sum_per_slice(acc2, red, B);
        if ((int)threadIdx.x < B) part[((size_t)grp * gridDim.x + blockIdx.x) * B + threadIdx.x] = r;
    }
}

// Index of the first entry in [lo, hi) of the sorted key array with key >= v.
__device__ __forceinline__ int lower_bound_i(const int *__restrict__ key, int lo, int hi, int v)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&key[mid]) < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// -------------------------------------------------------------- K2T ----
// Adjoint y-pass.  Each grid point (x, y) of the row gathers, in a fixed order,
// the contributions phix*phiy*f_j of the entries whose y footprint
// [iy0, iy0+13] covers y (or y - n1: the footprint is unwrapped); the
// reference gathers the same sums through its host-built CSR (NU:1078-1102).
// Then the inverse FFT along y (NU:1203), and the rows Y < N1 of the crop
// (NU:1104-1121: y = (Y + n1 - N1/2) % n1) go to G1[x][Y][b].
__global__ void __launch_bounds__(1024) k_ypass_adj(Geo g, const float2 *__restrict__ f, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    const int x = blockIdx.x, grp = blockIdx.y, B = g.B, n = g.n1, N1 = g.N1;
    const int e0 = g.row_off[x], e1 = g.row_off[x + 1];
    const float2 *fg = f + (size_t)grp * g.M * B;
    for (int y = threadIdx.x; y < n; y += blockDim.x) {
        float2 acc[8];
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[b] = make_float2(0.f, 0.f);
        // Unwrapped positions u of this y: y itself and y - n1.
#pragma unroll
        for (int al = 0; al < 2; ++al) {
            int u = y - al * n;
            int a = lower_bound_i(g.ent_iy0, e0, e1, u - (kTaps - 1));
            int c = lower_bound_i(g.ent_iy0, a, e1, u + 1);
            for (int e = a; e < c; ++e) {
                int jt = __ldg(&g.ent_jt[e]);
                int j = jt >> 4, t0 = jt & 15;
                int d = u - __ldg(&g.ent_iy0[e]);
                float coef = __ldg(&g.phix[(size_t)j * kTaps + t0]) * __ldg(&g.phiy[(size_t)j * kTaps + d]);
                const float2 *fj = fg + (size_t)j * B;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    if (b < B) {
                        float2 v = __ldg(&fj[b]);
                        acc[b].x = fmaf(v.x, coef, acc[b].x);
                        acc[b].y = fmaf(v.y, coef, acc[b].y);
                    }
                }
            }
        }
#pragma unroll
        for (int b = 0; b < 8; ++b)
            if (b < B) s[y * B + b] = acc[b];
    }
    __syncthreads();
    fft_smem(s, n, g.lg1, B, g.tw1, +1.f);
    const size_t obase = ((size_t)grp * g.n0 + x) * N1 * B;
    for (int idx = threadIdx.x; idx < N1 * B; idx += blockDim.x) {
        int b = idx % B, Y = idx / B;
        int y = (Y + n - N1 / 2) % n;
        G1[obase + idx] = s[y * B + b];
    }
}

// -------------------------------------------------------------- K1T ----
// Adjoint x-pass: inverse FFT along x of column Y, crop X < N0 with
// x = (X + n0 - N0/2) % n0, divide by ck = cx[X]*cy[Y] (NU:1104-1121).
// MODE 0: out = fhat.  MODE 1: out = fhat - Ahwb (complexMinusCU,
// NU:1563-1573) and per-slice partial sums of |out|^2 in double (alpha0,
// NU:1641-1650) into part[G][N1][B].  out/Ahwb: [G][N1][N0][B].
template <int MODE>
__global__ void __launch_bounds__(1024) k_xpass_adj(Geo g, const float2 *__restrict__ G1, float2 *__restrict__ out,
                            const float2 *__restrict__ Ahwb, double *__restrict__ part)
{
    extern __shared__ float2 s[];
    double *red = (double *)(s + (size_t)g.n0 * g.B);
    const int Y = blockIdx.x, grp = blockIdx.y, B = g.B, n = g.n0, N0 = g.N0;
    const size_t ibase = (size_t)grp * n * g.N1 * B;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        int b = idx % B, x = idx / B;
        s[idx] = G1[ibase + ((size_t)x * g.N1 + Y) * B + b];
    }
    __syncthreads();
    fft_smem(s, n, g.lg0, B, g.tw0, +1.f);
    const float cyY = g.cy[Y];
    const size_t obase = ((size_t)grp * g.N1 + Y) * N0 * B;
    double acc2 = 0.0;
    for (int idx = threadIdx.x; idx < N0 * B; idx += blockDim.x) {
        int b = idx % B, X = idx / B;
        int x = (X + n - N0 / 2) % n;
        float ck = g.cx[X] * cyY;
        float2 v = s[x * B + b];
        v.x = v.x / ck;
        v.y = v.y / ck;
        if (MODE == 1) {
            float2 a = Ahwb[obase + idx];
            v.x = v.x - a.x;
            v.y = v.y - a.y;
            acc2 += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
        }
        out[obase + idx] = v;
    }
    if (MODE == 1) {
        double r = block_sum_per_slice(acc2, red, B);
        if ((int)threadIdx.x < B) part[((size_t)grp * g.N1 + Y) * B + threadIdx.x] = r;
    }
}

// ------------------------------------------------------------ rows ----
// Input stage: per (tilt i, group) the 1-D NUFFT of the projection rows
// (cunfft_trafo_1d NU:1479-1516: pre-pass NU:1432-1452, FFT, interpolation
// NU:1454-1477 with taps summed in order), then f = b*w (NU:1539-1549).
// rows: [S][nz][nx] (caller layout).  f, bout: [G][M][B]; bout may be null.
__global__ void __launch_bounds__(1024) k_rows_fwd(Geo g, Geo1 g1, const float *__restrict__ rows, int S, float2 *__restrict__ f,
                           float2 *__restrict__ bout)
{
    extern __shared__ float2 s[];
    const int i = blockIdx.x, grp = blockIdx.y, B = g.B, n = g.n0, N = g.nx;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        int b = idx % B, x = idx / B;
        int X = (x + N / 2) % n;
        int sl = grp * B + b;
        float2 v = make_float2(0.f, 0.f);
        if (X < N && sl < S) {
            float c = g.cx[X];
            v.x = rows[((size_t)sl * g.nz + i) * N + X] / c;
            v.y = 0.f / c;
        }
        s[idx] = v;
    }
    __syncthreads();
    fft_smem(s, n, g.lg0, B, g.tw0, -1.f);
    for (int idx = threadIdx.x; idx < N * B; idx += blockDim.x) {
        int b = idx % B, k = idx / B;
        int l0 = __ldg(&g1.i10[k]);
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t = 0; t < kTaps; ++t) {
            int x = l0 + t;
            x += (x < 0) ? n : 0;
            x -= (x >= n) ? n : 0;
            float p = __ldg(&g1.phi1[(size_t)k * kTaps + t]);
            float2 v = s[x * B + b];
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        int j = i * N + k;
        size_t o = ((size_t)grp * g.M + j) * B + b;
        if (bout) bout[o] = acc;
        float w = __ldg(&g.w[j]);
        f[o] = make_float2(acc.x * w, acc.y * w);
    }
}

// 1-D adjoint NUFFT of the nx values of one line (cunfft_adjoint_1d,
// NU:1518-1536): gather in node order (the order of the reference's 1-D CSR),
// inverse FFT, crop, divide by the deapodisation, real part.
// f: [G][nx][B]; out: [S][nx] (caller layout).
__global__ void __launch_bounds__(1024) k_row_adj(Geo g, Geo1 g1, const float2 *__restrict__ f, float *__restrict__ out, int S)
{
    extern __shared__ float2 s[];
    const int grp = blockIdx.x, B = g.B, n = g.n0, N = g.nx;
    const float2 *fg = f + (size_t)grp * N * B;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        float2 acc[8];
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[b] = make_float2(0.f, 0.f);
#pragma unroll
        for (int al = 0; al < 2; ++al) {
            int u = x - al * n;
            int a = lower_bound_i(g1.i10, 0, N, u - (kTaps - 1));
            int c = lower_bound_i(g1.i10, a, N, u + 1);
            for (int k = a; k < c; ++k) {
                int d = u - __ldg(&g1.i10[k]);
                float p = __ldg(&g1.phi1[(size_t)k * kTaps + d]);
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    if (b < B) {
                        float2 v = fg[(size_t)k * B + b];
                        acc[b].x = fmaf(v.x, p, acc[b].x);
                        acc[b].y = fmaf(v.y, p, acc[b].y);
                    }
                }
            }
        }
#pragma unroll
        for (int b = 0; b < 8; ++b)
            if (b < B) s[x * B + b] = acc[b];
    }
    __syncthreads();
    fft_smem(s, n, g.lg0, B, g.tw0, +1.f);
    for (int idx = threadIdx.x; idx < N * B; idx += blockDim.x) {
        int b = idx % B, X = idx / B;
        int sl = grp * B + b;
        int x = (X + n - N / 2) % n;
        if (sl < S) out[(size_t)sl * N + X] = s[x * B + b].x / g.cx[X];
    }
}

// ----------------------------------------------------- layout moves ----
// Caller image [S][N0][N1] <-> batched [G][N1][N0][B]; slices >= S read as 0.
template <typename T>
__global__ void k_img_in(const T *__restrict__ src, T *__restrict__ dst, int S, int N0, int N1, int B, size_t total)
{
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total; o += (size_t)gridDim.x * blockDim.x) {
        int b = (int)(o % B);
        size_t r = o / B;
        int X = (int)(r % N0);
        r /= N0;
        int Y = (int)(r % N1);
        int grp = (int)(r / N1);
        int sl = grp * B + b;
        T v{};
        if (sl < S) v = src[((size_t)sl * N0 + X) * N1 + Y];
        dst[o] = v;
    }
}

template <typename T>
__global__ void k_img_out(const T *__restrict__ src, T *__restrict__ dst, int S, int N0, int N1, int B)
{
    size_t total = (size_t)S * N0 * N1;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int Y = (int)(i % N1);
        size_t r = i / N1;
        int X = (int)(r % N0);
        int sl = (int)(r / N0);
        int grp = sl / B, b = sl % B;
        dst[i] = src[(((size_t)grp * N1 + Y) * N0 + X) * B + b];
    }
}

// Caller nodes [S][M] <-> batched [G][M][B].
__global__ void k_nodes_in(const float2 *__restrict__ src, float2 *__restrict__ dst, int S, int M, int B, size_t total)
{
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total; o += (size_t)gridDim.x * blockDim.x) {
        int b = (int)(o % B);
        size_t r = o / B;
        int j = (int)(r % M);
        int grp = (int)(r / M);
        int sl = grp * B + b;
        dst[o] = (sl < S) ? src[(size_t)sl * M + j] : make_float2(0.f, 0.f);
    }
}

__global__ void k_nodes_out(const float2 *__restrict__ src, float2 *__restrict__ dst, int S, int M, int B)
{
    size_t total = (size_t)S * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(i % M);
        int sl = (int)(i / M);
        dst[i] = src[(((size_t)(sl / B)) * M + j) * B + (sl % B)];
    }
}

// ----------------------------------------------------- step length ----
// alpha = rtr / rtar, 0 when rtar == 0 (alpha2, NU:1663-1673), per slice.
// One block per group, one warp per slice; partial sums are added in a fixed
// order, so the result does not depend on scheduling.
__global__ void k_alpha(const double *__restrict__ part_rtr, int nr, const double *__restrict__ part_rtar, int na,
                        int B, double *__restrict__ alpha, double *__restrict__ hist_alpha, double *__restrict__ hist_rtr)
{
    const int grp = blockIdx.x, b = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (b >= B) return;
    double r1 = 0.0, r2 = 0.0;
    for (int i = lane; i < nr; i += 32) r1 += part_rtr[((size_t)grp * nr + i) * B + b];
    for (int i = lane; i < na; i += 32) r2 += part_rtar[((size_t)grp * na + i) * B + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    }
    if (lane == 0) {
        double a = (r2 != 0.0) ? r1 / r2 : 0.0;
        int sl = grp * B + b;
        alpha[sl] = a;
        if (hist_alpha) hist_alpha[sl] = a;
        if (hist_rtr) hist_rtr[sl] = r1;
    }
}

// m <- m - alpha*Re(rhat) computed in double and stored as float; ICON steps
// also clamp (ICONUpdateCU_R NU:1597-1616, INFRUpdateCU_R NU:1630-1639).
// m: [G][N1][N0][B] float, rhat: same layout float2.
// per_group = N1*N0*B elements.
__global__ void k_update(float *__restrict__ m, const float2 *__restrict__ rhat, const double *__restrict__ alpha,
                         int B, size_t per_group, size_t total, int clamp, int data_type, float thr)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int sl = (int)(i / per_group) * B + (int)(i % B);
        float v = (float)((double)m[i] - alpha[sl] * (double)rhat[i].x);
        if (clamp) {
            if (data_type == 1) {
                if (v > thr) v = thr;
            } else {
                if (v < thr) v = thr;
            }
        }
        m[i] = v;
    }
}

}  // namespace icon
