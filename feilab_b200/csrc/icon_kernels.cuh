// icon_kernels.cuh -- the sm_100a kernels of the ICON hot path.
//
// The reference (ICON-GPU v1.2.9, NU = nufft_gpu_v8.cu) computes a NUFFT as
// pre-pass -> full 2-D cuFFT of the n0 x n1 grid -> interpolation (forward), or
// CSR gather onto the grid -> 2-D cuFFT -> crop (adjoint), one slice at a time.
// Here a group of B slices moves through two FFT passes whose far ends are
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
//   adjoint   K2T ypass_adj   per (row x, group): every buffer row gathers
//                             the window entries covering it (sorted, no
//                             atomics), inverse FFT along y, keep the N1 rows
//                             the crop keeps -> G1[x][Y][b]
//             K1T xpass_adj   per (column Y, group): inverse FFT along x,
//                             crop, divide by the deapodisation
//                             (+ r = fhat - Ahwb and ||r||^2 partial sums)
//
// Rows of the y-pass are held in shared memory rotated by n1/2, so that the
// unwrapped tap position u = iy0 + t1 in [-n1/2-6, n1/2+6] is row u + n1/2 of
// the buffer, with 8 halo rows on each side (copies of the other end); no tap
// needs a modulo.  The rotation costs nothing: multiplying the FFT input by
// (-1)^y shifts its output by n1/2, and an input rotated by n1/2 gives the
// output times (-1)^k.
#pragma once
#include "icon_device.cuh"
#include "ws_tc.cuh"

namespace icon {

constexpr int kHalo = 8;      // halo rows on each side of a rotated row buffer
constexpr int kLdPhiy = 16;   // phiy rows padded to 16 floats (four 16-byte loads)

// Device view of one tilt-series geometry (all pointers are device memory).
struct Geo {
    int N0, N1, n0, n1, lg0, lg1, M, nx, nz, B;
    int tlo, thi;          // taps that can be non-zero: 0..13 (Gaussian), 3..10 (Kaiser-Bessel)
    const float *w;        // [M] density weights (Weight, weight.cu:8-41), group g's at w + g*wstride
    size_t wstride;        // 0: one weight vector for every group; M: one per group
    const float *phix;     // [M][14] window values, x taps   (NU:221-235)
    const float *phiy;     // [M][16] window values, y taps, 2 zero pads
    const int *ix0;        // [M] first x tap, unwrapped: floor(n0*x0) - 6
    const int *iy0;        // [M] first y tap, unwrapped
    const float *cx;       // [N0] deapodisation factor along x (NU:22-42)
    const float *cy;       // [N1] deapodisation factor along y
    const float *rcx;      // [N0] 1/cx, rounded once from double
    const float *rcy;      // [N1] 1/cy
    const int *row_off;    // [n0+1] entry range of every grid row x
    const int *ent_jt;     // [M*14] entry: node*16 + x tap, sorted by (row, iy0, node)
    const int *ent_iy0;    // [M*14] iy0 of the entry's node (sort key within a row)
    const unsigned short *ent_lb;   // [n0][n1+17] per-row lower bounds of r0 (k_ypass_adj)
    const float *ent_phiy; // [M*14][16] phiy of the entry's node, in entry order
    const float *ent_pxy;  // [M*14][16] phix[j][t0] * phiy[j][t1], in entry order
    const float2 *tw0;     // [n0] exp(-2 pi i q / n0)
    const float2 *tw0h;    // [n0/2] exp(-2 pi i q / (n0/2))
    const float2 *tw1;     // [n1] exp(-2 pi i q / n1)
    const float *Kt;       // [n0][n1] Toeplitz kernel of A^H W A, group g's at Kt + kidx[g]*kstride
    size_t kstride;        // 0: one kernel for every group; n0*n1: one per distinct weight set
    const int *kidx;       // [G] kernel of each group (per-group weights), or null

};

// 1-D row-transform tables (cunfft_initPlan_1d, NU:1298-1391).
struct Geo1 {
    const float *phi1;     // [nx][14]
    const int *i10;        // [nx] first tap, unwrapped, nondecreasing in k
};

#ifndef ICON_KERNELS_TEMPLATES_ONLY
// ------------------------------------------------------------- tables ----
// Window taps exactly as nufft_Phi2d_1dCU (NU:221-235) computes them, in float:
// l = floor(n*x) - m + t, x1 = x - l/n, phi = bf*exp(-(n*x1)^2/b).  Rows of
// ld >= 14 floats, the pad zeroed.  kb > 0 selects the Kaiser-Bessel window
// of half-width kKbHalf in the same taps (non-zero on taps 3..10 only): with
// u = n*x1 (exact in float, n a power of two),
// phi = sinh(kb sqrt(K^2 - u^2)) / sqrt(K^2 - u^2) * inv for |u| < K, else 0,
// evaluated in double and rounded once (inv = 1/(pi I0(kb K))).
__global__ void k_window(const float *__restrict__ x, int stride, int M, int n, float b, float bf,
                         float *__restrict__ phi, int ld, int *__restrict__ l0out, double kb, double inv)
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
        if (kb > 0.0) {
            const double u = (double)(n * x1);
            const double q = (double)(kKbHalf * kKbHalf) - u * u;
            phi[(size_t)j * ld + t] = q > 0.0 ? (float)(sinh(kb * sqrt(q)) / sqrt(q) * inv) : 0.f;
        } else {
            phi[(size_t)j * ld + t] = bf * expf(-((n * x1) * (n * x1) / b));
        }
    }
    for (int t = kTaps; t < ld; ++t) phi[(size_t)j * ld + t] = 0.f;
}

// Window values copied into entry order (entry e = node j, x tap t0), so the
// y-passes read them as contiguous streams: ephiy[e] = phiy[j] (16 floats)
// and epxy[e][t1] = phix[j][t0] * phiy[j][t1], the product the reference's
// adjoint CSR stores per grid point and node (NU:44-218).
__global__ void k_entry_tables(const int *__restrict__ jt, int E, const float *__restrict__ phiy,
                               const float *__restrict__ phix, float *__restrict__ ephiy, float *__restrict__ epxy)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    int v = jt[e], j = v >> 4, t0 = v & 15;
    const float px = phix[(size_t)j * kTaps + t0];
#pragma unroll
    for (int t = 0; t < kLdPhiy; ++t) {
        float py = phiy[(size_t)j * kLdPhiy + t];
        ephiy[(size_t)e * kLdPhiy + t] = py;
        epxy[(size_t)e * kLdPhiy + t] = px * py;
    }
}

#endif  // ICON_KERNELS_TEMPLATES_ONLY

// Which Toeplitz kernel slice group grp uses: groups with equal weights share one.
__device__ __forceinline__ size_t toep_kernel_index(const Geo &g, int grp)
{
    return g.kidx ? (size_t)__ldg(&g.kidx[grp]) : (size_t)grp;
}

// Loads B consecutive float2 (16-byte vector loads when B is even).
template <int B>
__device__ __forceinline__ void load_b(const float2 *__restrict__ p, float2 (&v)[B])
{
    if constexpr (B % 2 == 0) {
#pragma unroll
        for (int i = 0; i < B / 2; ++i) {
            float4 t = reinterpret_cast<const float4 *>(p)[i];
            v[2 * i] = make_float2(t.x, t.y);
            v[2 * i + 1] = make_float2(t.z, t.w);
        }
    } else {
#pragma unroll
        for (int i = 0; i < B; ++i) v[i] = p[i];
    }
}

template <int B>
__device__ __forceinline__ void store_b(float2 *__restrict__ p, const float2 (&v)[B])
{
    if constexpr (B % 2 == 0) {
#pragma unroll
        for (int i = 0; i < B / 2; ++i)
            reinterpret_cast<float4 *>(p)[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
    } else {
#pragma unroll
        for (int i = 0; i < B; ++i) p[i] = v[i];
    }
}

// Launch bound of the FFT kernels: blockDim = n*B/E <= 512 threads for E = 32
// (so up to 128 registers), <= 1024 for E = 16.
#define FFT_BOUNDS(E) __launch_bounds__((E) == 32 ? 512 : 1024)

// --------------------------------------------------------------- K1 ----
// Forward x-pass.  in: [G][N1][N0][B] real (m) or complex; out G1 [G][n0][N1][B].
// Pre-pass of NU:784-809 / NU:754-781: grid x holds img[X]/ck(X,Y) with
// X = (x + N0/2) % n0 when X < N0, else 0; ck = cx[X]*cy[Y] (the division is
// a multiplication by the reciprocals, within 2 ulp of the reference's
// quotient).  The first FFT pass reads the image column directly, the last
// writes G1.
template <bool REAL_IN, int B, int E, bool FULL = false>
__global__ void FFT_BOUNDS(E) k_xpass_fwd(Geo g, const void *__restrict__ in, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    const int Y = blockIdx.x, grp = blockIdx.y, n = g.n0, N0 = g.N0, N1 = g.N1;
    const float rcyY = g.rcy[Y];
    const float *rcx = g.rcx;
    const size_t ibase = ((size_t)grp * N1 + Y) * N0 * B;
    float2 *out = G1 + (size_t)grp * n * N1 * B + (size_t)Y * B;
    // Copy the column [N0][B] (contiguous in global memory) and 1/cx behind
    // it; the first FFT pass reads both, deapodising as it reads, before
    // anything is written to s.
    const size_t vbytes = REAL_IN ? sizeof(float) : sizeof(float2);
    char *raw = reinterpret_cast<char *>(s);
    float *rcs = reinterpret_cast<float *>(raw + (((size_t)N0 * B * vbytes + 15) & ~(size_t)15));
    copy_async(raw, (const char *)in + ibase * vbytes, (size_t)N0 * B * vbytes);
    copy_async(rcs, rcx, (size_t)N0 * sizeof(float));
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    auto ld = [=](int x, int b) -> float2 {
        int X = (x + N0 / 2) & (n - 1);
        if (X >= N0) return make_float2(0.f, 0.f);
        float r = rcs[X] * rcyY;
        if (REAL_IN) return make_float2(reinterpret_cast<const float *>(raw)[X * B + b] * r, 0.f);
        float2 v = reinterpret_cast<const float2 *>(raw)[X * B + b];
        return make_float2(v.x * r, v.y * r);
    };
    // A real image's rows n0/2+1.. are the conjugates of rows n0/2-1..1;
    // the forward y-pass (HERM) reads rows 0..n0/2 only (FULL: all rows).
    auto st = [=](int x, int b, float2 v) {
        if (!REAL_IN || FULL || x <= (n >> 1)) out[(size_t)x * N1 * B + b] = v;
    };
    fft_fused<B, B, E>(s, n, g.lg0, g.tw0, -1.f, ld, st);
}

// Forward x-pass of a real image (the reference's R2C transform,
// NU:984-1076) with half-length FFTs: the n0 real values x(t) of a slice's
// column are packed as z(m) = x(2m) + i x(2m+1), m < N = n0/2, one FFT of
// length N per slice (blockDim = N*B/E), and with Z = FFT(z), W = exp(-2 pi i/n0):
//   X(k) = (Z(k) + conj Z(N-k)) / 2 - i W^k (Z(k) - conj Z(N-k)) / 2,
// indices of Z mod N, written for k = 0..n0/2 (the rows the Hermitian y-pass
// reads) and, with FULL, also for k = n0/2+1..n0-1 as the conjugates
// X(n0 - k)* (the Toeplitz y-pass takes every row).  Each slice stays its own
// transform, so results do not depend on which slices share a group.
template <int B, int E, bool FULL = false>
__global__ void FFT_BOUNDS(E) k_xpass_fwd_r2c(Geo g, const float *__restrict__ in, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    const int Y = blockIdx.x, grp = blockIdx.y, n = g.n0, N = g.n0 / 2, N0 = g.N0, N1 = g.N1;
    const float rcyY = g.rcy[Y];
    const size_t ibase = ((size_t)grp * N1 + Y) * N0 * B;
    float2 *out = G1 + (size_t)grp * n * N1 * B + (size_t)Y * B;
    // The column [N0][B] and 1/cx, read by the first FFT pass before it
    // writes s (N0 <= n0/2, so both fit in the N*B*8 bytes of s).
    char *raw = reinterpret_cast<char *>(s);
    float *rcs = reinterpret_cast<float *>(raw + (((size_t)N0 * B * sizeof(float) + 15) & ~(size_t)15));
    copy_async(raw, in + ibase, (size_t)N0 * B * sizeof(float));
    copy_async(rcs, g.rcx, (size_t)N0 * sizeof(float));
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const float *rin = reinterpret_cast<const float *>(raw);
    auto xval = [=](int t, int b) -> float {
        int X = (t + N0 / 2) & (n - 1);
        return X < N0 ? rin[X * B + b] * (rcs[X] * rcyY) : 0.f;
    };
    auto ld = [=](int m, int b) -> float2 { return make_float2(xval(2 * m, b), xval(2 * m + 1, b)); };
    auto st = [=](int k, int b, float2 v) { s[k * B + b] = v; };
    fft_fused<B, B, E>(s, N, g.lg0 - 1, g.tw0h, -1.f, ld, st);
    __syncthreads();
    for (int idx = threadIdx.x; idx < (N + 1) * B; idx += blockDim.x) {
        const int k = idx / B, b = idx - k * B;
        const float2 zk = s[(k & (N - 1)) * B + b], zm = s[((N - k) & (N - 1)) * B + b];
        const float2 fe = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 fo = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 w = __ldg(&g.tw0[k]);
        const float2 v = cadd(fe, cmul(w, fo));
        out[(size_t)k * N1 * B + b] = v;
        if (FULL && k > 0 && k < N) out[(size_t)(n - k) * N1 * B + b] = make_float2(v.x, -v.y);
    }
}

// Copies the wrap-around halo rows of a rotated row buffer (rows 0..7 and
// n+8..n+15 of s[(n + 16)][SB]).
template <int B, int SB>
__device__ __forceinline__ void fill_halo(float2 *s, int n)
{
    constexpr int LB = Log2B<B>::v;
    for (int idx = threadIdx.x; idx < kHalo * B; idx += blockDim.x) {
        int b = idx & (B - 1), i = idx >> LB;
        s[i * SB + b] = s[(i + n) * SB + b];
        s[(n + kHalo + i) * SB + b] = s[(kHalo + i) * SB + b];
    }
}

// --------------------------------------------------------------- K2 ----
// Entries of a row whose tables k_ypass_fwd copies into shared memory before
// its FFT (the copy overlaps the FFT); one record is the phiy window (16
// floats), the node*16 + x tap and iy0.
constexpr int kPreEntries = 256;
constexpr int kPreRecord = kLdPhiy * 4 + 8;
__host__ __device__ inline size_t ypass_fwd_pre_bytes() { return (size_t)kPreEntries * kPreRecord; }

// The y-passes copy the FFT's twiddle table (n1 float2) into shared memory
// when it fits beside their buffers (n1 <= 2048); longer rows read it from
// global memory.
__host__ __device__ inline bool ypass_tw_shared(int n1) { return n1 <= 2048; }
__host__ __device__ inline size_t ypass_tw_bytes(int n1) { return ypass_tw_shared(n1) ? (size_t)n1 * 8 : 0; }

// Row stride (float2) of k_ypass_fwd's rotated row buffer: unpadded for
// B = 8 (64-byte rows; the interpolation reads pairs of rows as 128-byte
// blocks, conflict-free), the padded RowStride otherwise.
template <int B>
struct YfStride {
    static constexpr int v = (B == 8) ? 8 : RowStride<B>::v;
};
__host__ __device__ inline size_t ypass_fwd_smem(int n1, int B)
{
    size_t sb = (B == 8) ? 8 : (B == 4) ? 6 : B;
    return (size_t)(n1 + 2 * kHalo) * sb * sizeof(float2) + ypass_fwd_pre_bytes() + ypass_tw_bytes(n1);
}

// Forward y-pass fused with the y-direction interpolation.  Row x of G1 holds
// the N1 nonzero columns; column Y sits at y with (y + N1/2) % n1 == Y.
// P[G][M][14][B]: P[j][t0] = sum_t1 phiy[j][t1] * G[x][(iy0_j + t1) mod n1],
// x = (ix0_j + t0) mod n0.  (NU:669-727 sum the same 196 products per node.)
// The row is copied to shared memory and the tables of the row's first
// entries are copied behind it; the FFT waits only for the row.  One thread
// per entry then computes all B slices of it from the rotated row; entries
// past the copied ones are loaded one round ahead.
//
// HERM (the forward transform of a real image, cunfft_trafo_2d_R2C2,
// NU:984-1076, whose cuFFT R2C keeps half the spectrum): G1 row n0 - x is the
// conjugate of row x, so its FFT along y is the conjugate mirror of row x's,
// buf'[q] = conj(buf[-q mod n1]).  The grid then covers rows x = 0..n0/2
// only; each CTA also interpolates the entries of row n0 - x, reading the 14
// taps of an entry from the mirrored window in reverse order and storing the
// conjugate of the sum.  The x-pass writes only rows 0..n0/2 of G1.
template <int B, int E, bool HERM>
__global__ void FFT_BOUNDS(E) k_ypass_fwd(Geo g, const float2 *__restrict__ G1, float2 *__restrict__ P)
{
    extern __shared__ float2 s[];
    constexpr int SB = YfStride<B>::v;
    constexpr bool kPairs = (B == 8);   // 64-byte rows read as 128-byte row pairs
    const int grp = blockIdx.x, x = blockIdx.y, n = g.n1, N1 = g.N1;
    const int xp = (g.n0 - x) & (g.n0 - 1);   // the mirror row (HERM)
    const int T = blockDim.x;
    const float2 *rowin = G1 + ((size_t)grp * g.n0 + x) * N1 * B;
    float2 *row = s + kHalo * SB;
    float *pre_phi = reinterpret_cast<float *>(s + (size_t)(n + 2 * kHalo) * SB);   // [kPreEntries][16]
    int *pre_jt = reinterpret_cast<int *>(pre_phi + kPreEntries * kLdPhiy);           // [kPreEntries]
    int *pre_iy = pre_jt + kPreEntries;                                                 // [kPreEntries]
    float2 *tw_s = reinterpret_cast<float2 *>(pre_iy + kPreEntries);                    // [n] twiddles
    const float2 *tws = ypass_tw_shared(n) ? tw_s : g.tw1;
    // Entries: row x's (ca of them), then with HERM and xp != x the mirror
    // row's (cb); i-th entry of the combined list at global index ent(i).
    const int ea = g.row_off[x], ca = g.row_off[x + 1] - ea;
    const int eb = (HERM && xp != x) ? g.row_off[xp] : 0;
    const int cb = (HERM && xp != x) ? g.row_off[xp + 1] - eb : 0;
    const int cnt = ca + cb;
    auto ent = [=](int i) { return i < ca ? ea + i : eb + (i - ca); };
    const int staged = min(cnt, min(T, kPreEntries));
    // Group 1: the N1 nonzero values of the row (contiguous in G1) and the
    // FFT's twiddle table.
    copy_async(row, rowin, (size_t)N1 * B * sizeof(float2));
    if (ypass_tw_shared(n)) copy_async(tw_s, g.tw1, (size_t)n * sizeof(float2));
    cp_async_commit();
    // Group 2: tables of the first entries.
    if ((int)threadIdx.x < staged) {
        const int e = ent(threadIdx.x);
        const float *src = g.ent_phiy + (size_t)e * kLdPhiy;
        float *dst = pre_phi + threadIdx.x * kLdPhiy;
#pragma unroll
        for (int q = 0; q < kLdPhiy / 4; ++q) cp_async<16>(dst + 4 * q, src + 4 * q);
        cp_async<4>(pre_jt + threadIdx.x, g.ent_jt + e);
        cp_async<4>(pre_iy + threadIdx.x, g.ent_iy0 + e);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    auto ld = [=](int y, int b) -> float2 {
        int Y = (y + N1 / 2) & (n - 1);
        float2 v = (Y < N1) ? row[Y * B + b] : make_float2(0.f, 0.f);
        return (y & 1) ? make_float2(-v.x, -v.y) : v;      // rotates the output by n/2
    };
    auto st = [=](int q, int b, float2 v) { row[q * SB + b] = v; };
    fft_fused<B, SB, E, false, kPairs, true>(row, n, g.lg1, tws, -1.f, ld, st);
    cp_async_wait<0>();
    __syncthreads();
    fill_halo<B, SB>(s, n);
    __syncthreads();
    const size_t pbase = (size_t)grp * g.M * kTaps * B;
    const int rofs = n / 2 + kHalo;
    struct Ent {
        int jt, iy;
        float4 py[4];
    };
    auto load_global = [&](int e, Ent &r) {
        r.jt = __ldg(&g.ent_jt[e]);
        r.iy = __ldg(&g.ent_iy0[e]);
        const float4 *py4 = reinterpret_cast<const float4 *>(g.ent_phiy + (size_t)e * kLdPhiy);
#pragma unroll
        for (int q = 0; q < 4; ++q) r.py[q] = __ldg(&py4[q]);
    };
    int i = threadIdx.x;
    Ent cur, nxt;
    if (i < staged) {
        cur.jt = pre_jt[i];
        cur.iy = pre_iy[i];
        const float4 *py4 = reinterpret_cast<const float4 *>(pre_phi + i * kLdPhiy);
#pragma unroll
        for (int q = 0; q < 4; ++q) cur.py[q] = py4[q];
    } else if (i < cnt) {
        load_global(ent(i), cur);
    }
    while (i < cnt) {
        const int i2 = i + T;             // never among the copied entries (staged <= T)
        if (i2 < cnt) load_global(ent(i2), nxt);
        const int j = cur.jt >> 4, t0 = cur.jt & 15;
        // A mirror-row entry's tap t1 is buffer row rm - t1, rm = n1/2 - iy0
        // + kHalo: the window starts at rm - 13 and is read in reverse.
        const bool mir = HERM && i >= ca;
        const int r0 = mir ? (n / 2 - cur.iy + kHalo - (kTaps - 1)) : (cur.iy + rofs);
        const float2 *sr = s + r0 * SB;
        float py0[16], py[kTaps];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            py0[4 * q] = cur.py[q].x;
            py0[4 * q + 1] = cur.py[q].y;
            py0[4 * q + 2] = cur.py[q].z;
            py0[4 * q + 3] = cur.py[q].w;
        }
#pragma unroll
        for (int t1 = 0; t1 < kTaps; ++t1) py[t1] = mir ? py0[kTaps - 1 - t1] : py0[t1];
        if constexpr (kPairs) {
            // Taps 2p and 2p+1 are rows r and r+1, one 128-byte block = eight
            // 16-byte chunks (chunk c: row r + c/4, slices 2(c%4), 2(c%4)+1),
            // whose bank slots are (4r + c) % 8.  At step k lane l reads the
            // chunk in slot (l + k) % 8, so the eight lanes of each quarter
            // warp hit eight different slots: no bank conflicts, whatever the
            // rows of the lanes' entries.  acc[k % 4] then always holds the
            // slices of quad (l + k) % 4.
            const int lane8 = threadIdx.x & 7;
            const char *rb = reinterpret_cast<const char *>(s) + (size_t)r0 * (SB * sizeof(float2));
            const int o = lane8 + ((r0 & 1) << 2);
            float4 acc[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int pr = 0; pr < kTaps / 2; ++pr) {
                if (2 * pr + 1 < g.tlo || 2 * pr > g.thi) continue;   // both taps zero (Kaiser-Bessel)
                const float wa = py[2 * pr], wb = py[2 * pr + 1];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int c = (o + k) & 7;
                    const float4 v = *reinterpret_cast<const float4 *>(rb + pr * 128 + c * 16);
                    const float w = (c & 4) ? wb : wa;
                    const float2 ww = make_float2(w, w);
                    float4 &a = acc[k & 3];
                    const float2 lo = fma2(make_float2(v.x, v.y), ww, make_float2(a.x, a.y));
                    const float2 hi = fma2(make_float2(v.z, v.w), ww, make_float2(a.z, a.w));
                    a = make_float4(lo.x, lo.y, hi.x, hi.y);
                }
            }
            float4 *dst = reinterpret_cast<float4 *>(P + pbase + ((size_t)j * kTaps + t0) * B);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (mir) acc[k] = make_float4(acc[k].x, -acc[k].y, acc[k].z, -acc[k].w);
                dst[(lane8 + k) & 3] = acc[k];
            }
        } else {
            float2 acc[B];
#pragma unroll
            for (int b = 0; b < B; ++b) acc[b] = make_float2(0.f, 0.f);
#pragma unroll
            for (int t1 = 0; t1 < kTaps; ++t1) {
                if (t1 < g.tlo || t1 > g.thi) continue;   // zero tap (Kaiser-Bessel)
                float2 v[B];
                load_b<B>(sr + t1 * SB, v);
#pragma unroll
                for (int b = 0; b < B; ++b) {
                    acc[b].x = fmaf(v[b].x, py[t1], acc[b].x);
                    acc[b].y = fmaf(v[b].y, py[t1], acc[b].y);
                }
            }
            if (mir) {
#pragma unroll
                for (int b = 0; b < B; ++b) acc[b].y = -acc[b].y;
            }
            store_b<B>(P + pbase + ((size_t)j * kTaps + t0) * B, acc);
        }
        cur = nxt;
        i = i2;
    }
}

// --------------------------------------------------------------- K3 ----
// f_j = sum_t0 phix[j][t0] * P[j][t0].  MODE 0: store f.  MODE 1: store
// f*w (complexMulDoubleCU, NU:1539-1549).  MODE 2: store nothing; per-slice
// partial sums of w*|f|^2 in double (alpha1, NU:1652-1661) into
// part[G][gridDim.x][B].
template <int MODE, int B>
__global__ void k_interp_fin(Geo g, const float2 *__restrict__ P, float2 *__restrict__ f, double *__restrict__ part)
{
    __shared__ double red[256];
    constexpr int LB = Log2B<B>::v;
    const int grp = blockIdx.y;
    const int item = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = item >> LB, b = item & (B - 1);
    double acc2 = 0.0;
    if (j < g.M) {
        const float *px = g.phix + (size_t)j * kTaps;
        const float2 *pp = P + ((size_t)grp * g.M + j) * kTaps * B + b;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t0 = 0; t0 < kTaps; ++t0) {
            if (t0 < g.tlo || t0 > g.thi) continue;   // taps without entries (Kaiser-Bessel)
            float2 v = pp[(size_t)t0 * B];
            float p = __ldg(&px[t0]);
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        if (MODE == 0) {
            f[((size_t)grp * g.M + j) * B + b] = acc;
        } else if (MODE == 1) {
            float w = __ldg(&g.w[(size_t)grp * g.wstride + j]);
            f[((size_t)grp * g.M + j) * B + b] = make_float2(acc.x * w, acc.y * w);
        } else {
            double w = (double)__ldg(&g.w[(size_t)grp * g.wstride + j]);
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

// Index of the first of the sorted keys key[lo..hi) that is >= v (shared memory).
__device__ __forceinline__ int lower_bound_s(const int *key, int lo, int hi, int v)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (key[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Entries of a row staged at a time by the adjoint gather, and the padded
// stride of a staged phiy window (so that neighbouring windows fall in
// different shared-memory banks).
constexpr int kChunk = 304;
constexpr int kLdPs = 20;

// Entries of grid row x whose first y tap r0 (in the rotated buffer with a
// halo of kHalo rows on each side, r0 = iy0 + n1/2 + kHalo) is below v, for
// v = 0..n1+16: [x][lb_ld] counts relative to the row's first entry, rows
// padded to 16 bytes.
__host__ __device__ inline int lb_ld(int n1) { return (n1 + 2 * kHalo + 1 + 7) & ~7; }

// Shared-memory layout of k_ypass_adj.  Two chunk buffers of staged entries
// (f values, phix*phiy window, iy0) and the row's lower-bound table are live
// while the rows are gathered into registers; the rotated row (padded
// stride) is written after the last chunk and shares the same bytes.
__host__ __device__ inline size_t ypass_adj_chunk_bytes(int B)
{
    size_t sb = (B == 8) ? 10 : (B == 4) ? 6 : B;
    return (size_t)kChunk * (sb * sizeof(float2) + kLdPs * sizeof(float) + sizeof(int));
}
__host__ __device__ inline size_t ypass_adj_region(int n1, int B)
{
    size_t sb = (B == 8) ? 10 : (B == 4) ? 6 : B;
    size_t row = (size_t)n1 * sb * sizeof(float2);
    size_t gather = 2 * ypass_adj_chunk_bytes(B) + (((size_t)lb_ld(n1) * sizeof(unsigned short) + 15) & ~(size_t)15);
    return row > gather ? row : gather;
}
// The region above plus the FFT's twiddle table behind it.
__host__ __device__ inline size_t ypass_adj_smem(int n1, int B)
{
    return ypass_adj_region(n1, B) + ypass_tw_bytes(n1);
}

// Adds the staged entries covering buffer rows i0 .. i0+R-1 (r0 in
// [i0 - 13, i0 + R - 1]) to acc[k] of row i0 + k: entry e puts
// (phix * phiy)_e[i0 + k - r0_e] * f_e on row i0 + k when that tap is in
// 0..13.  Rs holds iy0 (r0 = iy0 + r0ofs); lb is the row's lower-bound
// table (last index lbmax) and off the index of the chunk's first entry.
template <int B, int SB, int R>
__device__ __forceinline__ void gather_rows(int i0, int r0ofs, const unsigned short *lb, int lbmax, int off, int cn,
                                            const float2 *Qs, const float *Ps, const int *Rs, float2 (&acc)[R][B],
                                            int tlo, int thi)
{
    // lb[lbmax] counts every entry of the row, so clamping an index past it
    // (alias ranges of wide thread strips) is exact.  Only taps tlo..thi of a
    // window can be non-zero, so the entries with r0 in [i0 - thi, i0 + R - 1 - tlo]
    // are the ones that reach these rows.
    int lo = min(max((int)lb[min(max(i0 - thi, 0), lbmax)] - off, 0), cn);
    int hi = min(max((int)lb[min(max(i0 + R - tlo, 0), lbmax)] - off, 0), cn);
    const int iu = i0 - r0ofs;
    for (int e = lo; e < hi; ++e) {
        const int t0 = iu - Rs[e];        // tap of row i0; row i0 + k uses t0 + k
        const float *pe = Ps + e * kLdPs;
        float p[R];
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = ((unsigned)(t0 + k) < (unsigned)kTaps) ? pe[t0 + k] : 0.f;
        float2 q[B];
        load_b<B>(Qs + e * SB, q);
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const float2 pp = make_float2(p[k], p[k]);
#pragma unroll
            for (int b = 0; b < B; ++b) acc[k][b] = fma2(q[b], pp, acc[k][b]);
        }
    }
}


// -------------------------------------------------------------- K2T ----
// Adjoint y-pass.  Entry e (node j, x tap t0) of row x adds
// phiy[j][t1] * phix[j][t0] * f_j to the rotated buffer row r0_e + t1,
// t1 = 0..13; the reference sums the same terms per grid point through its
// host-built CSR (NU:1078-1102).  Here a thread owns whole buffer rows and
// gathers: entries are sorted by r0, so those covering row i are the
// contiguous range r0 in [i - 13, i], read from the precomputed lower-bound
// table.  The 8 halo rows on each side alias rows n-8..n-1 and 0..7, so
// those rows also gather the range of their alias.  Entries are copied in
// chunks with cp.async (f_j, the phix*phiy window, iy0), the next chunk in
// flight while the current one is gathered; a thread keeps its rows' sums in
// registers across chunks, so every row gets its terms in a fixed order, with
// no atomics.  The sums then go to the rotated row buffer and the inverse FFT
// along y (NU:1203) reads the rotated row, and its last pass writes the rows
// Y < N1 of the crop (NU:1104-1121: y = (Y + n1 - N1/2) % n1) straight to
// G1[x][Y][b].  blockDim.x is max(32, n1*B/E); GUARD when that is more than
// the FFT's n1*B/E threads.
template <int B, int E, bool GUARD>
__global__ void FFT_BOUNDS(E) k_ypass_adj(Geo g, const float2 *__restrict__ f, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    constexpr int SB = RowStride<B>::v;
    constexpr int R = E / B;               // rows per thread: thread t owns rows t + k*T, k < R
    const int grp = blockIdx.x, x = blockIdx.y, n = g.n1, N1 = g.N1;
    char *const base = reinterpret_cast<char *>(s);
    const size_t cbytes = ypass_adj_chunk_bytes(B);
    unsigned short *lb = reinterpret_cast<unsigned short *>(base + 2 * cbytes);
    const int e0 = g.row_off[x], cnt = g.row_off[x + 1] - e0;
    const float2 *fg = f + (size_t)grp * g.M * B;
    const int T = blockDim.x, ldl = lb_ld(n);
    const int r0ofs = n / 2 + kHalo;
    const int nch = (cnt + kChunk - 1) / kChunk;
    // Chunk c lives in buffer c & 1: Qs [kChunk][SB], Ps [kChunk][kLdPs], Rs [kChunk].
    auto bufQ = [&](int c) { return reinterpret_cast<float2 *>(base + (c & 1) * cbytes); };
    auto bufP = [&](int c) { return reinterpret_cast<float *>(bufQ(c) + kChunk * SB); };
    auto bufR = [&](int c) { return reinterpret_cast<int *>(bufP(c) + kChunk * kLdPs); };
    auto issue = [&](int c) {
        const int c0 = e0 + c * kChunk, cn = min(kChunk, e0 + cnt - c0);
        float2 *Qs = bufQ(c);
        float *Ps = bufP(c);
        int *Rs = bufR(c);
        for (int i = threadIdx.x; i < cn; i += T) {
            const int j = __ldg(&g.ent_jt[c0 + i]) >> 4;
            const float2 *src = fg + (size_t)j * B;
            if constexpr (B >= 2) {
#pragma unroll
                for (int q = 0; q < B / 2; ++q) cp_async<16>(Qs + i * SB + 2 * q, src + 2 * q);
            } else {
                cp_async<8>(Qs + i * SB, src);
            }
            const float *pxy = g.ent_pxy + (size_t)(c0 + i) * kLdPhiy;
#pragma unroll
            for (int q = 0; q < kLdPhiy / 4; ++q) cp_async<16>(Ps + i * kLdPs + 4 * q, pxy + 4 * q);
            cp_async<4>(Rs + i, g.ent_iy0 + c0 + i);
        }
        cp_async_commit();
    };
    // Thread t owns NS strips of RS consecutive rows, strip t + k*T starting
    // at row RS*(t + k*T); one gather of a strip loads each covering entry
    // once for its RS rows.
    constexpr int RS = (B == 8 && R % 2 == 0) ? 2 : 1;
    constexpr int NS = R / RS;
    float2 acc[NS][RS][B];
#pragma unroll
    for (int k = 0; k < NS; ++k)
#pragma unroll
        for (int j = 0; j < RS; ++j)
#pragma unroll
            for (int b = 0; b < B; ++b) acc[k][j][b] = make_float2(0.f, 0.f);
    float2 *tw_s = reinterpret_cast<float2 *>(base + ypass_adj_region(n, B));   // [n] twiddles
    const float2 *tws = ypass_tw_shared(n) ? tw_s : g.tw1;
    if (ypass_tw_shared(n)) copy_async(tw_s, g.tw1, (size_t)n * sizeof(float2));
    cp_async_commit();
    if (nch > 0) {
        copy_async(lb, g.ent_lb + (size_t)x * ldl, (size_t)ldl * sizeof(unsigned short));
        issue(0);
    }
    for (int c = 0; c < nch; ++c) {
        cp_async_wait<0>();
        __syncthreads();                  // chunk c landed; chunk c-1's buffer is free
        if (c + 1 < nch) issue(c + 1);
        const int off = c * kChunk, cn = min(kChunk, cnt - off);
        const float2 *Qs = bufQ(c);
        const float *Ps = bufP(c);
        const int *Rs = bufR(c);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const int r = RS * (threadIdx.x + k * T);
            if (r < n) {
                gather_rows<B, SB, RS>(r + kHalo, r0ofs, lb, ldl - 1, off, cn, Qs, Ps, Rs, acc[k], g.tlo, g.thi);
                // Rows 0..7 and n-8..n-1 also take the halo rows that alias
                // them (kHalo is a multiple of RS, so no strip straddles).
                if (r < kHalo)
                    gather_rows<B, SB, RS>(r + kHalo + n, r0ofs, lb, ldl - 1, off, cn, Qs, Ps, Rs, acc[k], g.tlo, g.thi);
                if (r >= n - kHalo)
                    gather_rows<B, SB, RS>(r + kHalo - n, r0ofs, lb, ldl - 1, off, cn, Qs, Ps, Rs, acc[k], g.tlo, g.thi);
            }
        }
    }
    cp_async_wait<0>();                   // the twiddles (rows without entries wait here)
    __syncthreads();                      // the row buffer reuses the chunk buffers
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const int r = RS * (threadIdx.x + k * T);
        if (r < n) {
#pragma unroll
            for (int j = 0; j < RS; ++j) store_b<B>(s + (size_t)(r + j) * SB, acc[k][j]);
        }
    }
    __syncthreads();
    float2 *row = s;
    float2 *out = G1 + ((size_t)grp * g.n0 + x) * N1 * B;
    auto ld = [=](int q, int b) -> float2 { return row[q * SB + b]; };
    auto st = [=](int kq, int b, float2 v) {
        int Y = (kq + N1 / 2) & (n - 1);
        if (Y < N1) out[(size_t)Y * B + b] = (kq & 1) ? make_float2(-v.x, -v.y) : v;   // undoes the rotation
    };
    fft_fused<B, SB, E, GUARD, false, true>(row, n, g.lg1, tws, +1.f, ld, st);
}

// -------------------------------------------------------------- K1T ----
// Adjoint x-pass: inverse FFT along x of column Y (first pass reads G1), and
// the last pass crops X < N0 with x = (X + n0 - N0/2) % n0 and divides by
// ck = cx[X]*cy[Y] (NU:1104-1121).  MODE 0: out = fhat.  MODE 1: out = fhat -
// Ahwb (complexMinusCU, NU:1563-1573) and per-slice partial sums of |out|^2 in
// double (alpha0, NU:1641-1650) into part[G][N1][B].  out/Ahwb: [G][N1][N0][B].
template <int MODE, int B, int E>
__global__ void FFT_BOUNDS(E) k_xpass_adj(Geo g, const float2 *__restrict__ G1, float2 *__restrict__ out,
                                          const float2 *__restrict__ Ahwb, double *__restrict__ part)
{
    extern __shared__ float2 s[];
    double *red = (double *)(s + (size_t)g.n0 * B);
    const int Y = blockIdx.x, grp = blockIdx.y, n = g.n0, N0 = g.N0, N1 = g.N1;
    const float2 *colin = G1 + (size_t)grp * n * N1 * B + (size_t)Y * B;
    const float rcyY = g.rcy[Y];
    const float *rcx = g.rcx;
    const size_t obase = ((size_t)grp * N1 + Y) * N0 * B;
    // Column Y of G1: B values per x, n0 rows N1*B apart.
    if constexpr (B >= 2) {
        constexpr int C = B / 2;                      // 16-byte pieces per x
        for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
            int xq = idx / C, c = idx - xq * C;
            cp_async<16>(s + xq * B + 2 * c, colin + (size_t)xq * N1 * B + 2 * c);
        }
    } else {
        for (int xq = threadIdx.x; xq < n; xq += blockDim.x) cp_async<8>(s + xq, colin + (size_t)xq * N1);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    auto ld = [=](int xq, int b) -> float2 { return s[xq * B + b]; };
    struct Crop {
        const float *rcx;
        float rcyY;
        int n, N0;
        size_t obase;
        const float2 *Ahwb;
        float2 *out;
        double acc2;
        __device__ __forceinline__ void operator()(int k, int b, float2 v)
        {
            int X = (k + N0 / 2) & (n - 1);
            if (X < N0) {
                float r = rcx[X] * rcyY;
                v.x = v.x * r;
                v.y = v.y * r;
                size_t o = obase + (size_t)X * B + b;
                if (MODE == 1) {
                    float2 a = Ahwb[o];
                    v.x = v.x - a.x;
                    v.y = v.y - a.y;
                    acc2 += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
                }
                out[o] = v;
            }
        }
    } st{rcx, rcyY, n, N0, obase, Ahwb, out, 0.0};
    fft_fused<B, B, E>(s, n, g.lg0, g.tw0, +1.f, ld, st);
    const double acc2 = st.acc2;
    if (MODE == 1) {
        double r = block_sum_per_slice(acc2, red, B);
        if ((int)threadIdx.x < B) part[((size_t)grp * N1 + Y) * B + threadIdx.x] = r;
    }
}

// ------------------------------------------------------------ rows ----
// Input stage: per (tilt i, group) the 1-D NUFFT of the projection rows
// (cunfft_trafo_1d NU:1479-1516: pre-pass NU:1432-1452, FFT, interpolation
// NU:1454-1477 with taps summed in order), then f = b*w (NU:1539-1549).
// Row of slice sl for tilt i: rows[sl*sstride + sec*istride .. + nx), with
// sec = i, or i + 1 from tilt `skip` on (a stack section left out).  The
// caller layout [S][nz][nx] is sstride = nz*nx, istride = nx; a tilt stack
// in file order [sections][ny][nx] is sstride = nx, istride = ny*nx.
// f, bout: [G][M][B]; bout may be null.
template <int B, int E>
__global__ void FFT_BOUNDS(E) k_rows_fwd(Geo g, Geo1 g1, const float *__restrict__ rows, size_t sstride,
                                         size_t istride, int skip, int S, float2 *__restrict__ f,
                                         float2 *__restrict__ bout)
{
    extern __shared__ float2 s[];
    constexpr int LB = Log2B<B>::v;
    const int i = blockIdx.x, grp = blockIdx.y, n = g.n0, N = g.nx;
    const float *rcx = g.rcx;
    const float *rowi = rows + (size_t)(i < skip ? i : i + 1) * istride;
    for (int idx = threadIdx.x; idx < N * B; idx += blockDim.x) {
        int b = idx / N, X = idx % N;                      // coalesced along X
        int sl = grp * B + b;
        s[X * B + b] = make_float2(sl < S ? rowi[(size_t)sl * sstride + X] * rcx[X] : 0.f, 0.f);
    }
    __syncthreads();
    auto ld = [=](int x, int b) -> float2 {
        int X = (x + N / 2) & (n - 1);
        return (X < N) ? s[X * B + b] : make_float2(0.f, 0.f);
    };
    auto st = [=](int k, int b, float2 v) { s[k * B + b] = v; };
    fft_fused<B, B, E>(s, n, g.lg0, g.tw0, -1.f, ld, st);
    __syncthreads();
    for (int idx = threadIdx.x; idx < N * B; idx += blockDim.x) {
        int b = idx & (B - 1), k = idx >> LB;
        int l0 = __ldg(&g1.i10[k]);
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t = 0; t < kTaps; ++t) {
            int xq = (l0 + t) & (n - 1);
            float p = __ldg(&g1.phi1[(size_t)k * kTaps + t]);
            float2 v = s[xq * B + b];
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        int j = i * N + k;
        size_t o = ((size_t)grp * g.M + j) * B + b;
        if (bout) bout[o] = acc;
        float w = __ldg(&g.w[(size_t)grp * g.wstride + j]);
        f[o] = make_float2(acc.x * w, acc.y * w);
    }
}

// 1-D adjoint NUFFT of the nx values of one line (cunfft_adjoint_1d,
// NU:1518-1536): gather in node order (the order of the reference's 1-D CSR),
// inverse FFT, crop, divide by the deapodisation, real part.
// f: [G][nx][B]; out: [S][nx] (caller layout).
template <int B, int E>
__global__ void FFT_BOUNDS(E) k_row_adj(Geo g, Geo1 g1, const float2 *__restrict__ f, float *__restrict__ out, int S)
{
    extern __shared__ float2 s[];
    const int grp = blockIdx.x, n = g.n0, N = g.nx;
    const float2 *fg = f + (size_t)grp * N * B;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        float2 acc[B];
#pragma unroll
        for (int b = 0; b < B; ++b) acc[b] = make_float2(0.f, 0.f);
#pragma unroll
        for (int al = 0; al < 2; ++al) {
            int u = x - al * n;
            int a = lower_bound_i(g1.i10, 0, N, u - (kTaps - 1));
            int c = lower_bound_i(g1.i10, a, N, u + 1);
            for (int k = a; k < c; ++k) {
                int d = u - __ldg(&g1.i10[k]);
                float p = __ldg(&g1.phi1[(size_t)k * kTaps + d]);
                float2 v[B];
                load_b<B>(fg + (size_t)k * B, v);
#pragma unroll
                for (int b = 0; b < B; ++b) {
                    acc[b].x = fmaf(v[b].x, p, acc[b].x);
                    acc[b].y = fmaf(v[b].y, p, acc[b].y);
                }
            }
        }
        store_b<B>(s + x * B, acc);
    }
    __syncthreads();
    const float *rcx = g.rcx;
    auto ld = [=](int q, int b) -> float2 { return s[q * B + b]; };
    auto st = [=](int k, int b, float2 v) {
        int X = (k + N / 2) & (n - 1);
        int sl = grp * B + b;
        if (X < N && sl < S) out[(size_t)sl * N + X] = v.x * rcx[X];
    };
    fft_fused<B, B, E>(s, n, g.lg0, g.tw0, +1.f, ld, st);
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

// Batched image [G][N1][N0][B] -> file layout [S][N1][N0] (X fastest, the
// order saveMRC_real_inv writes a slice in, saveMRC_real.cu:49-53).  One
// thread per (Y, X) reads the B values of the point (one 32-byte run for
// B = 8) and writes them to the B slices, each store coalesced along X.
template <int B>
__global__ void k_img_out_file(const float *__restrict__ src, float *__restrict__ dst, int S, int N0, int N1)
{
    const size_t plane = (size_t)N0 * N1;
    const int G = (S + B - 1) / B;
    const size_t total = (size_t)G * plane;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int grp = (int)(i / plane);
        const size_t yx = i - (size_t)grp * plane;
        float v[B];
        if constexpr (B % 4 == 0) {
#pragma unroll
            for (int q = 0; q < B / 4; ++q) {
                float4 t = reinterpret_cast<const float4 *>(src + i * B)[q];
                v[4 * q] = t.x;
                v[4 * q + 1] = t.y;
                v[4 * q + 2] = t.z;
                v[4 * q + 3] = t.w;
            }
        } else {
#pragma unroll
            for (int b = 0; b < B; ++b) v[b] = src[i * B + b];
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int sl = grp * B + b;
            if (sl < S) dst[(size_t)sl * plane + yx] = v[b];
        }
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

#ifndef ICON_KERNELS_TEMPLATES_ONLY
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

// Relative step of the last measured update per slot:
// out[slot] = sqrt(sum (m_new - m_old)^2 / sum m_new^2) over the blocks'
// partial sums step_part[grp][nb][B][2] (fixed order); 0 when m_new = 0.
__global__ void k_step_reduce(const double *__restrict__ step_part, int nb, int B, int slots, double *__restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    const int grp = s / B, b = s % B;
    double d = 0.0, n = 0.0;
    for (int k = 0; k < nb; ++k) {
        const double *p = step_part + (((size_t)grp * nb + k) * B + b) * 2;
        d += p[0];
        n += p[1];
    }
    out[s] = n > 0.0 ? sqrt(d / n) : 0.0;
}

#endif  // ICON_KERNELS_TEMPLATES_ONLY

// m <- m - alpha*Re(rhat) computed in double and stored as float; ICON steps
// also clamp (ICONUpdateCU_R NU:1597-1616, INFRUpdateCU_R NU:1630-1639).
// m: [G][N1][N0][B] float, rhat: same layout float2.  blockIdx.y = group.
__device__ __forceinline__ float re_part(float2 v) { return v.x; }
__device__ __forceinline__ float re_part(float v) { return v; }

// rhat: complex r-hat, or (RT = float) its real part alone.
template <int B, bool MEASURE = false, typename RT = float2>
__global__ void k_update(float *__restrict__ m, const RT *__restrict__ rhat, const double *__restrict__ alpha,
                         int per_group, int clamp, int data_type, float thr, double *__restrict__ step_part = nullptr)
{
    const int grp = blockIdx.y;
    float *mg = m + (size_t)grp * per_group;
    const RT *rg = rhat + (size_t)grp * per_group;
    double dd = 0.0, mm = 0.0;   // MEASURE: sums of (m_new - m_old)^2 and m_new^2 of this thread's slot
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < per_group; i += gridDim.x * blockDim.x) {
        double a = alpha[grp * B + (i & (B - 1))];
        const float old = mg[i];
        float v = (float)((double)old - a * (double)re_part(rg[i]));
        if (clamp) {
            if (data_type == 1) {
                if (v > thr) v = thr;
            } else {
                if (v < thr) v = thr;
            }
        }
        mg[i] = v;
        if (MEASURE) {
            const double d = (double)v - (double)old;
            dd += d * d;
            mm += (double)v * (double)v;
        }
    }
    if (MEASURE) {
        // The grid stride is a multiple of B, so thread t always updates slot
        // t % B: sum the block's threads of each slot in a fixed order into
        // step_part[grp][block][slot][2].
        __shared__ double red[2][256];
        red[0][threadIdx.x] = dd;
        red[1][threadIdx.x] = mm;
        __syncthreads();
        if ((int)threadIdx.x < B) {
            double s0 = 0.0, s1 = 0.0;
            for (int t = threadIdx.x; t < (int)blockDim.x; t += B) {
                s0 += red[0][t];
                s1 += red[1][t];
            }
            double *o = step_part + (((size_t)grp * gridDim.x + blockIdx.x) * B + threadIdx.x) * 2;
            o[0] = s0;
            o[1] = s1;
        }
    }
}

// ------------------------------------------------------------ Toeplitz ----
// The normal operator of the iteration, A^H W A, as a two-dimensional
// convolution.  For the exact transform, (A^H W A m)[X] = sum_X' m[X'] t[X - X']
// with t[d] = sum_j w_j exp(+2 pi i x_j . d) for |d_k| < N_k: a Toeplitz
// matrix.  On the n0 x n1 grid (n_k >= 2 N_k, so the circular convolution of
// the zero-padded image with t is the linear one on the image), with
// unnormalised FFTs F (e^{-2 pi i}) and F^-1 (e^{+2 pi i}):
//   A^H W A m = crop F^-1( K . F(pad m) ),
//   K[k0][k1] = F(t)[k] / (n0 n1)
//             = 1/(n0 n1) sum_j w_j D_N0(x_j0 - k0/n0) D_N1(x_j1 - k1/n1),
// with the Dirichlet kernel D_N(u) = sum_{|d|<N} e^{2 pi i u d}
//                                  = sin(pi u (2N-1)) / sin(pi u)   (2N-1 at integer u).
// K is real.  The step length's denominator sum_j w_j |(A r)_j|^2 is the
// quadratic form r^H A^H W A r = sum_k K[k] |F(pad r)[k]|^2.  The reference
// evaluates both with its Gaussian-window NUFFTs (Iteration2.cu:53-96,
// alpha_new2.cu:26-114); this is the same operator without the window's
// approximation (they differ by the window error, ~1e-6 relative).
//
// K is a sum over the M nodes of rank-one products, computed in double as a
// matrix product: a CTA owns a 64 x 64 tile of K (thread: 4 x 4 entries),
// takes the nodes 32 at a time, evaluates their Dirichlet factors for the
// tile's 64 k0 and 64 k1 into shared memory, and accumulates.  sin(pi u) and
// sin(pi u (2N-1)) at u = x - k/n are formed from per-node and per-k sines
// and cosines by the angle-difference formula; every argument is exact in
// double (x is a float, k/n a dyadic fraction).
constexpr int kToepTile = 64;
constexpr int kToepNodes = 32;

// u = x - k/n is exact in double; at an integer u the angle-difference
// formula leaves rounding noise in both sines, so integers are caught first.
__device__ __forceinline__ double dirichlet(double x, double kn, double sa, double ca, double sb, double cb,
                                            double sk, double ck, double skb, double ckb, double twoNm1)
{
    const double u = x - kn;
    if (u == rint(u)) return twoNm1;
    const double den = sa * ck - ca * sk;           // sin(pi (x - k/n))
    const double num = sb * ckb - cb * skb;         // sin(pi (2N-1) (x - k/n))
    return num / den;
}

#ifndef ICON_KERNELS_TEMPLATES_ONLY
// xy: [M][2] node coordinates, w: [M] weights (group g's at w + g*wstride for
// blockIdx.z = g); K: [G][n0][n1] float.  With perm_r > 0 each row is stored
// in the order k_ytoep4 reads it: frequency k1 of row k0 at
// (k1 mod R) * 32 + k1 / R, R = perm_r = n1 / 32.
__global__ void __launch_bounds__(256) k_toep_kernel(const float *__restrict__ xy, const float *__restrict__ w,
                                                     size_t wstride, int M, int N0, int N1, int n0, int n1,
                                                     int perm_r, float *__restrict__ K)
{
    __shared__ __align__(16) double F0[kToepNodes][kToepTile];   // w_j D_N0(x_j0 - k0/n0)
    __shared__ __align__(16) double F1[kToepNodes][kToepTile];   // D_N1(x_j1 - k1/n1)
    __shared__ double nd[kToepNodes][10];            // per node: sin, cos of pi x0, pi (2N0-1) x0, same for x1; x0, x1
    const int t = threadIdx.x;
    const int k1b = blockIdx.x * kToepTile, k0b = blockIdx.y * kToepTile, grp = blockIdx.z;
    const float *wg = w + (size_t)grp * wstride;
    const double a0 = 2.0 * N0 - 1.0, a1 = 2.0 * N1 - 1.0;
    // This thread's k for the factor tables: column c = t % 64 of both tiles,
    // nodes t / 64 + 4 i.
    const int c = t & (kToepTile - 1), r0 = t >> 6;
    double sk0, ck0, skb0, ckb0, sk1, ck1, skb1, ckb1;
    const double u0 = (double)(k0b + c) / n0, u1 = (double)(k1b + c) / n1;
    {
        sincospi(u0, &sk0, &ck0);
        sincospi(a0 * u0, &skb0, &ckb0);
        sincospi(u1, &sk1, &ck1);
        sincospi(a1 * u1, &skb1, &ckb1);
    }
    const int ty = t >> 4, tx = t & 15;              // outputs k0 = 4 ty + i, k1 = 4 tx + j
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int j0 = 0; j0 < M; j0 += kToepNodes) {
        __syncthreads();                             // the previous chunk's tables are consumed
        if (t < kToepNodes) {
            const int j = j0 + t;
            double x0 = 0.0, x1 = 0.0;
            if (j < M) {
                x0 = (double)xy[2 * (size_t)j];
                x1 = (double)xy[2 * (size_t)j + 1];
            }
            sincospi(x0, &nd[t][0], &nd[t][1]);
            sincospi(a0 * x0, &nd[t][2], &nd[t][3]);
            sincospi(x1, &nd[t][4], &nd[t][5]);
            sincospi(a1 * x1, &nd[t][6], &nd[t][7]);
            nd[t][8] = x0;
            nd[t][9] = x1;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kToepNodes / 4; ++i) {
            const int r = r0 + 4 * i, j = j0 + r;
            const double wj = j < M ? (double)wg[j] : 0.0;
            F0[r][c] = wj * dirichlet(nd[r][8], u0, nd[r][0], nd[r][1], nd[r][2], nd[r][3], sk0, ck0, skb0, ckb0, a0);
            F1[r][c] = dirichlet(nd[r][9], u1, nd[r][4], nd[r][5], nd[r][6], nd[r][7], sk1, ck1, skb1, ckb1, a1);
        }
        __syncthreads();
#pragma unroll 4
        for (int r = 0; r < kToepNodes; ++r) {
            const double2 p0 = *reinterpret_cast<const double2 *>(&F0[r][4 * ty]);
            const double2 p1 = *reinterpret_cast<const double2 *>(&F0[r][4 * ty + 2]);
            const double2 q0 = *reinterpret_cast<const double2 *>(&F1[r][4 * tx]);
            const double2 q1 = *reinterpret_cast<const double2 *>(&F1[r][4 * tx + 2]);
            const double a[4] = {p0.x, p0.y, p1.x, p1.y}, b[4] = {q0.x, q0.y, q1.x, q1.y};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fma(a[i], b[jj], acc[i][jj]);
        }
    }
    const double scale = 1.0 / ((double)n0 * (double)n1);
    float *Kg = K + (size_t)grp * n0 * n1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int k0 = k0b + 4 * ty + i;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int k1 = k1b + 4 * tx + jj;
            const int pos = perm_r > 0 ? (k1 % perm_r) * 32 + k1 / perm_r : k1;
            if (k0 < n0 && k1 < n1) Kg[(size_t)k0 * n1 + pos] = (float)(acc[i][jj] * scale);
        }
    }
}
#endif  // ICON_KERNELS_TEMPLATES_ONLY

// Shared memory of the Toeplitz y-passes: the row buffer [n1][SB], the
// kernel's row [n1] float and the twiddle table (n1 <= 2048).
__host__ __device__ inline size_t ypass_toep_smem(int n1, int B)
{
    size_t sb = (B == 8) ? 8 : (B == 4) ? 6 : B;
    return (size_t)n1 * sb * sizeof(float2) + (size_t)n1 * sizeof(float) + ypass_tw_bytes(n1);
}

// Toeplitz y-pass: per (group, grid row x) the row of the x-transformed
// padded image (the N1 values of G1 row x, placed at y = Y), FFT along y,
// times K[x][.], inverse FFT along y, the N1 values y = Y < N1 written back to
// row x of G1 (in place: a CTA reads its row whole before it writes).  One of
// the two y-passes of A^H W A m; the x-passes are k_xpass_fwd_r2c<FULL> and
// k_xpass_adj with unit deapodisation.
template <int B, int E>
__global__ void FFT_BOUNDS(E) k_ypass_toep(Geo g, float2 *__restrict__ G1)
{
    extern __shared__ float2 s[];
    constexpr int SB = YfStride<B>::v;
    constexpr bool kSwz = (B == 8);
    const int grp = blockIdx.x, x = blockIdx.y, n = g.n1, N1 = g.N1;
    float2 *buf = s;
    float *krow = reinterpret_cast<float *>(s + (size_t)n * SB);
    float2 *tw_s = reinterpret_cast<float2 *>(krow + n);
    const float2 *tws = ypass_tw_shared(n) ? tw_s : g.tw1;
    float2 *row = G1 + ((size_t)grp * g.n0 + x) * N1 * B;
    copy_async(buf, row, (size_t)N1 * B * sizeof(float2));        // [N1][B], contiguous
    copy_async(krow, g.Kt + toep_kernel_index(g, grp) * g.kstride + (size_t)x * n, (size_t)n * sizeof(float));
    if (ypass_tw_shared(n)) copy_async(tw_s, g.tw1, (size_t)n * sizeof(float2));
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const float2 *in = buf;
    auto ld = [=](int y, int b) -> float2 { return y < N1 ? in[y * B + b] : make_float2(0.f, 0.f); };
    auto st2 = [=](int q, int b, float2 v) {
        if (q < N1) row[(size_t)q * B + b] = v;
    };
    auto st = [=](int q, int b, float2 v) {
        const float k = krow[q];
        buf[q * SB + b] = make_float2(v.x * k, v.y * k);
    };
    fft_fused<B, SB, E, false, kSwz, true>(buf, n, g.lg1, tws, -1.f, ld, st);
    __syncthreads();
    auto ld2 = [=](int q, int b) -> float2 { return buf[q * SB + b]; };
    fft_fused<B, SB, E, false, kSwz, true>(buf, n, g.lg1, tws, +1.f, ld2, st2);
}

// The quadratic form of the step length, sum_k K[k] |F(pad r)[k]|^2, for the
// x-transformed r-hat in G1: per (group, row x) the FFT along y of the row
// and the FP64 sum of K[x][k1] |.|^2 per slice into part[G][n0][B] (alpha1,
// NU:1652-1661, in its Toeplitz form).  Nothing else is written.
template <int B, int E>
__global__ void FFT_BOUNDS(E) k_ypass_toep_quad(Geo g, const float2 *__restrict__ G1, double *__restrict__ part)
{
    extern __shared__ float2 s[];
    constexpr int SB = YfStride<B>::v;
    constexpr bool kSwz = (B == 8);
    const int grp = blockIdx.x, x = blockIdx.y, n = g.n1, N1 = g.N1;
    float2 *buf = s;
    float *krow = reinterpret_cast<float *>(s + (size_t)n * SB);
    float2 *tw_s = reinterpret_cast<float2 *>(krow + n);
    const float2 *tws = ypass_tw_shared(n) ? tw_s : g.tw1;
    const float2 *row = G1 + ((size_t)grp * g.n0 + x) * N1 * B;
    copy_async(buf, row, (size_t)N1 * B * sizeof(float2));
    copy_async(krow, g.Kt + toep_kernel_index(g, grp) * g.kstride + (size_t)x * n, (size_t)n * sizeof(float));
    if (ypass_tw_shared(n)) copy_async(tw_s, g.tw1, (size_t)n * sizeof(float2));
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const float2 *in = buf;
    auto ld = [=](int y, int b) -> float2 { return y < N1 ? in[y * B + b] : make_float2(0.f, 0.f); };
    struct Quad {
        const float *krow;
        double acc;
        __device__ __forceinline__ void operator()(int q, int, float2 v)
        {
            acc += (double)krow[q] * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
        }
    } st{krow, 0.0};
    fft_fused<B, SB, E, false, kSwz, true>(buf, n, g.lg1, tws, -1.f, ld, st);
    __syncthreads();
    double *red = reinterpret_cast<double *>(buf);
    const double r = block_sum_per_slice(st.acc, red, B);
    if ((int)threadIdx.x < B) part[((size_t)grp * g.n0 + x) * B + threadIdx.x] = r;
}

// ------------------------------------------- Toeplitz y-passes, 4-step ----
// The y-direction transforms of the Toeplitz passes for a padded length
// n1 = 32 R (R a power of two from 4 to 32, or 3 or 5 times one: 6, 10, 12,
// 20, 24) as a four-step FFT held in registers.  The convolution of the
// thickness-N1 rows with a kernel of support 2 N1 - 1 needs a circular length
// of at least 2 N1 - 1 and nothing more, so the plan takes the smallest such
// 32 R (640 for N1 = 300, where the NUFFT grid's power of two is 1024).  With
// y = 32 a + c (a < R, c < 32) and k = k1 + R k2 (k1 < R, k2 < 32):
//   X[k1 + R k2] = sum_c w32^(c k2) [ wn^(c k1) sum_a x[32 a + c] wR^(a k1) ],
// w_L = exp(-2 pi i / L).  A thread of slice b owns 32 values: first the
// R-point DFTs over a of its columns c = u, u + R, ... (< 32), then, after
// one transpose through shared memory, the 32-point DFT over c of its
// k1 = u.  It then holds X[k1 + R k2] for every k2: a strided set of
// frequencies, which is all that the pointwise product with K and the
// quadratic form need.  The inverse runs the same steps backwards from there
// (32-point inverse DFT, conjugate twiddles, one transpose, R-point inverse
// DFTs), so the forward-multiply-inverse round trip takes two transposes and
// no reordering pass.  The N1 inputs of a row are loaded from global memory
// straight into registers (the B slices of a point are B consecutive float2,
// so a warp reads 256 contiguous bytes) and the N1 outputs stored from
// registers; the zero padding is never loaded.  Shared memory holds only the
// transposed [32][R][B] values, with k1 XOR-swizzled by the low bits of c so
// that the column-wise writes and row-wise reads of a warp spread over the
// banks (for a power-of-two R two wavefronts per 32 x 8 bytes).  Each
// slice's values stay its own, so a slice's result does not depend on its
// group mates.
template <int B, int R>
__device__ __forceinline__ int ytoep4_sidx(int c, int k1, int b)
{
    constexpr int LB = Log2B<B>::v;
    // XOR mask: below 16/B (a quarter warp's columns) and within the largest
    // power of two dividing R, so that k1 ^ mask stays below R.
    constexpr int LOW = R & -R, CAP = 16 / B;
    constexpr int SWM = (LOW < CAP ? LOW : CAP) - 1;
    return ((c * R + (k1 ^ (c & SWM))) << LB) + b;
}

// Lengths R of the first step k_ytoep4 is built for.
__host__ __device__ constexpr bool ytoep4_radix_ok(int R)
{
    return R == 4 || R == 6 || R == 8 || R == 10 || R == 12 || R == 16 || R == 20 || R == 24 || R == 32;
}

// MODE 0: row x of G1 <- crop F^-1(K[x][.] . F(pad row)), in place (the
// Toeplitz y-pass of A^H W A m).  MODE 1: part[G][n0][B] <- per slice
// sum_k K[x][k] |F(pad row)[k]|^2 in FP64 (the step length's denominator).
// g.n1 = 32 R and g.tw1 its twiddles (the Toeplitz view of the plan).
// Launch bounds: blocks of R B threads, at least 512 threads per SM; the
// 640-point transform of 8-slice groups (the 1024x300 workload) asks for four
// blocks per SM (96 registers, a few spilled bytes), which measured 8% faster
// for MODE 1 and the same for MODE 0 than three blocks at 128 registers.
template <int B, int R, int MODE>
__global__ void __launch_bounds__(R * B, (R == 20 && B == 8) ? 4 : (512 / (R * B) < 32 ? 512 / (R * B) : 32))
    k_ytoep4(Geo g, float2 *__restrict__ G1, double *__restrict__ part)
{
    constexpr int LB = Log2B<B>::v;
    constexpr int NI = (32 + R - 1) / R;     // columns per thread in the first step (the last may be short)
    extern __shared__ float2 s[];
    const int grp = blockIdx.x, x = blockIdx.y, N1 = g.N1;
    const int t = threadIdx.x, b = t & (B - 1), u = t >> LB;
    float2 *row = G1 + ((size_t)grp * g.n0 + x) * N1 * B;
    const float *krow = g.Kt + toep_kernel_index(g, grp) * g.kstride + (size_t)x * (32 * R);
    // The twiddle table wn^q, q < 32 R, copied behind the transposed values;
    // every twiddle of the two steps is read from it.
    float2 *tws = s + 32 * R * B;
    for (int q = t; q < 32 * R / 2; q += R * B) cp_async<16>(tws + 2 * q, g.tw1 + 2 * q);
    cp_async_commit();

    // Step 1: R-point DFTs over a, twiddles wn^(c k1), transpose.
    {
        float2 v[NI][R];
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int c = u + R * i;
            if (c >= 32) break;
            const float2 *rb = row + (c * B + b);   // point y = 32 a + c at rb[32 B a]
            const int na = (N1 - c + 31) >> 5;      // points y < N1
#pragma unroll
            for (int a = 0; a < R; ++a) v[i][a] = a < na ? rb[32 * B * a] : make_float2(0.f, 0.f);
        }
        cp_async_wait<0>();
        __syncthreads();   // the twiddle table is in shared memory
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int c = u + R * i;
            if (c >= 32) break;
            dft_nat<R>(v[i], -1.f);
#pragma unroll
            for (int k1 = 1; k1 < R; ++k1) v[i][k1] = cmul(v[i][k1], tws[c * k1]);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) s[ytoep4_sidx<B, R>(c, k1, b)] = v[i][k1];
        }
    }
    __syncthreads();
    // Step 2: 32-point DFT over c for k1 = u: w[k2] = X[u + R k2].
    float2 w[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) w[brev5(c)] = s[ytoep4_sidx<B, R>(c, u, b)];
    dft_inplace<32>(w, -1.f);
    // K[x][u + R k2] for k2 = 0..31: 32 consecutive floats of the permuted row.
    const float4 *kq = reinterpret_cast<const float4 *>(krow + 32 * u);
    if constexpr (MODE == 1) {
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 k4 = __ldg(&kq[q]);
            const float kv[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 a = w[4 * q + j];
                acc += (double)kv[j] * ((double)a.x * (double)a.x + (double)a.y * (double)a.y);
            }
        }
        __syncthreads();   // every read of s is done before the reduction reuses it
        const double r = block_sum_per_slice(acc, reinterpret_cast<double *>(s), B);
        if (t < B) part[((size_t)grp * g.n0 + x) * B + t] = r;
    } else {
        // Pointwise product with K, 32-point inverse DFT over k2, twiddles
        // conj(wn^(c k1)), transpose back.
        // In place: w[k2] *= K, then the DIF inverse leaves Z[c] at w[brev5(c)].
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 k4 = __ldg(&kq[q]);
            const float kv[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) w[4 * q + j] = make_float2(w[4 * q + j].x * kv[j], w[4 * q + j].y * kv[j]);
        }
        dft_dif_inplace<32>(w, +1.f);
#pragma unroll
        for (int c = 1; c < 32; ++c) {   // conj(wn^(c u)) from the table
            float2 tw = tws[c * u];
            tw.y = -tw.y;
            w[brev5(c)] = cmul(w[brev5(c)], tw);
        }
        __syncthreads();   // every read of s is done before it is overwritten
#pragma unroll
        for (int c = 0; c < 32; ++c) s[ytoep4_sidx<B, R>(c, u, b)] = w[brev5(c)];
        __syncthreads();
        // R-point inverse DFTs over k1 for columns c = u + R i; rows y < N1 out.
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int c = u + R * i;
            if (c >= 32) break;
            float2 v[R];
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = s[ytoep4_sidx<B, R>(c, k1, b)];
            dft_nat<R>(v, +1.f);
            float2 *rb = row + (c * B + b);
            const int na = (N1 - c + 31) >> 5;
#pragma unroll
            for (int a = 0; a < R; ++a)
                if (a < na) rb[32 * B * a] = v[a];
        }
    }
}

__host__ __device__ inline size_t ytoep4_smem(int n1, int B) { return (size_t)n1 * (B + 1) * sizeof(float2); }
// n1 sizes k_ytoep4 takes (n1 = 32 R, R in ytoep4_radix_ok).
__host__ __device__ inline bool ytoep4_fits(int n1) { return n1 % 32 == 0 && ytoep4_radix_ok(n1 / 32); }

}  // namespace icon

namespace icon {

// ------------------------------------------- Toeplitz x-passes, 3-step ----
// The x-direction transforms of the Toeplitz iteration, n0 = 32 NA NB
// (NA = 2^LA, NB = 2^LNB), as a register-resident three-step FFT over the
// BH slices (of a B-slice group) that one CTA takes.  With
// x = 32 NB a + 32 b + c (a < NA, b < NB, c < 32) and
// k = ka + NA kb + NA NB kc:
//   X[k] = sum_c w32^(c kc) wn^(NA c kb) sum_b wNB^(b kb) wn^((32 b + c) ka)
//          sum_a wNA^(a ka) x[32 NB a + 32 b + c].
// Thread u (of U = NA NB per slice) does the NA-point DFTs over a of the
// columns tau = 32 b + c = u + U i (i < 32 / NA), then, after a transpose,
// the NB-point DFTs over b of (ka, c) = (tau >> 5, tau & 31) for
// tau = u + U i (i < 32 / NB), then, after a second transpose, the 32-point
// DFT over c of (ka, kb) = (u mod NA, u / NA): it ends holding frequencies
// u + U kc, which go straight to rows u + U kc of G1.  The inverse reads those
// rows into the same registers and runs the steps backwards, ending with the
// values of x = 32 NB a + tau for its columns tau: the columns its forward
// step 1 starts from.  So the adjoint x-pass (crop, r-hat = . - Ahwb, |r-hat|^2)
// and the forward x-pass of r-hat fuse into one kernel whose r-hat never
// leaves registers between the two transforms, and the update
// m <- m - alpha Re r-hat (with the clamp) fuses into the forward x-pass of m.
// Inputs and outputs are read and written straight from and to global memory
// (a warp covers consecutive x, i.e. 32/BH points of BH x 8 bytes); the two
// transposes go through one shared buffer, [ka][tau][BH] after step 1 and
// [ka][kb][c][BH] after step 2, with the innermost index XOR-swizzled by the
// low bits of ka where a warp's lanes differ in ka, so that every access
// takes the minimum two wavefronts.  Each slice stays its own transform.
struct XtArgs {
    int N0, N1, n0;
    const float2 *tw0;       // [n0] exp(-2 pi i q / n0)
    float2 *G1;              // [G][n0][N1][B]
    float *m;                // [G][N1][N0][B] real image (forward input; updated in place when upd)
    const float *rre_in;     // update: Re r-hat of the iteration being finished, [G][N1][N0][B]
    const double *alpha;     // update: [G*B] step lengths
    int upd, clamp, data_type;
    float thr;
    float2 *rhat;            // adjoint: the adjoint (or r-hat) out, [G][N1][N0][B]
    float *rre;              // mid: Re r-hat out, [G][N1][N0][B] (the update needs only the real part)
    const float2 *Ahwb;      // mid / adjoint with resid: [G][N1][N0][B]
    double *part_rtr;        // mid / adjoint with resid: [G][N1][B] partial |r-hat|^2 per column
    const float *rcx, *rcy;  // adjoint: deapodisation reciprocals 1/cx [N0], 1/cy [N1]
    int resid;               // adjoint: subtract Ahwb and sum |.|^2 (else the plain adjoint)
    // TMA staging of the columns (use_tma; BH >= 2): the plan's G1 as 2-D
    // [Gcap n0 rows][N1 B 2 floats], its Ahwb and r-hat as 3-D
    // [Gcap N1][N0][B 2 floats], and (tma_m; BH >= 4) its m and Re r-hat
    // as [Gcap N1][N0][B floats]; boxes of BH slices by box_g1 / box_img rows.
    // Every wait on the loads is bounded and reports through err.
    CUtensorMap tm_g1, tm_ahwb, tm_rre, tm_m;
    int use_tma, tma_m, box_g1, box_img;
    int *err;
};

// Bounded wait of all threads of a CTA on a TMA barrier; false (the same in
// every thread) when any thread's wait ran out, after recording the error
// and giving the loads a second bounded wait to land.
__device__ __forceinline__ bool xt_tma_wait(uint64_t *bar, int *err)
{
    bool ok = ws::mbar_wait(bar, 0, err, ws::kErrLoadWait);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) ws::mbar_wait(bar, 0, err, ws::kErrLoadWait);
    return ok;
}

template <int BH, int LA, int LNB>
struct XtShape {
    static constexpr int NA = 1 << LA, NB = 1 << LNB, U = NA * NB, T = U * BH;
    static constexpr int N = 32 * U;
    static constexpr int NI1 = 32 / NA, NI2 = 32 / NB;
    static constexpr int SW = 16 / BH - 1;
    // unit (float2) index of (ka, tau, s) after step 1 and of (ka, kb, c, s)
    // after step 2
    __device__ static __forceinline__ int e1(int ka, int tau, int s)
    {
        const int t = (NB == 1) ? (tau ^ (ka & SW)) : tau;
        return (ka * 32 * NB + t) * BH + s;
    }
    __device__ static __forceinline__ int e2(int ka, int kb, int c, int s)
    {
        return ((ka * NB + kb) * 32 + (c ^ (ka & SW))) * BH + s;
    }
};

// x^(e) times wn^(base*j) for j = 1..R-1 in place, the twiddles formed from
// the table at multiples of 8 and by products in between; CONJ: conjugates.
template <int R, bool CONJ>
__device__ __forceinline__ void xt_twiddle(float2 (&v)[R], const float2 *__restrict__ tw, int base)
{
    float2 w1 = __ldg(&tw[base]);
    if (CONJ) w1.y = -w1.y;
    float2 t = w1;
#pragma unroll
    for (int j = 1; j < R; ++j) {
        if ((j & 7) == 0) {
            t = __ldg(&tw[base * j]);
            if (CONJ) t.y = -t.y;
        } else if (j > 1) {
            t = cmul(t, w1);
        }
        v[j] = cmul(v[j], t);
    }
}

// Forward transform from the step-1 registers v[i][a] (input at
// x = 32 NB a + u + U i) to G1 rows u + U kc of column `col` (pointer to
// row 0 of the column for this thread's slice; rows N1*B float2 apart).
template <int BH, int LA, int LNB>
__device__ __forceinline__ void xt_forward(float2 (&v)[32 >> LA][1 << LA], float2 *s, int u, int sl,
                                           const float2 *__restrict__ tw, float2 *col, size_t rstride)
{
    using S = XtShape<BH, LA, LNB>;
    constexpr int NA = S::NA, NB = S::NB, U = S::U;
#pragma unroll
    for (int i = 0; i < S::NI1; ++i) {
        const int tau = u + U * i;
        float2 a[NA];
#pragma unroll
        for (int j = 0; j < NA; ++j) a[brev5(j) >> (5 - LA)] = v[i][j];
        dft_inplace<NA>(a, -1.f);
        if (tau) xt_twiddle<NA, false>(a, tw, tau);
#pragma unroll
        for (int ka = 0; ka < NA; ++ka) s[S::e1(ka, tau, sl)] = a[ka];
    }
    __syncthreads();
    if constexpr (NB > 1) {
        float2 v2[S::NI2][NB];
#pragma unroll
        for (int i = 0; i < S::NI2; ++i) {
            const int t2 = u + U * i, c = t2 & 31, ka = t2 >> 5;
#pragma unroll
            for (int b = 0; b < NB; ++b) v2[i][brev5(b) >> (5 - LNB)] = s[S::e1(ka, 32 * b + c, sl)];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < S::NI2; ++i) {
            const int t2 = u + U * i, c = t2 & 31, ka = t2 >> 5;
            dft_inplace<NB>(v2[i], -1.f);
            if (c) xt_twiddle<NB, false>(v2[i], tw, NA * c);
#pragma unroll
            for (int kb = 0; kb < NB; ++kb) s[S::e2(ka, kb, c, sl)] = v2[i][kb];
        }
        __syncthreads();
    }
    float2 w[32];
    {
        const int ka = u % NA, kb = u / NA;
#pragma unroll
        for (int c = 0; c < 32; ++c) w[brev5(c)] = (NB > 1) ? s[S::e2(ka, kb, c, sl)] : s[S::e1(ka, c, sl)];
    }
    dft_inplace<32>(w, -1.f);
    float2 *p = col + (size_t)u * rstride;
    const size_t step = (size_t)U * rstride;
#pragma unroll
    for (int kc = 0; kc < 32; ++kc, p += step) *p = w[kc];
}

// Inverse transform from the column staged in s ([x][BH], rows u + U kc
// of this thread's slice) to the step-1 registers v[i][a] (value at
// x = 32 NB a + u + U i).  Ends after a barrier-free last step: the caller
// syncs before writing s again.
template <int BH, int LA, int LNB>
__device__ __forceinline__ void xt_inverse(float2 (&v)[32 >> LA][1 << LA], float2 *s, int u, int sl,
                                           const float2 *__restrict__ tw)
{
    using S = XtShape<BH, LA, LNB>;
    constexpr int NA = S::NA, NB = S::NB, U = S::U;
    {
        // The column, staged in s as [x][BH]: rows u + U kc of this slice.
        float2 w[32];
#pragma unroll
        for (int kc = 0; kc < 32; ++kc) w[kc] = s[(u + U * kc) * BH + sl];
        __syncthreads();                              // the staged column is consumed before s is rewritten
        dft_dif_inplace<32>(w, +1.f);                 // Z[c] at w[brev5(c)]
        const int ka = u % NA, kb = u / NA;
        if constexpr (NB > 1) {
            if (kb) {
                float2 z[32];
#pragma unroll
                for (int c = 0; c < 32; ++c) z[c] = w[brev5(c)];
                xt_twiddle<32, true>(z, tw, NA * kb);
#pragma unroll
                for (int c = 0; c < 32; ++c) w[brev5(c)] = z[c];
            }
#pragma unroll
            for (int c = 0; c < 32; ++c) s[S::e2(ka, kb, c, sl)] = w[brev5(c)];
        } else {
#pragma unroll
            for (int c = 0; c < 32; ++c) s[S::e1(ka, c, sl)] = w[brev5(c)];
        }
    }
    __syncthreads();
    if constexpr (NB > 1) {
        float2 v2[S::NI2][NB];
#pragma unroll
        for (int i = 0; i < S::NI2; ++i) {
            const int t2 = u + U * i, c = t2 & 31, ka = t2 >> 5;
#pragma unroll
            for (int kb = 0; kb < NB; ++kb) v2[i][kb] = s[S::e2(ka, kb, c, sl)];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < S::NI2; ++i) {
            const int t2 = u + U * i, c = t2 & 31, ka = t2 >> 5;
            dft_dif_inplace<NB>(v2[i], +1.f);          // Z[b] at v2[brev(b)]
#pragma unroll
            for (int b = 0; b < NB; ++b) s[S::e1(ka, 32 * b + c, sl)] = v2[i][brev5(b) >> (5 - LNB)];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < S::NI1; ++i) {
        const int tau = u + U * i;
        float2 a[NA];
#pragma unroll
        for (int ka = 0; ka < NA; ++ka) a[ka] = s[S::e1(ka, tau, sl)];
        if (tau) xt_twiddle<NA, true>(a, tw, tau);
        dft_dif_inplace<NA>(a, +1.f);                  // x at a[brev(a)]
#pragma unroll
        for (int j = 0; j < NA; ++j) v[i][j] = a[brev5(j) >> (5 - LA)];
    }
}

// MODE 0: G1 <- F_x(pad m) for every row, m first updated (upd: m <- m -
// alpha Re r-hat_in, clamped on ICON steps, as k_update).  MODE 1: r-hat =
// crop F_x^-1(G1) - Ahwb (stored, |r-hat|^2 partial sums per column), then
// G1 <- F_x(pad r-hat) in place.  MODE 2: the last x-pass of the NUFFT
// adjoint (k_xpass_adj's work): out = crop F_x^-1(G1) / (cx cy), with resid
// minus Ahwb and the |.|^2 partial sums.  Grid: (N1 * B/BH, G), half-group
// fastest.
template <int B, int BH, int LA, int LNB, int MODE>
__global__ void __launch_bounds__(XtShape<BH, LA, LNB>::T, (XtShape<BH, LA, LNB>::T >= 256) ? 2 : 4)
    k_xtoep(const __grid_constant__ XtArgs g)
{
    using S = XtShape<BH, LA, LNB>;
    constexpr int NA = S::NA, NB = S::NB, U = S::U, H = B / BH;
    extern __shared__ __align__(128) float2 s[];
    __shared__ __align__(8) uint64_t bar[2];   // TMA: [0] the G1 or m column, [1] the Ahwb or r-hat column
    constexpr bool kTma = BH >= 2;
    const bool tma = kTma && g.use_tma;
    double *red = reinterpret_cast<double *>(s + S::N * BH);
    const int Y = blockIdx.x / H, h = blockIdx.x % H, grp = blockIdx.y;
    const int t = threadIdx.x, sl = t % BH, u = t / BH, bsl = h * BH + sl;   // bsl: slice within the group
    const int N0 = g.N0, N1 = g.N1, n = S::N, half = N0 / 2;
    const size_t rstride = (size_t)N1 * B;
    float2 *col = g.G1 + ((size_t)grp * n * N1 + Y) * B + bsl;       // row x at col[x * rstride]
    const size_t ibase = ((size_t)grp * N1 + Y) * N0 * B + bsl;        // image point X at ibase + X*B
    float2 v[S::NI1][NA];
    // mid: this CTA's Ahwb column, [N0][BH], at a 128-byte boundary (a TMA destination)
    float2 *As = s + ((S::N * BH + S::T + 15) & ~15);
    if (tma) {
        if (t == 0) {
            ws::mbar_init(&bar[0], 1);
            ws::mbar_init(&bar[1], 1);
            ws::mbar_fence_init();
        }
        __syncthreads();
    }
    if (MODE >= 1 && tma) {
        // One thread issues the column's loads: the G1 column in boxes of
        // box_g1 rows x BH values into s as [x][BH], then the Ahwb column in
        // boxes of box_img points into As (rows past N0 read as zeros and
        // land inside As, whose n0/2 rows are a multiple of the box).
        if (t == 0) {
            ws::mbar_expect_tx(&bar[0], (uint32_t)(n * BH * sizeof(float2)));
            for (int x0 = 0; x0 < n; x0 += g.box_g1)
                ws::tma_load_2d(s + x0 * BH, &g.tm_g1, (Y * B + h * BH) * 2, grp * n + x0, &bar[0]);
            if (MODE == 1 || g.resid) {
                const int nbox = (N0 + g.box_img - 1) / g.box_img;
                ws::mbar_expect_tx(&bar[1], (uint32_t)(nbox * g.box_img * BH * sizeof(float2)));
                for (int k = 0; k < nbox; ++k)
                    ws::tma_load_3d(As + k * g.box_img * BH, &g.tm_ahwb, h * BH * 2, k * g.box_img, grp * N1 + Y,
                                    &bar[1]);
            }
        }
    } else if constexpr (MODE >= 1) {
        // The G1 column (n0 rows of BH values, rows N1*B float2 apart) into s
        // as [x][BH], then the Ahwb column, staged while the inverse runs.
        const float2 *gsrc = g.G1 + ((size_t)grp * n * N1 + Y) * B + h * BH;
        if constexpr (BH >= 2) {
            constexpr int P = BH / 2;
            for (int idx = t; idx < n * P; idx += S::T) {
                const int x = idx / P, c = idx - x * P;
                cp_async<16>(s + x * BH + 2 * c, gsrc + (size_t)x * rstride + 2 * c);
            }
        } else {
            for (int x = t; x < n; x += S::T) cp_async<8>(s + x, gsrc + (size_t)x * rstride);
        }
        cp_async_commit();
        if (MODE == 1 || g.resid) {
            const float2 *src = g.Ahwb + ((size_t)grp * N1 + Y) * N0 * B + h * BH;
            if constexpr (BH >= 2) {
                constexpr int P = BH / 2;                     // 16-byte pieces per point
                for (int idx = t; idx < N0 * P; idx += S::T) {
                    const int X = idx / P, c = idx - X * P;
                    cp_async<16>(As + X * BH + 2 * c, src + (size_t)X * B + 2 * c);
                }
            } else {
                for (int X = t; X < N0; X += S::T) cp_async<8>(As + X, src + (size_t)X * B);
            }
        }
        cp_async_commit();
    }
    if constexpr (MODE == 0) {
        // The m column (N0 x BH floats) into s and, for the update, the r-hat
        // column into As, by cp.async; then into registers.
        float *Ms = reinterpret_cast<float *>(s);
        float *Rs = reinterpret_cast<float *>(As);   // Re r-hat column, [N0][BH] floats
        if (tma && g.tma_m) {
            // m and (for the update) the Re r-hat column by TMA, boxes of
            // box_img points: m as [X][BH] floats into s, Re r-hat into Rs.
            const int nbox = (N0 + g.box_img - 1) / g.box_img;
            if (t == 0) {
                ws::mbar_expect_tx(&bar[0], (uint32_t)(nbox * g.box_img * BH * sizeof(float)));
                for (int k = 0; k < nbox; ++k)
                    ws::tma_load_3d(Ms + k * g.box_img * BH, &g.tm_m, h * BH, k * g.box_img, grp * N1 + Y, &bar[0]);
                if (g.upd) {
                    ws::mbar_expect_tx(&bar[1], (uint32_t)(nbox * g.box_img * BH * sizeof(float)));
                    for (int k = 0; k < nbox; ++k)
                        ws::tma_load_3d(Rs + k * g.box_img * BH, &g.tm_rre, h * BH, k * g.box_img, grp * N1 + Y,
                                        &bar[1]);
                }
            }
            if (!xt_tma_wait(&bar[0], g.err)) return;
            if (g.upd && !xt_tma_wait(&bar[1], g.err)) return;
        } else {
            const float *msrc = g.m + ibase - sl;           // point X of this CTA's slices at msrc + X*B
            const float *rsrc = g.rre_in + ibase - sl;
            for (int X = t; X < N0; X += S::T) {
                if constexpr (BH == 4) cp_async<16>(Ms + X * 4, msrc + (size_t)X * B);
                else if constexpr (BH == 2) cp_async<8>(Ms + X * 2, msrc + (size_t)X * B);
                else if constexpr (BH == 1) cp_async<4>(Ms + X, msrc + (size_t)X * B);
                else {
                    cp_async<16>(Ms + X * BH, msrc + (size_t)X * B);
                    cp_async<16>(Ms + X * BH + 4, msrc + (size_t)X * B + 4);
                }
            }
            if (g.upd) {
                for (int X = t; X < N0; X += S::T) {
                    if constexpr (BH == 4) cp_async<16>(Rs + X * 4, rsrc + (size_t)X * B);
                    else if constexpr (BH == 2) cp_async<8>(Rs + X * 2, rsrc + (size_t)X * B);
                    else if constexpr (BH == 1) cp_async<4>(Rs + X, rsrc + (size_t)X * B);
                    else {
                        cp_async<16>(Rs + X * BH, rsrc + (size_t)X * B);
                        cp_async<16>(Rs + X * BH + 4, rsrc + (size_t)X * B + 4);
                    }
                }
            }
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
        }
        if (g.upd) {
            // m <- m - alpha Re r-hat (k_update's arithmetic), clamped on ICON
            // steps, over the staged column by all threads (coalesced stores).
            float *mdst = g.m + ibase - sl;
            for (int idx = t; idx < N0 * BH; idx += S::T) {
                const int X = idx / BH, q = idx - X * BH;
                const double al = g.alpha[grp * B + h * BH + q];
                float nv = (float)((double)Ms[idx] - al * (double)Rs[idx]);
                if (g.clamp) {
                    if (g.data_type == 1) {
                        if (nv > g.thr) nv = g.thr;
                    } else {
                        if (nv < g.thr) nv = g.thr;
                    }
                }
                Ms[idx] = nv;
                mdst[(size_t)X * B + q] = nv;
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < S::NI1; ++i) {
            const int tau = u + U * i;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int X = (32 * NB * a + tau + half) & (n - 1);
                v[i][a] = make_float2(X < N0 ? Ms[X * BH + sl] : 0.f, 0.f);
            }
        }
        __syncthreads();   // the staged m is read before step 1 rewrites s
        xt_forward<BH, LA, LNB>(v, s, u, sl, g.tw0, col, rstride);
    } else if constexpr (MODE == 2) {
        if (tma) {
            if (!xt_tma_wait(&bar[0], g.err)) return;
        } else {
            cp_async_wait<1>();
            __syncthreads();
        }
        xt_inverse<BH, LA, LNB>(v, s, u, sl, g.tw0);
        if (tma) {
            if (g.resid && !xt_tma_wait(&bar[1], g.err)) return;
            __syncthreads();
        } else {
            cp_async_wait<0>();
            __syncthreads();
        }
        const float rcyY = g.rcy[Y];
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < S::NI1; ++i) {
            const int tau = u + U * i;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int X = (32 * NB * a + tau + half) & (n - 1);
                if (X < N0) {
                    const float r = g.rcx[X] * rcyY;         // as k_xpass_adj
                    float2 o = make_float2(v[i][a].x * r, v[i][a].y * r);
                    if (g.resid) {
                        const float2 av = As[X * BH + sl];
                        o.x = o.x - av.x;
                        o.y = o.y - av.y;
                        acc += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
                    }
                    g.rhat[ibase + (size_t)X * B] = o;
                }
            }
        }
        if (g.resid) {
            red[t] = acc;
            __syncthreads();
            for (int stride = S::T >> 1; stride >= BH; stride >>= 1) {
                if (t < stride) red[t] += red[t + stride];
                __syncthreads();
            }
            if (t < BH) g.part_rtr[((size_t)grp * N1 + Y) * B + h * BH + t] = red[t];
        }
    } else {
        if (tma) {
            if (!xt_tma_wait(&bar[0], g.err)) return;
        } else {
            cp_async_wait<1>();    // the column group (Ahwb may still be landing)
            __syncthreads();
        }
        xt_inverse<BH, LA, LNB>(v, s, u, sl, g.tw0);
        if (tma) {
            if (!xt_tma_wait(&bar[1], g.err)) return;
            __syncthreads();   // every read of s by the inverse is done
        } else {
            cp_async_wait<0>();
            __syncthreads();   // Ahwb staged; every read of s by the inverse is done
        }
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < S::NI1; ++i) {
            const int tau = u + U * i;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int x = 32 * NB * a + tau;
                const int X = (x + half) & (n - 1);
                float2 r = make_float2(0.f, 0.f);
                if (X < N0) {
                    const float2 av = As[X * BH + sl];
                    r = make_float2(v[i][a].x - av.x, v[i][a].y - av.y);
                    acc += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
                    g.rre[ibase + (size_t)X * B] = r.x;
                }
                v[i][a] = r;
            }
        }
        xt_forward<BH, LA, LNB>(v, s, u, sl, g.tw0, col, rstride);
        // per-slice FP64 sum in a fixed order (thread t holds slice t % BH)
        red[t] = acc;
        __syncthreads();
        for (int stride = S::T >> 1; stride >= BH; stride >>= 1) {
            if (t < stride) red[t] += red[t + stride];
            __syncthreads();
        }
        if (t < BH) g.part_rtr[((size_t)grp * N1 + Y) * B + h * BH + t] = red[t];
    }
}

// Shared memory of k_xtoep: the transposed values, the reduction scratch
// and (mid) the staged Ahwb column of N0 <= n0 / 2 points.
__host__ __device__ inline size_t xtoep_smem(int n0, int BH)
{
    return (size_t)n0 * BH * sizeof(float2) + (size_t)(n0 * BH / 32) * sizeof(double) + 128 +
           (size_t)(n0 / 2) * BH * sizeof(float2);
}

}  // namespace icon
