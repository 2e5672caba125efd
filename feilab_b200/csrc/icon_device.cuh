// icon_device.cuh -- device helpers shared by the ICON kernels: complex
// arithmetic, the in-register DFTs and the shared-memory Stockham FFT used by
// every x- and y-pass.
//
// Batched layout convention: a "group" holds B slices that share a tilt
// geometry; the slice index b is the fastest-varying index of every batched
// array, so a group's values for one grid point / node / pixel are B
// consecutive float2 (64 bytes for B = 8).  Shared-memory FFT buffers are
// [n][B] float2 with the same convention.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace icon {

constexpr int kTaps = 14;   // 2m+2 taps per dimension, m = 6 (nufft_gpu_v8.cuh:5, NU:226)
constexpr int kHalf = 6;    // window half-width m
constexpr int kKbHalf = 4;  // half-width K of the Kaiser-Bessel window (taps 3..10 of the 14)
constexpr int kKbTlo = kHalf - kKbHalf + 1, kKbThi = kHalf + kKbHalf;

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// a + b and a - b on both components with one packed Blackwell instruction
// (add/sub.rn.f32x2): the same rounding as two scalar adds.
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// a * b + c on both components with one packed Blackwell instruction
// (fma.rn.f32x2); each component is rounded exactly as fmaf rounds it.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// exp(dir * 2*pi*i * k / 16), k in [0, 16), dir = -1 (forward) or +1 (inverse).
// Called with compile-time k only, so the table folds into immediates.
__device__ __forceinline__ float2 w16(int k, float dir)
{
    constexpr float C[16] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                             0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f,
                             -1.0f, -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f,
                             0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f};
    constexpr float S[16] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
                             1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                             0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f,
                             -1.0f, -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f};
    return make_float2(C[k], dir * S[k]);
}

// out[q] = sum_r in[r*IS] * exp(dir*2*pi*i*r*q/R): radix-2 decimation in time,
// fully unrolled into registers (R <= 16).
template <int R, int IS>
__device__ __forceinline__ void dft(const float2 *in, float2 *out, float dir)
{
    if constexpr (R == 1) {
        out[0] = in[0];
    } else {
        float2 e[R / 2], o[R / 2];
        dft<R / 2, 2 * IS>(in, e, dir);
        dft<R / 2, 2 * IS>(in + IS, o, dir);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            float2 t = (k == 0) ? o[k] : cmul(w16((k * (16 / R)) & 15, dir), o[k]);
            out[k] = cadd(e[k], t);
            out[k + R / 2] = csub(e[k], t);
        }
    }
}

// One self-sorting (Stockham) radix-R pass over a shared-memory batch
// s[n][B].  blockDim.x * 16 == n * B: each thread owns 16 values, i.e.
// 16/R butterflies.  tw[q] = exp(-2*pi*i*q/n) for q in [0, n).
template <int R>
__device__ __forceinline__ void fft_pass(float2 *s, int n, int B, int Ns, const float2 *__restrict__ tw, float dir)
{
    constexpr int Q = 16 / R;
    const int nb = n / R;
    const int T = blockDim.x;
    const int step = n / (Ns * R);
    float2 v[Q][R];
    int jq[Q], bq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int item = threadIdx.x + q * T;
        int b = item % B, j = item / B;
        jq[q] = j;
        bq[q] = b;
        int k = j & (Ns - 1);
        float2 in[R];
#pragma unroll
        for (int r = 0; r < R; ++r) in[r] = s[(j + r * nb) * B + b];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(&tw[(r * k * step) & (n - 1)]);
                w.y = -dir * w.y;
                in[r] = cmul(in[r], w);
            }
        }
        dft<R, 1>(in, v[q], dir);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int j = jq[q], b = bq[q];
        int k = j & (Ns - 1);
        int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) s[(base + r * Ns) * B + b] = v[q][r];
    }
    __syncthreads();
}

// Unnormalised FFT of length n = 2^lg (16 <= n) for each of the B columns of
// s[n][B]; dir = -1 is cuFFT's CUFFT_FORWARD, +1 its CUFFT_INVERSE.
// Requires blockDim.x == n*B/16 and a __syncthreads() before the call.
__device__ __forceinline__ void fft_smem(float2 *s, int n, int lg, int B, const float2 *__restrict__ tw, float dir)
{
    int Ns = 1;
    switch (lg & 3) {
    case 1: fft_pass<2>(s, n, B, Ns, tw, dir); Ns = 2; break;
    case 2: fft_pass<4>(s, n, B, Ns, tw, dir); Ns = 4; break;
    case 3: fft_pass<8>(s, n, B, Ns, tw, dir); Ns = 8; break;
    default: break;
    }
    while (Ns < n) {
        fft_pass<16>(s, n, B, Ns, tw, dir);
        Ns *= 16;
    }
}

// ---- batched FFT with compile-time batch B and row stride SB (>= B) ----
// Same Stockham passes as fft_pass/fft_smem over s[n][SB] (values of slice b
// at s[pos*SB + b]); B and SB are powers of two or padded strides known at
// compile time, so all index arithmetic is shifts and masks.
template <int B>
struct Log2B {
    static constexpr int v = (B >= 8) ? 3 : (B >= 4) ? 2 : (B >= 2) ? 1 : 0;
};

template <int R, int B, int SB>
__device__ __forceinline__ void fft_pass_b(float2 *s, int n, int Ns, const float2 *__restrict__ tw, float dir)
{
    constexpr int Q = 16 / R;
    constexpr int LB = Log2B<B>::v;
    const int nb = n / R;
    const int T = blockDim.x;
    const int step = n / (Ns * R);
    float2 v[Q][R];
    int jq[Q], bq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int item = threadIdx.x + q * T;
        int b = item & (B - 1), j = item >> LB;
        jq[q] = j;
        bq[q] = b;
        int k = j & (Ns - 1);
        float2 in[R];
#pragma unroll
        for (int r = 0; r < R; ++r) in[r] = s[(j + r * nb) * SB + b];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(&tw[r * k * step]);
                w.y = -dir * w.y;
                in[r] = cmul(in[r], w);
            }
        }
        dft<R, 1>(in, v[q], dir);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int j = jq[q], b = bq[q];
        int k = j & (Ns - 1);
        int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) s[(base + r * Ns) * SB + b] = v[q][r];
    }
    __syncthreads();
}

// blockDim.x == n*B/16; call after a __syncthreads().
template <int B, int SB>
__device__ __forceinline__ void fft_batched(float2 *s, int n, int lg, const float2 *__restrict__ tw, float dir)
{
    int Ns = 1;
    switch (lg & 3) {
    case 1: fft_pass_b<2, B, SB>(s, n, Ns, tw, dir); Ns = 2; break;
    case 2: fft_pass_b<4, B, SB>(s, n, Ns, tw, dir); Ns = 4; break;
    case 3: fft_pass_b<8, B, SB>(s, n, Ns, tw, dir); Ns = 8; break;
    default: break;
    }
    while (Ns < n) {
        fft_pass_b<16, B, SB>(s, n, Ns, tw, dir);
        Ns *= 16;
    }
}

// ---- fused FFT: E values per thread, I/O through functors ---------------
// exp(dir * 2*pi*i * k / 32) for compile-time k.
__device__ __forceinline__ float2 w32(int k, float dir)
{
    constexpr float C[32] = {
        1.0f, 0.98078528040323043f, 0.92387953251128674f, 0.83146961230254524f, 0.70710678118654752f,
        0.55557023301960218f, 0.38268343236508977f, 0.19509032201612826f, 0.0f, -0.19509032201612826f,
        -0.38268343236508977f, -0.55557023301960218f, -0.70710678118654752f, -0.83146961230254524f,
        -0.92387953251128674f, -0.98078528040323043f, -1.0f, -0.98078528040323043f, -0.92387953251128674f,
        -0.83146961230254524f, -0.70710678118654752f, -0.55557023301960218f, -0.38268343236508977f,
        -0.19509032201612826f, 0.0f, 0.19509032201612826f, 0.38268343236508977f, 0.55557023301960218f,
        0.70710678118654752f, 0.83146961230254524f, 0.92387953251128674f, 0.98078528040323043f};
    return make_float2(C[k & 31], dir * C[(k + 24) & 31]);
}

// out[q] = sum_r in[r*IS] exp(dir*2*pi*i*r*q/R), R <= 32, unrolled.
template <int R, int IS>
__device__ __forceinline__ void dft32(const float2 *in, float2 *out, float dir)
{
    if constexpr (R == 1) {
        out[0] = in[0];
    } else {
        float2 e[R / 2], o[R / 2];
        dft32<R / 2, 2 * IS>(in, e, dir);
        dft32<R / 2, 2 * IS>(in + IS, o, dir);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            float2 t = (k == 0) ? o[k] : cmul(w32(k * (32 / R), dir), o[k]);
            out[k] = cadd(e[k], t);
            out[k + R / 2] = csub(e[k], t);
        }
    }
}

// Bit reversal of r < 32 over 5 bits, branch- and loop-free so that it folds
// to a constant for unrolled r.
__host__ __device__ constexpr int brev5(int r)
{
    return ((r & 1) << 4) | ((r & 2) << 2) | (r & 4) | ((r & 8) >> 2) | ((r & 16) >> 4);
}

template <int R>
struct Lg {
    static constexpr int v = R >= 32 ? 5 : R >= 16 ? 4 : R >= 8 ? 3 : R >= 4 ? 2 : R >= 2 ? 1 : 0;
};

// One radix-2 stage (butterfly span LEN) of the in-place DIT DFT below, then
// the next stage; template recursion keeps every index a compile-time constant.
template <int R, int LEN>
__device__ __forceinline__ void dft_stage(float2 (&a)[R], float dir)
{
#pragma unroll
    for (int i = 0; i < R; i += LEN) {
#pragma unroll
        for (int k = 0; k < LEN / 2; ++k) {
            float2 o = a[i + k + LEN / 2];
            float2 t = (k == 0) ? o : cmul(w32((k * (32 / LEN)) & 31, dir), o);
            a[i + k + LEN / 2] = sub2(a[i + k], t);
            a[i + k] = add2(a[i + k], t);
        }
    }
    if constexpr (LEN < R) dft_stage<R, 2 * LEN>(a, dir);
}

// In-place radix-2 DIT DFT of R values held in registers, a[] given in
// bit-reversed order; on return a[q] = sum_r x[r] exp(dir*2*pi*i*r*q/R).
// Only the R values are live, so a 32-point DFT needs 64 registers.
template <int R>
__device__ __forceinline__ void dft_inplace(float2 (&a)[R], float dir)
{
    if constexpr (R >= 2) dft_stage<R, 2>(a, dir);
}

// ----------------------------------------------- mixed-radix (3, 5) DFTs ----
// Twiddles of DFT lengths that are not powers of two, as compile-time
// constants: cos and sin of 2 pi m / n by their Taylor series in double after
// reduction to [-pi, pi] (16 terms leave an error below 1e-18), rounded to
// float once.
constexpr double kTwoPiD = 6.283185307179586476925286766559;
__host__ __device__ constexpr double ct_angle(int m, int n)
{
    const double t = kTwoPiD * (double)(((m % n) + n) % n) / (double)n;
    return t > kTwoPiD / 2 ? t - kTwoPiD : t;
}
__host__ __device__ constexpr double ct_sin(double x)
{
    double term = x, sum = x;
    for (int k = 1; k < 16; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double ct_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 16; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}

// v * exp(dir * 2 pi i m / n), the factor a compile-time constant.
template <int N, int M>
__device__ __forceinline__ float2 tw_mul(float2 v, float dir)
{
    if constexpr (M % N == 0) {
        return v;
    } else {
        constexpr float c = (float)ct_cos(ct_angle(M, N)), s = (float)ct_sin(ct_angle(M, N));
        const float sd = dir * s;
        return make_float2(fmaf(v.x, c, -sd * v.y), fmaf(v.x, sd, v.y * c));
    }
}

// 3- and 5-point DFTs in place (natural order), sign dir.  With
// w = exp(dir 2 pi i / P): X_k = sum_r x_r w^(r k), written as sums and
// differences of the symmetric pairs x_r +- x_(P-r).
__device__ __forceinline__ void dft3(float2 (&a)[3], float dir)
{
    constexpr float h = 0.8660254037844386f;   // sin(2 pi / 3)
    const float2 s = add2(a[1], a[2]), d = sub2(a[1], a[2]);
    const float2 m = make_float2(fmaf(-0.5f, s.x, a[0].x), fmaf(-0.5f, s.y, a[0].y));
    const float hd = dir * h;
    const float2 id = make_float2(-hd * d.y, hd * d.x);   // i dir h (x1 - x2)
    a[0] = add2(a[0], s);
    a[1] = add2(m, id);
    a[2] = sub2(m, id);
}

__device__ __forceinline__ void dft5(float2 (&a)[5], float dir)
{
    constexpr float c1 = (float)ct_cos(ct_angle(1, 5)), c2 = (float)ct_cos(ct_angle(2, 5));
    constexpr float s1 = (float)ct_sin(ct_angle(1, 5)), s2 = (float)ct_sin(ct_angle(2, 5));
    const float2 t1 = add2(a[1], a[4]), t2 = add2(a[2], a[3]), t3 = sub2(a[1], a[4]), t4 = sub2(a[2], a[3]);
    const float2 x0 = a[0];
    const float2 p1 = make_float2(fmaf(c2, t2.x, fmaf(c1, t1.x, x0.x)), fmaf(c2, t2.y, fmaf(c1, t1.y, x0.y)));
    const float2 p2 = make_float2(fmaf(c1, t2.x, fmaf(c2, t1.x, x0.x)), fmaf(c1, t2.y, fmaf(c2, t1.y, x0.y)));
    // q1 = dir (s1 t3 + s2 t4), q2 = dir (s2 t3 - s1 t4); X1,4 = p1 +- i q1, X2,3 = p2 +- i q2
    const float2 q1 = make_float2(dir * fmaf(s1, t3.x, s2 * t4.x), dir * fmaf(s1, t3.y, s2 * t4.y));
    const float2 q2 = make_float2(dir * fmaf(s2, t3.x, -s1 * t4.x), dir * fmaf(s2, t3.y, -s1 * t4.y));
    a[0] = add2(x0, add2(t1, t2));
    a[1] = make_float2(p1.x - q1.y, p1.y + q1.x);
    a[4] = make_float2(p1.x + q1.y, p1.y - q1.x);
    a[2] = make_float2(p2.x - q2.y, p2.y + q2.x);
    a[3] = make_float2(p2.x + q2.y, p2.y - q2.x);
}

template <int P>
__device__ __forceinline__ void dft_small(float2 (&a)[P], float dir)
{
    static_assert(P == 3 || P == 5, "radix 3 or 5");
    if constexpr (P == 3) dft3(a, dir);
    else dft5(a, dir);
}

// Twiddles y[q][k1] *= exp(dir 2 pi i q k1 / R) of the mixed-radix step,
// each factor a compile-time constant (index sequences unroll q and k1).
template <int R, int P, int Q, int q, int... K1>
__device__ __forceinline__ void tw_row(float2 (&yq)[P], float dir, std::integer_sequence<int, K1...>)
{
    ((yq[K1] = tw_mul<R, q * K1>(yq[K1], dir)), ...);
}
template <int R, int P, int Q, int... Qs>
__device__ __forceinline__ void tw_all(float2 (&y)[Q][P], float dir, std::integer_sequence<int, Qs...>)
{
    (tw_row<R, P, Q, Qs>(y[Qs], dir, std::make_integer_sequence<int, P>{}), ...);
}

// DFT of R values in registers, natural order in and out:
// a[k] <- sum_r a[r] exp(dir 2 pi i r k / R).  R a power of two (radix-2
// DIT above, after a bit-reversal that only renames registers) or R = P Q with
// P = 3 or 5 and Q a power of two (Cooley-Tukey: P-point DFTs over
// r = Q p + q, twiddles exp(dir 2 pi i q k1 / R), Q-point DFTs over q, k =
// k1 + P k2).
template <int R>
__device__ __forceinline__ void dft_nat(float2 (&a)[R], float dir)
{
    if constexpr ((R & (R - 1)) == 0) {
        constexpr int L = Lg<R>::v;
        float2 t[R];
#pragma unroll
        for (int r = 0; r < R; ++r) t[brev5(r) >> (5 - L)] = a[r];
        dft_inplace<R>(t, dir);
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = t[r];
    } else {
        constexpr int P = (R % 5 == 0) ? 5 : 3, Q = R / P;
        static_assert(R % P == 0 && (Q & (Q - 1)) == 0 && Q <= 32, "R = 3 or 5 times a power of two");
        constexpr int LQ = Lg<Q>::v;
        float2 y[Q][P];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
#pragma unroll
            for (int p = 0; p < P; ++p) y[q][p] = a[Q * p + q];
            dft_small<P>(y[q], dir);
        }
        tw_all<R, P, Q>(y, dir, std::make_integer_sequence<int, Q>{});
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            float2 u[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) u[LQ ? (brev5(q) >> (5 - LQ)) : 0] = y[q][k1];
            dft_inplace<Q>(u, dir);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) a[k1 + P * k2] = u[k2];
        }
    }
}

// One radix-2 decimation-in-frequency stage (butterfly span LEN), then the
// next, shorter one.
template <int R, int LEN>
__device__ __forceinline__ void dif_stage(float2 (&a)[R], float dir)
{
#pragma unroll
    for (int i = 0; i < R; i += LEN) {
#pragma unroll
        for (int k = 0; k < LEN / 2; ++k) {
            const float2 p = a[i + k], q = a[i + k + LEN / 2];
            a[i + k] = add2(p, q);
            const float2 d = sub2(p, q);
            a[i + k + LEN / 2] = (k == 0) ? d : cmul(w32((k * (32 / LEN)) & 31, dir), d);
        }
    }
    if constexpr (LEN > 2) dif_stage<R, LEN / 2>(a, dir);
}

// In-place radix-2 DIF DFT of R values held in registers, a[] given in
// natural order; on return a[brev(q)] = sum_r x[r] exp(dir*2*pi*i*r*q/R)
// (brev over log2 R bits).  The mirror of dft_inplace: the two compose
// without a register permutation in between.
template <int R>
__device__ __forceinline__ void dft_dif_inplace(float2 (&a)[R], float dir)
{
    if constexpr (R >= 2) dif_stage<R, R>(a, dir);
}

// Position of point p in the intermediate buffer s.  With SWZ, points p and
// p ^ 1 trade places when bit zs of p is set (zs = log2 of the first pass's
// radix).  The first pass writes points j*R + r, so with an unpadded stride
// of 64 bytes (SB = B = 8) the four butterflies j of a warp would all land on
// the same 16 banks; the swap puts two of them on the other 16, and the
// contiguous accesses of the later passes keep two even and two odd rows per
// warp, so every 8-byte access of the FFT is conflict-free.
template <bool SWZ>
__device__ __forceinline__ int swz_pos(int p, int zs)
{
    if constexpr (SWZ) return p ^ ((p >> zs) & 1);
    else return p;
}

// One Stockham pass of radix R over n points for B slices, E values per
// thread (E/R butterflies).  FIRST: inputs come from ld(pos, b) instead of
// s[pos*SB + b]; LAST: outputs go to st(pos, b, value) instead of s.  A
// barrier separates the reads of a pass from its writes, so ld may read s
// and st may write s; the caller syncs after a LAST pass if st wrote s.
template <int R, int B, int SB, int E, bool FIRST, bool LAST, bool GUARD, bool SWZ, bool TWS, class Ld, class St>
__device__ __forceinline__ void fpass(float2 *s, int n, int Ns, const float2 *tw, float dir, Ld &ld, St &st,
                                      int T, int zs)
{
    constexpr int Q = E / R;
    constexpr int LB = Log2B<B>::v;
    const int nb = n / R;
    const bool act = !GUARD || (int)threadIdx.x < T;
    const int step = n / (Ns * R);
    float2 v[Q][R];
    if (act) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int item = threadIdx.x + q * T;
            int b = item & (B - 1), j = item >> LB;
            int k = j & (Ns - 1);
            // Inter-pass twiddle w^(r k step), w = exp(-dir 2 pi i / n): read
            // from the table for r = 0, 8, 16, 24 and stepped by w^(k step)
            // in between (at most 7 products from a table value).
            // With TWS the table is in shared memory and every twiddle is
            // read from it (r k step < n).
            float2 w1 = make_float2(1.f, 0.f), w = w1;
            if (!TWS && !FIRST && Ns > 1) {
                w1 = __ldg(&tw[k * step]);
                w1.y = -dir * w1.y;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 x;
                if constexpr (FIRST) x = ld(j + r * nb, b);
                else x = s[swz_pos<SWZ>(j + r * nb, zs) * SB + b];
                if (TWS && !FIRST && r > 0 && Ns > 1) {
                    w = tw[r * k * step];
                    w.y = -dir * w.y;
                    x = cmul(x, w);
                } else if (!FIRST && r > 0 && Ns > 1) {
                    if ((r & 7) == 0) {
                        w = __ldg(&tw[r * k * step]);
                        w.y = -dir * w.y;
                    } else {
                        w = (r & 7) == 1 ? ((r == 1) ? w1 : cmul(w, w1)) : cmul(w, w1);
                    }
                    x = cmul(x, w);
                }
                v[q][brev5(r) >> (5 - Lg<R>::v)] = x;
            }
            dft_inplace<R>(v[q], dir);
        }
    }
    __syncthreads();   // all reads of s (or of ld's buffer) done before any write
    if (act) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int item = threadIdx.x + q * T;
            int b = item & (B - 1), j = item >> LB;
            int k = j & (Ns - 1);
            int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (LAST) st(base + r * Ns, b, v[q][r]);
                else s[swz_pos<SWZ>(base + r * Ns, zs) * SB + b] = v[q][r];
            }
        }
    }
    if constexpr (!LAST) __syncthreads();
}

template <int R, int B, int SB, int E, bool GUARD, bool SWZ, bool TWS, class Ld, class St>
__device__ __forceinline__ void fpass_any(bool first, bool last, float2 *s, int n, int Ns, const float2 *tw, float dir,
                                          Ld &ld, St &st, int T, int zs)
{
    if (first) {
        if (last) fpass<R, B, SB, E, true, true, GUARD, SWZ, TWS>(s, n, Ns, tw, dir, ld, st, T, zs);
        else fpass<R, B, SB, E, true, false, GUARD, SWZ, TWS>(s, n, Ns, tw, dir, ld, st, T, zs);
    } else {
        if (last) fpass<R, B, SB, E, false, true, GUARD, SWZ, TWS>(s, n, Ns, tw, dir, ld, st, T, zs);
        else fpass<R, B, SB, E, false, false, GUARD, SWZ, TWS>(s, n, Ns, tw, dir, ld, st, T, zs);
    }
}

// Unnormalised FFT of length n = 2^lg for each of B slices, computed by the
// first n*B/E threads of the block: blockDim.x == n*B/E unless GUARD, in which
// case extra threads only take part in the barriers.  The first pass reads ld(pos, b) (natural order), the last pass
// hands st(pos, b, value) the outputs in natural order; intermediate passes
// use s[n][SB] (positions permuted by swz_pos<SWZ>).  The first pass has no
// twiddles (Ns = 1).  E is 16 or 32: passes of radix E after one pass of
// radix 2^(lg mod log2 E).
// TWS: tw is a copy of the table in shared memory (every twiddle read from
// it); otherwise tw is global and twiddles between table reads are products.
template <int B, int SB, int E, bool GUARD = false, bool SWZ = false, bool TWS = false, class Ld, class St>
__device__ __forceinline__ void fft_fused(float2 *s, int n, int lg, const float2 *tw, float dir, Ld &ld, St &st)
{
    constexpr int LE = (E == 32) ? 5 : 4;
    const int T = n * B / E;
    const int rem = lg % LE;
    const int zs = rem ? rem : LE;   // log2 of the first pass's radix
    int Ns = 1;
    bool first = true;
    if (rem) {
        bool last = (1 << rem) == n;
        switch (rem) {
        case 1: fpass_any<2, B, SB, E, GUARD, SWZ, TWS>(first, last, s, n, Ns, tw, dir, ld, st, T, zs); break;
        case 2: fpass_any<4, B, SB, E, GUARD, SWZ, TWS>(first, last, s, n, Ns, tw, dir, ld, st, T, zs); break;
        case 3: fpass_any<8, B, SB, E, GUARD, SWZ, TWS>(first, last, s, n, Ns, tw, dir, ld, st, T, zs); break;
        default:
            if constexpr (E == 32) fpass_any<16, B, SB, E, GUARD, SWZ, TWS>(first, last, s, n, Ns, tw, dir, ld, st, T, zs);
            break;
        }
        Ns = 1 << rem;
        first = false;
    }
    while (Ns < n) {
        bool last = Ns * E == n;
        fpass_any<E, B, SB, E, GUARD, SWZ, TWS>(first, last, s, n, Ns, tw, dir, ld, st, T, zs);
        Ns *= E;
        first = false;
    }
}

// Row stride (in float2) of the gather buffers: padded so that 16-byte loads
// of eight neighbouring rows fall in different banks.
// Asynchronous global -> shared copies (cp.async): the copies of a thread
// are all in flight at once; commit_group closes a group, wait_group<N>
// waits until at most N of the thread's groups are pending.
__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

template <int N>
__device__ __forceinline__ void cp_async(void *dst, const void *src)
{
    static_assert(N == 4 || N == 8 || N == 16, "cp.async copies 4, 8 or 16 bytes");
    if constexpr (N == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst)), "l"(src), "n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Block-wide asynchronous copy of `bytes` (a multiple of 4) in the widest
// units that the two addresses and the size allow.
__device__ __forceinline__ void copy_async(void *dst, const void *src, size_t bytes)
{
    const size_t al = (size_t)dst | (size_t)src | bytes;
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    if ((al & 15) == 0) {
        for (size_t o = (size_t)threadIdx.x * 16; o < bytes; o += (size_t)blockDim.x * 16) cp_async<16>(d + o, s + o);
    } else if ((al & 7) == 0) {
        for (size_t o = (size_t)threadIdx.x * 8; o < bytes; o += (size_t)blockDim.x * 8) cp_async<8>(d + o, s + o);
    } else {
        for (size_t o = (size_t)threadIdx.x * 4; o < bytes; o += (size_t)blockDim.x * 4) cp_async<4>(d + o, s + o);
    }
}

template <int B>
struct RowStride {
    static constexpr int v = (B == 8) ? 10 : (B == 4) ? 6 : B;
};

// Deterministic block reduction of per-thread doubles where thread t holds a
// value for slice t % B; blockDim.x is a multiple of B and a power of two.
// Returns, in threads t < B, the sum for slice t.  scratch: blockDim.x doubles.
__device__ __forceinline__ double block_sum_per_slice(double v, double *scratch, int B)
{
    scratch[threadIdx.x] = v;
    __syncthreads();
    // A block of T threads that is not a power of two (the Toeplitz y-pass
    // of a mixed-radix length) first folds threads P2.. onto 0.. (P2 the
    // largest power of two below T, a multiple of B, so slices stay apart).
    const int P2 = 1 << (31 - __clz((int)blockDim.x));
    if (P2 < (int)blockDim.x) {
        if ((int)threadIdx.x < (int)blockDim.x - P2) scratch[threadIdx.x] += scratch[threadIdx.x + P2];
        __syncthreads();
    }
    for (int stride = P2 >> 1; stride >= B; stride >>= 1) {
        if ((int)threadIdx.x < stride) scratch[threadIdx.x] += scratch[threadIdx.x + stride];
        __syncthreads();
    }
    double r = scratch[threadIdx.x];
    __syncthreads();
    return r;
}

}  // namespace icon
