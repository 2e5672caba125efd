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

namespace icon {

constexpr int kTaps = 14;   // 2m+2 taps per dimension, m = 6 (nufft_gpu_v8.cuh:5, NU:226)
constexpr int kHalf = 6;    // window half-width m

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
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

// Deterministic block reduction of per-thread doubles where thread t holds a
// value for slice t % B; blockDim.x is a multiple of B and a power of two.
// Returns, in threads t < B, the sum for slice t.  scratch: blockDim.x doubles.
__device__ __forceinline__ double block_sum_per_slice(double v, double *scratch, int B)
{
    scratch[threadIdx.x] = v;
    __syncthreads();
    for (int stride = blockDim.x >> 1; stride >= B; stride >>= 1) {
        if ((int)threadIdx.x < stride) scratch[threadIdx.x] += scratch[threadIdx.x + stride];
        __syncthreads();
    }
    double r = scratch[threadIdx.x];
    __syncthreads();
    return r;
}

}  // namespace icon
