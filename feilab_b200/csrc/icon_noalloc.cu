// icon_noalloc.cu -- icon_rows_forward_noalloc: the 1-D NUFFT of projection
// rows without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc -- a process that hands
// all device memory to its own pool allocator at start-up and forbids other
// allocations, or a real-time acquisition loop that must not allocate because
// cudaMalloc can block on and synchronise the device.  Such callers cannot
// create an icon_plan (plans own their scratch).  This entry point does the
// work of icon_rows_forward with its scratch -- the window, index,
// deapodisation and twiddle tables -- in one file-scope __device__ array of
// fixed size, so the only memory it touches besides the caller's input and
// output is that array.
//
// The array is a static of this library's device code.  It is allocated when
// the library's device code is loaded on a GPU and stays until the process
// exits.  With lazy module loading (the CUDA default since 12.2) that load
// happens at the first use of the library's device code on each device --
// for a caller of this entry point alone, its first call there -- and the
// load allocates device memory and may synchronise.  So make the first call
// on each device before a pool allocator takes the device's memory and before
// any real-time region or stream capture, or run with
// CUDA_MODULE_LOADING=EAGER, which loads it when the context is created.
// Later calls allocate nothing.
//
// All calls share the array and it keeps the last call's contents; every
// call rewrites all of the tables it reads, so nothing in it has to start at
// zero.  Calls that overlap on a GPU (different streams, or different host
// threads) race on the array and must not be issued.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "icon_b200.h"
#include "icon_device.cuh"

namespace {

constexpr int kNx = ICON_NOALLOC_MAX_NX;
constexpr int kN = 2 * ICON_NOALLOC_MAX_NX;   // largest oversampled length, 2*nextpow2(nx)

// Table layout inside the scratch array (offsets in bytes, 256-aligned).
constexpr size_t kOffPhi = 0;                                                     // float [nx][14]
constexpr size_t kOffIdx = (kOffPhi + sizeof(float) * kNx * icon::kTaps + 255) / 256 * 256;   // int [nx]
constexpr size_t kOffCk = (kOffIdx + sizeof(int) * kNx + 255) / 256 * 256;       // float [nx]
constexpr size_t kOffTw = (kOffCk + sizeof(float) * kNx + 255) / 256 * 256;      // float2 [n]
constexpr size_t kEnd = kOffTw + sizeof(float2) * kN;
static_assert(kEnd <= ICON_NOALLOC_SCRATCH_BYTES, "scratch array too small for its tables");

__device__ __align__(256) unsigned char g_scratch[ICON_NOALLOC_SCRATCH_BYTES];

}  // namespace

extern "C" void icon_internal_set_error(const char *msg);   // icon_api.cu: message for icon_last_error()

namespace {

icon_status na_fail(icon_status st, const std::string &m)
{
    icon_internal_set_error(m.c_str());
    return st;
}

// One thread per row node k (and per twiddle q): the tables of
// cunfft_initPlan_1d (NU:1298-1391) for nodes (k - nx/2)/nx on the n-point
// grid -- window taps as nufft_Phi1dCU (NU:1242-1256), deapodisation as
// nufft_ck1d (NU:1258-1271) -- plus the FFT twiddles exp(-2 pi i q/n).
__global__ void k_na_tables(unsigned char *scr, int nx, int n, float b, float bf)
{
    float *phi = (float *)(scr + kOffPhi);
    int *idx = (int *)(scr + kOffIdx);
    float *ck = (float *)(scr + kOffCk);
    float2 *tw = (float2 *)(scr + kOffTw);
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nx) {
        float x = (float)(((double)(float)t - (double)(float)nx / 2.0) / (double)(float)nx);
        int l0 = (int)(floorf(n * x) - icon::kHalf);
        idx[t] = l0;
#pragma unroll
        for (int q = 0; q < icon::kTaps; ++q) {
            int l = l0 + q;
            float x1 = x - (float)l / (float)n;
            phi[t * icon::kTaps + q] = bf * expf(-((n * x1) * (n * x1) / b));
        }
        double kk = (double)(t - nx / 2);
        const double pi = 3.1415926535898;
        ck[t] = (float)exp(-(double)b * ((pi * kk / (double)n) * (pi * kk / (double)n)));
    }
    if (t < n) {
        double s, c;
        sincospi(2.0 * (double)t / (double)n, &s, &c);
        tw[t] = make_float2((float)c, (float)-s);
    }
}

// Per (tilt i, group of B slices): pad/deapodise row i of each slice, FFT of
// length n in shared memory, interpolate the nx nodes with the 14 taps in
// order (cunfft_trafo_1d, NU:1479-1516), and write b[s][i*nx + k] directly in
// the caller's layout.
__global__ void __launch_bounds__(1024) k_na_rows(const unsigned char *__restrict__ scr, const float *__restrict__ rows,
                                                  float2 *__restrict__ out, int nx, int nz, int n, int lg, int S, int B)
{
    extern __shared__ float2 s[];
    const float *phi = (const float *)(scr + kOffPhi);
    const int *idx = (const int *)(scr + kOffIdx);
    const float *ck = (const float *)(scr + kOffCk);
    const float2 *tw = (const float2 *)(scr + kOffTw);
    const int i = blockIdx.x, grp = blockIdx.y;
    for (int e = threadIdx.x; e < n * B; e += blockDim.x) {
        int b = e % B, x = e / B;
        int X = (x + nx / 2) % n;
        int sl = grp * B + b;
        float2 v = make_float2(0.f, 0.f);
        if (X < nx && sl < S) {
            float c = ck[X];
            v.x = rows[((size_t)sl * nz + i) * nx + X] / c;
            v.y = 0.f / c;
        }
        s[e] = v;
    }
    __syncthreads();
    icon::fft_smem(s, n, lg, B, tw, -1.f);
    const size_t M = (size_t)nx * nz;
    for (int e = threadIdx.x; e < nx * B; e += blockDim.x) {
        int b = e % B, k = e / B;
        int sl = grp * B + b;
        int l0 = idx[k];
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < icon::kTaps; ++q) {
            int x = l0 + q;
            x += (x < 0) ? n : 0;
            x -= (x >= n) ? n : 0;
            float p = phi[k * icon::kTaps + q];
            float2 v = s[x * B + b];
            acc.x = fmaf(v.x, p, acc.x);
            acc.y = fmaf(v.y, p, acc.y);
        }
        if (sl < S) out[(size_t)sl * M + (size_t)i * nx + k] = acc;
    }
}

// On every call, with the device current: the device address of the scratch
// array in the current context (host code cannot use the symbol itself as a
// pointer) and the shared-memory limit of the row kernel.  Both are looked up
// again each time rather than cached, so a context that was reset
// (cudaDeviceReset) and recreated, with the module loaded anew, is handled;
// neither call allocates once the module is loaded.
icon_status device_setup(unsigned char **out)
{
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess) return na_fail(ICON_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    e = cudaFuncSetAttribute(k_na_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * (int)sizeof(float2));
    if (e != cudaSuccess) return na_fail(ICON_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    *out = (unsigned char *)ptr;
    return ICON_OK;
}

}  // namespace

extern "C" icon_status icon_rows_forward_noalloc(const float *d_rows, int nx, int ntilt, int S, void *d_b, void *stream)
{
    if (!d_rows || !d_b) return na_fail(ICON_ERR_INVALID, "null buffer");
    if (nx < 8 || nx > ICON_NOALLOC_MAX_NX)
        return na_fail(ICON_ERR_INVALID, "nx must be in [8, " + std::to_string(ICON_NOALLOC_MAX_NX) + "]");
    if (ntilt < 1 || S < 1) return na_fail(ICON_ERR_INVALID, "ntilt and S must be >= 1");
    unsigned char *scr = nullptr;
    icon_status rc = device_setup(&scr);
    if (rc != ICON_OK) return rc;
    // Grid of the reference: n = 2*nextpow2(nx), window parameters in float
    // (MainCode.cu:66-71, NU:1330-1331).
    float uptop = (float)std::pow(2.0, std::ceil(std::log10((double)nx) / std::log10(2.0)));
    float th = (float)(2.0 * uptop / (double)nx);
    int n = (int)std::ceil(th * (float)nx);
    const double pi = 3.1415926535898;
    float b = (float)((double)(2 * th * icon::kHalf) / ((double)(2 * th - 1) * pi));
    float bf = (float)(1.0 / std::sqrt(pi * (double)b));
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    int B = 8;
    while (B > 1 && (n * B > 16384 || B / 2 >= S)) B /= 2;
    int G = (S + B - 1) / B;
    cudaStream_t st = (cudaStream_t)stream;
    k_na_tables<<<(n + 255) / 256, 256, 0, st>>>(scr, nx, n, b, bf);
    k_na_rows<<<dim3(ntilt, G), n * B / 16, (size_t)n * B * sizeof(float2), st>>>(scr, d_rows, (float2 *)d_b, nx, ntilt, n,
                                                                                  lg, S, B);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(ICON_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ICON_OK;
}
