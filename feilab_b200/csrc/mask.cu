// mask.cu -- volume assembly with the cross-validation mask on the GPU:
// replaces ICONMask3 (sourceCode/ICONMask3/
// ICONCrossVMaskIn2D_weightOnlyOnSampled.cu, MK below).  C ABI in
// include/icon_tools.h.
//
// The filter is built on the host with the reference's float and double
// steps (sampling mask MK:1107-1139, genMask MK:369-456); each slice is then
// filtered by a 2-D FFT built from this library's fused FFT passes
// (icon_device.cuh): FFT of every row, then per column FFT, times the
// filter, inverse FFT, then the inverse FFT of only the rows the crop keeps,
// divided by n*n (MK:479-600).  The reference filters the half spectrum with
// R2C/C2R; here the full spectrum is filtered with the filter's Hermitian
// extension (value at (-ky, -kx) for kx > n/2) and the real part kept,
// which is what C2R computes, including on the kx = 0 and kx = n/2 columns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_device.cuh"
#include "icon_tools.h"

extern "C" void icon_internal_set_error(const char *msg);

namespace {

icon_status mask_fail(icon_status st, const std::string &msg)
{
    icon_internal_set_error(msg.c_str());
    return st;
}

constexpr double kPi180 = 0.01745329252;   // MK:8

template <int E>
__global__ void __launch_bounds__(512) k_mask_rows_fwd(const float *__restrict__ slices, float2 *__restrict__ C, int n,
                                                        int lg, const float2 *__restrict__ tw)
{
    extern __shared__ float2 s[];
    const int y = blockIdx.x, sl = blockIdx.y;
    const float *row = slices + ((size_t)sl * n + y) * n;
    float2 *crow = C + ((size_t)sl * n + y) * n;
    auto ld = [=](int q, int) -> float2 { return make_float2(row[q], 0.f); };
    auto st = [=](int k, int, float2 v) { crow[k] = v; };
    icon::fft_fused<1, 1, E>(s, n, lg, tw, -1.f, ld, st);
}

template <int E>
__global__ void __launch_bounds__(512) k_mask_cols(float2 *__restrict__ C, const float *__restrict__ M, int n, int lg,
                                                    const float2 *__restrict__ tw)
{
    extern __shared__ float2 s[];
    float2 *s2 = s + n;
    const int kx = blockIdx.x, sl = blockIdx.y;
    float2 *col = C + (size_t)sl * n * n + kx;
    auto ld1 = [=](int q, int) -> float2 { return col[(size_t)q * n]; };
    auto st1 = [=](int ky, int, float2 v) {
        const float m = M[(size_t)ky * n + kx];
        s2[ky] = make_float2(v.x * m, v.y * m);
    };
    icon::fft_fused<1, 1, E>(s, n, lg, tw, -1.f, ld1, st1);
    __syncthreads();
    auto ld2 = [=](int q, int) -> float2 { return s2[q]; };
    auto st2 = [=](int y, int, float2 v) { col[(size_t)y * n] = v; };
    icon::fft_fused<1, 1, E>(s, n, lg, tw, +1.f, ld2, st2);
}

template <int E>
__global__ void __launch_bounds__(512) k_mask_rows_inv(const float2 *__restrict__ C, float *__restrict__ out, int n,
                                                        int lg, const float2 *__restrict__ tw, int ystart,
                                                        int thickness, double norm)
{
    extern __shared__ float2 s[];
    const int r = blockIdx.x, sl = blockIdx.y;
    const float2 *crow = C + ((size_t)sl * n + ystart + r) * n;
    float *orow = out + ((size_t)sl * thickness + r) * n;
    auto ld = [=](int k, int) -> float2 { return crow[k]; };
    auto st = [=](int x, int, float2 v) { orow[x] = (float)((double)v.x / norm); };   // MK:598 divides by n*n
    icon::fft_fused<1, 1, E>(s, n, lg, tw, +1.f, ld, st);
}

__global__ void k_crop(const float *__restrict__ slices, float *__restrict__ out, int n, int S, int ystart, int thickness)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)S * thickness * n;
    if (i >= total) return;
    const int x = (int)(i % n), r = (int)((i / n) % thickness), sl = (int)(i / ((size_t)n * thickness));
    out[i] = slices[((size_t)sl * n + ystart + r) * n + x];
}

int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

}  // namespace

// Host part of the filter, exported to the C ABI below.
namespace icon_mask_host {

// MK:996-1016: fallback radius from the tilt span and the mean tilt step.
void angular_steps(const float *t, int nt, int &biggest_radius, float &mean_step)
{
    float hi = -1.f, lo = 1.f;
    for (int i = 0; i < nt; ++i) {
        if (hi < t[i]) hi = t[i];
        if (lo > t[i]) lo = t[i];
    }
    float span = hi - lo;
    biggest_radius = (int)std::ceil(2 * 180.0 / 3.1415926 / span);
    float m = 0.f;
    for (int i = 0; i < nt - 1; ++i) m += std::fabs(t[i + 1] - t[i]);
    mean_step = m / (nt - 1);
}

// MK:1107-1139: sampling mask [n][n].
std::vector<float> sampling_mask(int n, const float *t, int nt)
{
    const int nx = n, ny = n;
    std::vector<float> orig((size_t)n * n, 0.f), rot((size_t)n * n);
    for (int k = 0; k < nt; ++k) {
        const float c = (float)std::cos((-t[k] - 90) * kPi180), s = (float)std::sin((-t[k] - 90) * kPi180);
        std::fill(rot.begin(), rot.end(), 0.f);
        const int i = nx / 2;
        for (int j = 0; j < ny; ++j) {
            const float xf = (float)(i - nx / 2) * c - (float)(j - ny / 2) * s + nx / 2;
            const float yf = (float)(i - nx / 2) * s + (float)(j - ny / 2) * c + ny / 2;
            const int xi = (int)xf, yi = (int)yf;
            const float dx = xf - xi, dy = yf - yi;
            if (xi >= 0 && xi < nx && yi >= 0 && yi < ny) rot[(size_t)yi * nx + xi] += 1.0f * (1 - dx) * (1 - dy);
            if (xi >= 0 && xi < nx && yi + 1 >= 0 && yi + 1 < ny) rot[(size_t)(yi + 1) * nx + xi] += 1.0f * (1 - dx) * dy;
            if (xi + 1 >= 0 && xi + 1 < nx && yi >= 0 && yi < ny) rot[(size_t)yi * nx + xi + 1] += 1.0f * dx * (1 - dy);
            if (xi + 1 >= 0 && xi + 1 < nx && yi + 1 >= 0 && yi + 1 < ny) rot[(size_t)(yi + 1) * nx + xi + 1] += 1.0f * dx * dy;
        }
        for (size_t q = 0; q < orig.size(); ++q) orig[q] += rot[q];
    }
    for (auto &v : orig)
        if (v > 1) v = 1;
    return orig;
}

// MK:369-456 with MK:458-468: filter = realMask * weighting on [n][n/2+1].
std::vector<float> half_filter(int n, const float *t, int nt, float rate05, float rate03, int explicit_radius,
                               int gauss_width)
{
    std::vector<float> orig = sampling_mask(n, t, nt);
    int big;
    float mean_step;
    angular_steps(t, nt, big, mean_step);
    const int r_full = (int)std::ceil(2.0 / (mean_step / 360.0 * 2 * 3.1415926));
    const int radius05 = (int)((float)n / 2.0 * rate05);
    const int radius03 = (int)((float)n / 2.0 * rate03);
    long glmax;
    if (!explicit_radius) glmax = gauss_width > 0 ? gauss_width : radius03 - radius05;
    else glmax = gauss_width > 0 ? gauss_width : (long)(10.0 * (n / 150.0));
    if (glmax < 10.0 * (n / 150.0)) glmax = (long)(10.0 * (n / 150.0));
    const int radius = radius05;
    const long gradius = radius + glmax, glen = gradius - radius;
    const double c = (double)glen / 3.0;
    const double e0 = std::exp(-(double)(glen * glen) / (2 * c * c));
    const int nh = n / 2 + 1;
    std::vector<float> f((size_t)n * nh);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < nh; ++i) {
            const int i1 = (i + n / 2) % n, j1 = (j + n / 2) % n;
            const long rr = (long)std::sqrt((double)((i1 - n / 2) * (i1 - n / 2) + (j1 - n / 2) * (j1 - n / 2)));
            const double o = orig[(size_t)j1 * n + i1];
            float m = 1.f;
            if (rr >= radius) {
                if (rr <= gradius) {
                    const double x = (double)(rr - radius);
                    const double w2 = (std::exp(-(x * x) / (2 * c * c)) - e0) / (1 - e0);
                    m = (float)(o > w2 ? o : w2);
                } else {
                    m = (float)o;
                }
            }
            const float w = (rr > r_full && std::fabs(o) > 0.00001) ? (float)rr / (float)r_full : 1.f;
            f[(size_t)j * nh + i] = m * w;
        }
    return f;
}

}  // namespace icon_mask_host

struct icon_mask {
    int dev = 0, n = 0, lg = 0, cap = 0, E = 16;
    std::vector<float> half;
    float2 *C = nullptr, *tw = nullptr;
    float *M = nullptr;
    ~icon_mask()
    {
        cudaFree(C);
        cudaFree(tw);
        cudaFree(M);
    }
};

extern "C" {

icon_status icon_mask_radius(int n, const float *tilts, int ntilt, int radius, const float *crossv,
                             const float *fullrec, int frc_len, float *rate05, float *rate03, int *explicit_radius)
{
    if (n < 2 || !tilts || ntilt < 2 || !rate05 || !rate03 || !explicit_radius)
        return mask_fail(ICON_ERR_INVALID, "icon_mask_radius: bad argument");
    int big;
    float mean;
    icon_mask_host::angular_steps(tilts, ntilt, big, mean);
    if (radius < 0) {   // MK:1033-1100
        bool valid = crossv && fullrec && frc_len >= n / 2 - 1;
        if (valid) {
            std::vector<float> cv(crossv, crossv + frc_len);
            for (int i = 0; i < frc_len; ++i)
                if (fullrec[i] != 0) cv[i] /= fullrec[i];
            int r05 = frc_len - 1, r03 = frc_len - 1;
            while (r05 >= 0 && !(cv[r05] >= 0.5f)) --r05;
            while (r03 >= 0 && !(cv[r03] >= 0.3f)) --r03;
            if (r05 > r03 || r03 == 0) valid = false;
            if (valid) {
                *rate05 = (float)r05 / (float)frc_len;
                *rate03 = (float)r03 / (float)frc_len;
                *explicit_radius = 0;
                return ICON_OK;
            }
        }
        radius = big;
    }
    *rate05 = (float)((float)radius / ((float)n / 2.0));
    *rate03 = 0.f;
    *explicit_radius = 1;
    return ICON_OK;
}

icon_status icon_mask_create(int n, const float *tilts, int ntilt, float rate05, float rate03, int explicit_radius,
                             int gauss_width, int capacity, icon_mask **out)
{
    if (!out || !tilts || ntilt < 2 || capacity < 1) return mask_fail(ICON_ERR_INVALID, "icon_mask_create: bad argument");
    *out = nullptr;
    if (n < 16 || n > 8192 || (n & (n - 1)))
        return mask_fail(ICON_ERR_INVALID, "icon_mask_create: slice size must be a power of two in 16..8192");
    auto m = std::make_unique<icon_mask>();
    cudaGetDevice(&m->dev);
    m->n = n;
    m->lg = ilog2(n);
    m->cap = capacity;
    m->E = (n >= 1024) ? 32 : 16;
    m->half = icon_mask_host::half_filter(n, tilts, ntilt, rate05, rate03, explicit_radius, gauss_width);
    // Full-spectrum filter: the Hermitian partner's value for kx > n/2.
    const int nh = n / 2 + 1;
    std::vector<float> full((size_t)n * n);
    for (int ky = 0; ky < n; ++ky)
        for (int kx = 0; kx < n; ++kx)
            full[(size_t)ky * n + kx] = kx < nh ? m->half[(size_t)ky * nh + kx]
                                                : m->half[(size_t)((n - ky) % n) * nh + (n - kx)];
    std::vector<float2> tw(n);
    for (int q = 0; q < n; ++q) {
        const double a = 2.0 * M_PI * (double)q / (double)n;
        tw[q] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    if (cudaMalloc(&m->C, sizeof(float2) * (size_t)capacity * n * n) != cudaSuccess ||
        cudaMalloc(&m->tw, sizeof(float2) * n) != cudaSuccess || cudaMalloc(&m->M, sizeof(float) * (size_t)n * n) != cudaSuccess) {
        cudaGetLastError();
        return mask_fail(ICON_ERR_NOMEM, "icon_mask_create: device memory");
    }
    if (cudaMemcpy(m->tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->M, full.data(), sizeof(float) * full.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return mask_fail(ICON_ERR_CUDA, "icon_mask_create: copy of the filter");
    // The limit belongs to the kernel function, shared by masks of every
    // size: raise it to the device's opt-in maximum rather than to this
    // mask's need, which would lower it under a larger mask made earlier.
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess && (size_t)optin < sizeof(float2) * 2 * n)
        return mask_fail(ICON_ERR_INVALID, "icon_mask_create: slice too large for shared memory");
    if (e == cudaSuccess && m->E == 32) {
        e = cudaFuncSetAttribute(k_mask_cols<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mask_rows_fwd<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mask_rows_inv<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    } else if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_mask_cols<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    }
    if (e != cudaSuccess) return mask_fail(ICON_ERR_CUDA, std::string("icon_mask_create: ") + cudaGetErrorString(e));
    *out = m.release();
    return ICON_OK;
}

icon_status icon_mask_destroy(icon_mask *m)
{
    if (!m) return ICON_OK;
    cudaDeviceSynchronize();
    delete m;
    return ICON_OK;
}

icon_status icon_mask_filter(const icon_mask *m, float *h_filter)
{
    if (!m || !h_filter) return mask_fail(ICON_ERR_INVALID, "icon_mask_filter: null argument");
    std::copy(m->half.begin(), m->half.end(), h_filter);
    return ICON_OK;
}

icon_status icon_mask_apply(icon_mask *m, const float *d_slices, int S, int ystart, int thickness, float *d_out,
                            void *stream)
{
    if (!m || !d_slices || !d_out) return mask_fail(ICON_ERR_INVALID, "icon_mask_apply: null argument");
    if (S < 1 || S > m->cap) return mask_fail(ICON_ERR_CAPACITY, "icon_mask_apply: S outside 1..capacity");
    const int n = m->n;
    if (thickness < 1 || ystart < 0 || ystart + thickness > n)
        return mask_fail(ICON_ERR_INVALID, "zshift & thickness make the size of volume out of limitation");
    cudaStream_t st = (cudaStream_t)stream;
    const int T = n / m->E;
    const size_t smem1 = sizeof(float2) * n, smem2 = sizeof(float2) * 2 * n;
    const double norm = (double)n * (double)n;
    if (m->E == 32) {
        k_mask_rows_fwd<32><<<dim3(n, S), T, smem1, st>>>(d_slices, m->C, n, m->lg, m->tw);
        k_mask_cols<32><<<dim3(n, S), T, smem2, st>>>(m->C, m->M, n, m->lg, m->tw);
        k_mask_rows_inv<32><<<dim3(thickness, S), T, smem1, st>>>(m->C, d_out, n, m->lg, m->tw, ystart, thickness, norm);
    } else {
        k_mask_rows_fwd<16><<<dim3(n, S), T, smem1, st>>>(d_slices, m->C, n, m->lg, m->tw);
        k_mask_cols<16><<<dim3(n, S), T, smem2, st>>>(m->C, m->M, n, m->lg, m->tw);
        k_mask_rows_inv<16><<<dim3(thickness, S), T, smem1, st>>>(m->C, d_out, n, m->lg, m->tw, ystart, thickness, norm);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mask_fail(ICON_ERR_CUDA, std::string("icon_mask_apply: ") + cudaGetErrorString(e));
    return ICON_OK;
}

icon_status icon_mask_apply_host(icon_mask *m, const float *h_slices, int S, int ystart, int thickness, float *h_out)
{
    if (!m || !h_slices || !h_out || S < 1) return mask_fail(ICON_ERR_INVALID, "icon_mask_apply_host: bad argument");
    const int n = m->n;
    float *d_in = nullptr, *d_out = nullptr;
    const size_t in_b = sizeof(float) * (size_t)std::min(S, m->cap) * n * n;
    const size_t out_b = sizeof(float) * (size_t)std::min(S, m->cap) * std::max(thickness, 1) * n;
    if (cudaMalloc(&d_in, in_b) != cudaSuccess || cudaMalloc(&d_out, out_b) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_in);
        return mask_fail(ICON_ERR_NOMEM, "icon_mask_apply_host: device memory");
    }
    icon_status rc = ICON_OK;
    for (int s0 = 0; s0 < S && rc == ICON_OK; s0 += m->cap) {
        const int nb = std::min(m->cap, S - s0);
        cudaError_t e = cudaMemcpy(d_in, h_slices + (size_t)s0 * n * n, sizeof(float) * (size_t)nb * n * n,
                                   cudaMemcpyHostToDevice);
        if (e == cudaSuccess) rc = icon_mask_apply(m, d_in, nb, ystart, thickness, d_out, nullptr);
        if (e == cudaSuccess && rc == ICON_OK)
            e = cudaMemcpy(h_out + (size_t)s0 * thickness * n, d_out, sizeof(float) * (size_t)nb * thickness * n,
                           cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = mask_fail(ICON_ERR_CUDA, std::string("icon_mask_apply_host: ") + cudaGetErrorString(e));
    }
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}

icon_status icon_volume_crop(const float *d_slices, int n, int S, int ystart, int thickness, float *d_out, void *stream)
{
    if (!d_slices || !d_out || n < 1 || S < 1) return mask_fail(ICON_ERR_INVALID, "icon_volume_crop: bad argument");
    if (thickness < 1 || ystart < 0 || ystart + thickness > n)
        return mask_fail(ICON_ERR_INVALID, "zshift & thickness make the size of volume out of limitation");
    const size_t total = (size_t)S * thickness * n;
    k_crop<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_slices, d_out, n, S, ystart, thickness);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mask_fail(ICON_ERR_CUDA, std::string("icon_volume_crop: ") + cudaGetErrorString(e));
    return ICON_OK;
}

}  // extern "C"
