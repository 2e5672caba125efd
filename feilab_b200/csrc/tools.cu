// tools.cu -- the steps either side of the ICON solve that the reference does
// in its companion tools, on the GPU: stack pre-processing (ICONPreProcess)
// and, in mask.cu, volume assembly with the cross-validation mask
// (ICONMask3).  C ABI in include/icon_tools.h.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_tools.h"

extern "C" void icon_internal_set_error(const char *msg);

namespace {

icon_status tools_fail(icon_status st, const std::string &msg)
{
    icon_internal_set_error(msg.c_str());
    return st;
}

constexpr int kPreThreads = 1024;
constexpr int kPreMaxProjections = 1024;

// Variance factors of the projections, passed by value (8 KB of kernel
// parameters) so the call needs no device memory.
struct PreFactors {
    double f[kPreMaxProjections];
};

// Fixed-order block reduction of one double per thread (blockDim = 1024).
__device__ double block_sum(double v, double *red)
{
    red[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// One block per projection k of in[nz][ny][nx] (ICONPreProcess.c:29-85):
//   mode  = bin of the most pixels (first on ties) of a 256-bin histogram of
//           the central region (10 % margins), bin index
//           floor((v - min) / step), step = (max - min) / 256 in double; the
//           largest pixel falls in bin 256, which is not counted
//   v    -= mode                                (float result)
//   with factor[k] > 0: mean = sum (v / size in float), var = sum (v - mean)^2 / size
//           (double), v = v / sqrt(var) * sqrt(factor[k])
// out may equal in.
__global__ void __launch_bounds__(kPreThreads) k_preprocess(const float *in, float *out, int nx, int ny,
                                                            int normalize, const __grid_constant__ PreFactors factor)
{
    __shared__ double red[kPreThreads];
    __shared__ int hist[256];
    __shared__ float smin[kPreThreads], smax[kPreThreads];
    const size_t size = (size_t)nx * ny;
    const float *p = in + (size_t)blockIdx.x * size;
    float *q = out + (size_t)blockIdx.x * size;
    const int xe = (int)(nx * 0.1), ye = (int)(ny * 0.1);
    const int cw = nx - 2 * xe, ch = ny - 2 * ye;
    const int ncore = cw * ch;
    float lo = p[(size_t)ye * nx + xe], hi = lo;
    for (int i = threadIdx.x; i < ncore; i += blockDim.x) {
        const float v = p[(size_t)(ye + i / cw) * nx + xe + i % cw];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + o]);
            smax[threadIdx.x] = fmaxf(smax[threadIdx.x], smax[threadIdx.x + o]);
        }
        __syncthreads();
    }
    const double mn = smin[0], mx = smax[0];
    const double step = (mx - mn) / 256.0;
    double mode = mn;   // a constant core has no spread (the reference divides by zero there)
    if (step > 0.0) {
        for (int i = threadIdx.x; i < ncore; i += blockDim.x) {
            const float v = p[(size_t)(ye + i / cw) * nx + xe + i % cw];
            const int b = (int)floor(((double)v - mn) / step);
            if (b >= 0 && b < 256) atomicAdd(&hist[b], 1);
        }
        __syncthreads();
        // First bin with the largest count.
        if (threadIdx.x == 0) {
            int best = -1, bi = 0;
            for (int i = 0; i < 256; ++i)
                if (best < hist[i]) {
                    best = hist[i];
                    bi = i;
                }
            red[0] = bi * step + mn;
        }
        __syncthreads();
        mode = red[0];
        __syncthreads();
    }
    const double f = normalize ? factor.f[blockIdx.x] : 0.0;
    if (!(f > 0.0)) {
        for (size_t i = threadIdx.x; i < size; i += blockDim.x) q[i] = (float)((double)p[i] - mode);
        return;
    }
    const float fsize = (float)size;
    double s = 0.0;
    for (size_t i = threadIdx.x; i < size; i += blockDim.x) {
        const float v = (float)((double)p[i] - mode);
        s += (double)(v / fsize);
    }
    const double mean = block_sum(s, red);
    double s2 = 0.0;
    for (size_t i = threadIdx.x; i < size; i += blockDim.x) {
        const double d = (double)(float)((double)p[i] - mode) - mean;
        s2 += d * d / (double)size;
    }
    const double var = block_sum(s2, red);
    const double sv = sqrt(var), sf = sqrt(f);
    for (size_t i = threadIdx.x; i < size; i += blockDim.x) {
        const float v = (float)((double)p[i] - mode);
        q[i] = (float)((double)v / sv * sf);
    }
}

}  // namespace

extern "C" {

icon_status icon_preprocess(const float *d_in, float *d_out, int nx, int ny, int nz, const float *h_tilt_deg,
                            int thickness, void *stream)
{
    if (!d_in || !d_out || nx < 1 || ny < 1 || nz < 1) return tools_fail(ICON_ERR_INVALID, "icon_preprocess: bad argument");
    if ((nx - 2 * (int)(nx * 0.1)) < 1 || (ny - 2 * (int)(ny * 0.1)) < 1)
        return tools_fail(ICON_ERR_INVALID, "icon_preprocess: image too small");
    if (nz > kPreMaxProjections) return tools_fail(ICON_ERR_INVALID, "icon_preprocess: more than 1024 projections");
    cudaStream_t st = (cudaStream_t)stream;
    const bool norm = h_tilt_deg && thickness > 0;
    PreFactors f{};
    if (norm) {
        // ICONPreProcess.c:73-85 with angle = -tilt (:283): 0.33 t / cos(angle in radians, pi = 3.1415926)
        for (int k = 0; k < nz; ++k) {
            const float angle = -h_tilt_deg[k];
            f.f[k] = 0.33 * thickness / std::cos(angle / 180.0 * 3.1415926);
            if (!(f.f[k] > 0.0)) return tools_fail(ICON_ERR_INVALID, "icon_preprocess: tilt angle gives a non-positive variance");
        }
    }
    k_preprocess<<<nz, kPreThreads, 0, st>>>(d_in, d_out, nx, ny, norm ? 1 : 0, f);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tools_fail(ICON_ERR_CUDA, std::string("icon_preprocess: ") + cudaGetErrorString(e));
    return ICON_OK;
}

icon_status icon_preprocess_host(const float *h_in, float *h_out, int nx, int ny, int nz, const float *h_tilt_deg,
                                 int thickness)
{
    if (!h_in || !h_out || nx < 1 || ny < 1 || nz < 1) return tools_fail(ICON_ERR_INVALID, "icon_preprocess_host: bad argument");
    const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
    float *d = nullptr;
    if (cudaMalloc(&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        return tools_fail(ICON_ERR_NOMEM, "icon_preprocess_host: device memory for the stack");
    }
    icon_status rc = ICON_OK;
    cudaError_t e = cudaMemcpy(d, h_in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) rc = icon_preprocess(d, d, nx, ny, nz, h_tilt_deg, thickness, nullptr);
    if (e == cudaSuccess && rc == ICON_OK) e = cudaMemcpy(h_out, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return tools_fail(ICON_ERR_CUDA, std::string("icon_preprocess_host: ") + cudaGetErrorString(e));
    return rc;
}

}  // extern "C"
