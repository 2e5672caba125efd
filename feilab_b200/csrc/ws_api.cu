// ws_api.cu -- host side of the warm-start network: TMA tensor maps, launch
// of the tensor-core convolution, and the C ABI of include/icon_warmstart.h.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "icon_b200.h"
#include "icon_warmstart.h"
#include "ws_conv.cuh"

extern "C" void icon_internal_set_error(const char *msg);

namespace {

icon_status ws_fail(icon_status st, const std::string &msg)
{
    icon_internal_set_error(msg.c_str());
    return st;
}

#define WS_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return ws_fail(ICON_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

CUtensorMapSwizzle swizzle_for(int cc)
{
    return cc == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : cc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// NHWC BF16 activations [nimg][H][W][C]; box = cc channels x 128 pixels of
// one row.  Loads outside the image read zeros.
icon_status act_map(CUtensorMap *m, const void *ptr, int nimg, int H, int W, int C, int cc)
{
    EncodeTiled enc = encode_fn();
    if (!enc) return ws_fail(ICON_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)nimg};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)cc, (cuuint32_t)ws::kTileM, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cc), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return ws_fail(ICON_ERR_CUDA, "activation tensor map: error " + std::to_string((int)r));
    return ICON_OK;
}

// Weights [9][N][Cin] BF16; box = cc input channels x N output channels of one tap.
icon_status weight_map(CUtensorMap *m, const void *ptr, int N, int Cin, int cc)
{
    EncodeTiled enc = encode_fn();
    if (!enc) return ws_fail(ICON_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[3] = {(cuuint64_t)Cin, (cuuint64_t)N, 9};
    cuuint64_t strides[2] = {(cuuint64_t)Cin * 2, (cuuint64_t)N * Cin * 2};
    cuuint32_t box[3] = {(cuuint32_t)cc, (cuuint32_t)N, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cc), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return ws_fail(ICON_ERR_CUDA, "weight tensor map: error " + std::to_string((int)r));
    return ICON_OK;
}

int pick_cc(int cin0, int cin1)
{
    for (int cc : {64, 32, 16})
        if (cin0 % cc == 0 && (cin1 == 0 || cin1 % cc == 0)) return cc;
    return 0;
}

// Per-device error flag of the tensor-core kernels.
int *device_err_flag()
{
    static std::mutex mu;
    static int *flags[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!flags[dev]) {
        if (cudaMalloc(&flags[dev], sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(flags[dev], 0, sizeof(int)) != cudaSuccess) return nullptr;
    }
    return flags[dev];
}

}  // namespace

// Launches one convolution; used by the network code and exported for tests.
icon_status ws_conv3x3_launch(const void *in0, int cin0, const void *in1, int cin1, int nimg, int H, int W,
                              const void *w, const float *bias, int N, int relu, void *out0, int nsplit, int acc0,
                              void *out1, int acc1, cudaStream_t st, unsigned long long wait_ns = ws::kWaitNs,
                              int hold = 0)
{
    if (!in0 || !w || !out0 || nimg < 1 || H < 1 || W < 1) return ws_fail(ICON_ERR_INVALID, "conv3x3: bad argument");
    if (N < 16 || N > 256 || N % 16) return ws_fail(ICON_ERR_INVALID, "conv3x3: N must be a multiple of 16 in 16..256");
    if (in1 && cin1 < 16) return ws_fail(ICON_ERR_INVALID, "conv3x3: second input needs >= 16 channels");
    if (!in1) cin1 = 0;
    const int cc = pick_cc(cin0, cin1);
    if (!cc) return ws_fail(ICON_ERR_INVALID, "conv3x3: input channels must be multiples of 16");
    if (nsplit <= 0 || nsplit > N || nsplit % 16 || (nsplit < N && !out1))
        return ws_fail(ICON_ERR_INVALID, "conv3x3: bad output split");
    int *err = device_err_flag();
    if (!err) return ws_fail(ICON_ERR_CUDA, "conv3x3: error flag allocation failed");
    CUtensorMap m0, m1, mw;
    icon_status s;
    if ((s = act_map(&m0, in0, nimg, H, W, cin0, cc)) != ICON_OK) return s;
    if ((s = act_map(&m1, in1 ? in1 : in0, nimg, H, W, in1 ? cin1 : cin0, cc)) != ICON_OK) return s;
    if ((s = weight_map(&mw, w, N, cin0 + cin1, cc)) != ICON_OK) return s;
    ws::ConvArgs a;
    a.nin = in1 ? 2 : 1;
    a.cin0 = cin0;
    a.cin1 = cin1;
    a.H = H;
    a.W = W;
    a.cc = cc;
    a.N = N;
    a.nsplit = nsplit;
    a.out0 = (__nv_bfloat16 *)out0;
    a.out1 = (__nv_bfloat16 *)out1;
    a.acc0 = acc0;
    a.acc1 = acc1;
    a.bias = bias;
    a.relu = relu;
    a.err = err;
    a.wait_ns = wait_ns;
    a.hold = hold;
    const size_t smem = ws::conv_smem_bytes(N, cc);
    {
        // The shared-memory limit is a per-device attribute of the kernel.
        static std::mutex mu;
        static bool done[64] = {false};
        int dev = 0;
        WS_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> g(mu);
        if (dev < 0 || dev >= 64) return ws_fail(ICON_ERR_INVALID, "conv3x3: device index out of range");
        if (!done[dev]) {
            WS_CUDA(cudaFuncSetAttribute(ws::k_conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
            done[dev] = true;
        }
    }
    dim3 grid((W + ws::kTileM - 1) / ws::kTileM, H, nimg);
    ws::k_conv3x3_tc<<<grid, ws::kConvThreads, smem, st>>>(m0, m1, mw, a);
    WS_CUDA(cudaGetLastError());
    return ICON_OK;
}

extern "C" {

icon_status icon_ws_conv3x3(const void *in0, int cin0, const void *in1, int cin1, int nimg, int H, int W,
                            const void *w, const float *bias, int N, int relu, void *out0, int nsplit, int acc0,
                            void *out1, int acc1, void *stream)
{
    return ws_conv3x3_launch(in0, cin0, in1, cin1, nimg, H, W, w, bias, N, relu, out0, nsplit, acc0, out1, acc1,
                             (cudaStream_t)stream);
}

icon_status icon_ws_conv3x3_wait_test(const void *in0, int cin0, int nimg, int H, int W, const void *w, int N,
                                      void *out0, unsigned wait_us, void *stream)
{
    if (wait_us < 1 || wait_us > 1000000) return ws_fail(ICON_ERR_INVALID, "wait_us must be in 1..1000000");
    return ws_conv3x3_launch(in0, cin0, nullptr, 0, nimg, H, W, w, nullptr, N, 0, out0, N, 0, nullptr, 0,
                             (cudaStream_t)stream, 1000ull * wait_us, 1);
}

icon_status icon_ws_device_error(int *h_code)
{
    if (!h_code) return ws_fail(ICON_ERR_INVALID, "null argument");
    int *err = device_err_flag();
    if (!err) return ws_fail(ICON_ERR_CUDA, "error flag allocation failed");
    WS_CUDA(cudaMemcpy(h_code, err, sizeof(int), cudaMemcpyDeviceToHost));
    WS_CUDA(cudaMemset(err, 0, sizeof(int)));
    return ICON_OK;
}

}  // extern "C"
