// icon_warm.cu -- warm-started solve with the cold-start solve as judge and
// fallback (icon_solve_warm, include/icon_b200.h).
//
// The reference always starts a slice's solve from m = 0 (cudaMemset before
// the loop, Iteration2.cu:33).  A start predicted by the network
// (icon_ws_predict) is only a guess, so this routine accepts a warm result
// per slice only when it passes checks that cost a small part of a solve:
//   * finite (a broken network output gives NaN or infinity);
//   * converged: the ICON phase's last relative step ||m_new - m_old|| /
//     ||m_new|| is within the tolerance (icon_solve_until);
//   * close to what the cold start would see first: ||m - m_infr|| <=
//     max_dist ||m_infr||, m_infr the cold start's iterate after the first
//     INFR phase (the first cfg->infr_before iterations from m = 0).  A start
//     far off in the missing wedge survives the iterations there (the data
//     do not constrain it), and this bound rejects it.
// Every other slice is solved again from m = 0 with the full schedule, as
// the reference would, in a compact batch of the failed slices; slices do
// not interact in any kernel, so the redone slice equals icon_solve's cold
// result bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_internal.h"

namespace {

// Per slice (one block each) of a[S][n] and b[S][n]: out[s] = {sum (a-b)^2,
// sum b^2, count of non-finite a}, in double, summed in a fixed order.
__global__ void __launch_bounds__(256) k_warm_compare(const float *__restrict__ a, const float *__restrict__ b,
                                                      size_t n, double *__restrict__ out)
{
    __shared__ double red[3][256];
    const size_t s = blockIdx.x;
    const float *as = a + s * n, *bs = b + s * n;
    double dd = 0.0, bb = 0.0, bad = 0.0;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float x = as[i], y = bs[i];
        if (!isfinite(x)) {
            bad += 1.0;
            continue;
        }
        const double d = (double)x - (double)y;
        dd += d * d;
        bb += (double)y * (double)y;
    }
    red[0][threadIdx.x] = dd;
    red[1][threadIdx.x] = bb;
    red[2][threadIdx.x] = bad;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) out[s * 3 + k] = red[k][0];
}

struct DevMem {
    void *p = nullptr;
    ~DevMem()
    {
        if (p) cudaFree(p);
    }
};

#define WARM_CUDA(call)                                                                              \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return iconx::fail_msg(ICON_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define WARM_TRY(expr)                  \
    do {                                \
        icon_status s_ = (expr);        \
        if (s_ != ICON_OK) return s_;   \
    } while (0)

struct DeviceRestore {
    int prev = -1;
    explicit DeviceRestore(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceRestore()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" icon_status icon_solve_warm(icon_plan *p, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S,
                                       const icon_warm_cfg *wc, int *h_redone, int *h_iters, void *stream)
{
    if (!p || !cfg || !d_Ahwb || !d_m || !wc) return iconx::fail_msg(ICON_ERR_INVALID, "null argument");
    if (S < 1) return iconx::fail_msg(ICON_ERR_INVALID, "S must be >= 1");
    if (S > iconx::plan_capacity(p)) return iconx::fail_msg(ICON_ERR_CAPACITY, "S exceeds the plan's capacity");
    if (!(wc->tol > 0.0) || wc->check_every < 1 || !(wc->max_dist > 0.0))
        return iconx::fail_msg(ICON_ERR_INVALID, "icon_warm_cfg: tol > 0, check_every >= 1 and max_dist > 0 required");
    DeviceRestore guard(iconx::plan_device(p));
    cudaStream_t st = (cudaStream_t)stream;
    int dims[10];
    WARM_TRY(icon_plan_query(p, dims));
    const size_t NN = (size_t)dims[0] * dims[1];
    // The cold start's iterate after the first INFR phase, in the plan's
    // image buffer.
    float *m_infr = iconx::plan_out_buffer(p);
    icon_solve_cfg infr{cfg->infr_before, 0, 0, cfg->data_type, cfg->threshold};
    WARM_TRY(icon_solve(p, &infr, d_Ahwb, m_infr, S, 0, nullptr, nullptr, stream));
    // The warm solve, its ICON phase stopped at the tolerance.
    std::vector<double> step(S, 0.0);
    int iters = 0;
    WARM_TRY(icon_solve_until(p, cfg, d_Ahwb, d_m, S, 1, wc->tol, wc->check_every, &iters, step.data(), stream));
    if (h_iters) *h_iters = iters;
    DevMem stats;
    WARM_CUDA(cudaMalloc(&stats.p, sizeof(double) * 3 * S));
    k_warm_compare<<<S, 256, 0, st>>>(d_m, m_infr, NN, (double *)stats.p);
    WARM_CUDA(cudaGetLastError());
    std::vector<double> hs(3 * (size_t)S);
    WARM_CUDA(cudaMemcpyAsync(hs.data(), stats.p, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, st));
    WARM_CUDA(cudaStreamSynchronize(st));
    // With no ICON iterations in the schedule there is no step to judge.
    const bool judge_step = cfg->icon > 0;
    std::vector<int> why(S, ICON_WARM_ACCEPTED), redo;
    for (int s = 0; s < S; ++s) {
        const double dd = hs[3 * s], bb = hs[3 * s + 1], bad = hs[3 * s + 2];
        if (bad > 0.0 || !std::isfinite(dd)) why[s] = ICON_WARM_NOT_FINITE;
        else if (judge_step && !(step[s] <= wc->tol)) why[s] = ICON_WARM_NOT_CONVERGED;
        else if (!(std::sqrt(dd) <= wc->max_dist * std::sqrt(bb))) why[s] = ICON_WARM_TOO_FAR;
        if (why[s] != ICON_WARM_ACCEPTED) redo.push_back(s);
    }
    if (!redo.empty()) {
        // The failed slices' right-hand sides side by side, solved cold with
        // the full schedule into the plan's image buffer, then copied back.
        const int nf = (int)redo.size();
        DevMem ah;
        WARM_CUDA(cudaMalloc(&ah.p, sizeof(float) * 2 * NN * nf));
        for (int k = 0; k < nf; ++k)
            WARM_CUDA(cudaMemcpyAsync((float *)ah.p + 2 * NN * k, (const float *)d_Ahwb + 2 * NN * redo[k],
                                      sizeof(float) * 2 * NN, cudaMemcpyDeviceToDevice, st));
        WARM_TRY(icon_solve(p, cfg, ah.p, m_infr, nf, 0, nullptr, nullptr, stream));
        for (int k = 0; k < nf; ++k)
            WARM_CUDA(cudaMemcpyAsync(d_m + NN * redo[k], m_infr + NN * k, sizeof(float) * NN,
                                      cudaMemcpyDeviceToDevice, st));
        WARM_CUDA(cudaStreamSynchronize(st));
    }
    if (h_redone)
        for (int s = 0; s < S; ++s) h_redone[s] = why[s];
    return ICON_OK;
}
