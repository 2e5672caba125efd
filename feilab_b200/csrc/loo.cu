// loo.cu -- leave-one-out cross validation over all tilts of a series.
//
// The reference cross-validates one tilt: Lib_2D_crossV2
// (MainCode_crossV.cu:3-189) reconstructs every slice from the tilt series
// without the tilt of smallest |angle| (its own nodes and weights for the
// remaining tilts, readSlicePart_crossV.cu:3-34), reprojects at the omitted
// angle (reProject_NFFT2, reProject_NFFT.cu:25-42) and compares with the
// omitted projection by FRC (calFRC_nonsqure + frcSmooth).  Here every tilt
// takes that role in turn: one plan per omitted tilt, the slices in batches
// of the plan's capacity, FRC per omitted tilt.  Optionally each solve ends
// its ICON phase at a relative-step tolerance (icon_solve_until).  Every
// solve starts from m = 0: a start that holds the omitted projection (such
// as the reconstruction from all tilts) would leak it into the validation,
// since the solve never sees that projection's data and cannot remove it.
// C ABI in include/icon_tools.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_tools.h"

extern "C" void icon_internal_set_error(const char *msg);

namespace {

icon_status loo_fail(icon_status st, const std::string &msg)
{
    icon_internal_set_error(msg.c_str());
    return st;
}

struct DevArr {
    void *p = nullptr;
    ~DevArr() { cudaFree(p); }
};

struct Plan {
    icon_plan *p = nullptr;
    ~Plan() { icon_plan_destroy(p); }
};

}  // namespace

extern "C" icon_status icon_loo_sweep(const float *h_rows, int nx, int thickness, int nz, const float *tilt_deg,
                                      const icon_solve_cfg *cfg, int S, int capacity, double tol, int device,
                                      float *h_frc, float *h_reproj, int *h_iters)
{
    if (!h_rows || !tilt_deg || !cfg || !h_frc || nx < 2 || thickness < 1 || nz < 3 || S < 1 || capacity < 1)
        return loo_fail(ICON_ERR_INVALID, "icon_loo_sweep: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: cudaSetDevice");
    const int cap = std::min(capacity, S);
    const size_t NN = (size_t)nx * thickness;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    DevArr rows, Ahwb, m, rp;
    if (cudaMalloc(&rows.p, sizeof(float) * (size_t)cap * nz * nx) != cudaSuccess ||
        cudaMalloc(&Ahwb.p, sizeof(float) * 2 * (size_t)cap * NN) != cudaSuccess ||
        cudaMalloc(&m.p, sizeof(float) * (size_t)cap * NN) != cudaSuccess ||
        cudaMalloc(&rp.p, sizeof(float) * (size_t)cap * nx) != cudaSuccess) {
        cudaGetLastError();
        return loo_fail(ICON_ERR_NOMEM, "icon_loo_sweep: device memory");
    }
    icon_status rc = ICON_OK;
    std::vector<float> t1(nz - 1), r1((size_t)cap * (nz - 1) * nx), gt((size_t)S * nx), rps((size_t)S * nx);
    for (int omit = 0; omit < nz; ++omit) {
        for (int k = 0, q = 0; k < nz; ++k)
            if (k != omit) t1[q++] = tilt_deg[k];
        icon_geometry g{nx, thickness, nz - 1, t1.data(), cap, device};
        Plan P;
        if ((rc = icon_plan_create(&g, &P.p)) != ICON_OK) return rc;
        int iters_max = 0;
        for (int s0 = 0; s0 < S; s0 += cap) {
            const int nb = std::min(cap, S - s0);
            // rows of the batch without the omitted tilt (readSlicePart_crossV.cu:13-22)
            for (int s = 0; s < nb; ++s)
                for (int k = 0, q = 0; k < nz; ++k) {
                    const float *src = h_rows + ((size_t)(s0 + s) * nz + k) * nx;
                    if (k == omit) std::memcpy(&gt[(size_t)(s0 + s) * nx], src, sizeof(float) * nx);
                    else std::memcpy(&r1[((size_t)s * (nz - 1) + q++) * nx], src, sizeof(float) * nx);
                }
            cudaMemcpyAsync(rows.p, r1.data(), sizeof(float) * (size_t)nb * (nz - 1) * nx, cudaMemcpyHostToDevice, st);
            if ((rc = icon_prepare_rhs(P.p, (const float *)rows.p, Ahwb.p, nb, st)) != ICON_OK) return rc;
            int it = 0;
            rc = icon_solve_until(P.p, cfg, Ahwb.p, (float *)m.p, nb, 0, tol, 10, &it, nullptr, st);
            if (rc != ICON_OK) return rc;
            iters_max = std::max(iters_max, it);
            if ((rc = icon_reproject(P.p, (const float *)m.p, tilt_deg[omit], (float *)rp.p, nb, st)) != ICON_OK) return rc;
            cudaMemcpyAsync(&rps[(size_t)s0 * nx], rp.p, sizeof(float) * (size_t)nb * nx, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: stream error");
        }
        if (h_reproj) std::memcpy(h_reproj + (size_t)omit * S * nx, rps.data(), sizeof(float) * (size_t)S * nx);
        if (h_iters) h_iters[omit] = iters_max;
        // FRC of the reprojection against the omitted projection (ICONGPU.cu:560-586)
        if ((rc = icon_frc(gt.data(), rps.data(), nx, S, 10, h_frc + (size_t)omit * (nx / 2))) != ICON_OK) return rc;
    }
    return ICON_OK;
}
