// loo.cu -- leave-one-out cross validation over all tilts of a series.
//
// The reference cross-validates one tilt: Lib_2D_crossV2
// (MainCode_crossV.cu:3-189) reconstructs every slice from the tilt series
// without the tilt of smallest |angle| (its own nodes and weights for the
// remaining tilts, readSlicePart_crossV.cu:3-34), reprojects at the omitted
// angle (reProject_NFFT2, reProject_NFFT.cu:25-42) and compares with the
// omitted projection by FRC (calFRC_nonsqure + frcSmooth).  Here every tilt
// takes that role in turn, and all the left-out solves run as one batched
// schedule on one plan over all tilts: a work item is (omitted tilt k, B
// consecutive slices), one slice group; a batch is as many items as the
// capacity holds, each group with its own weights (icon_plan_set_group_weights):
// tilt k's nodes at 0 and the other tilts weighted as Weight() weights the
// series without k.  Weight 0 removes a node from every sum of the data
// term, so a group solves exactly the reduced series (up to the order in
// which the step length's double partial sums are combined), with no plan
// rebuilt per tilt and full batches however few slices there are.  Each
// group is reprojected at its omitted angle, and the FRC per omitted tilt
// compares those with the omitted projection.  Optionally each batch ends
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

// Makes `dev` current for the sweep and gives the calling thread its previous
// device back on every return path.
struct CurrentDevice {
    int prev = -1;
    bool ok = false;
    explicit CurrentDevice(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~CurrentDevice()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" icon_status icon_loo_sweep(const float *h_rows, int nx, int thickness, int nz, const float *tilt_deg,
                                      const icon_solve_cfg *cfg, int S, int capacity, double tol, int device,
                                      float *h_frc, float *h_reproj, int *h_iters, int op)
{
    if (!h_rows || !tilt_deg || !cfg || !h_frc || nx < 2 || thickness < 1 || nz < 3 || S < 1 || capacity < 1)
        return loo_fail(ICON_ERR_INVALID, "icon_loo_sweep: bad argument");
    CurrentDevice cur(device);
    if (!cur.ok) return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: cudaSetDevice");
    icon_status rc = ICON_OK;
    // One plan over all tilts; its capacity bounds a batch.
    const int cap = capacity;
    icon_geometry g{nx, thickness, nz, tilt_deg, cap, device};
    Plan P;
    if ((rc = icon_plan_create(&g, &P.p)) != ICON_OK) return rc;
    if ((rc = icon_plan_set_operator(P.p, op)) != ICON_OK) return rc;
    int dims[10];
    if ((rc = icon_plan_query(P.p, dims)) != ICON_OK) return rc;
    const int M = dims[4], B = dims[6];
    const int per_item = std::min(B, cap);             // slices of one work item (one group)
    const int items_per_batch = std::max(1, cap / B);  // groups of a batch
    const size_t NN = (size_t)nx * thickness;
    // Weights of each left-out series, in the full plan's node order.
    std::vector<float> wk((size_t)nz * M), wred((size_t)(nz - 1) * nx), t1(nz - 1);
    for (int k = 0; k < nz; ++k) {
        for (int i = 0, q = 0; i < nz; ++i)
            if (i != k) t1[q++] = tilt_deg[i];
        if ((rc = icon_weights(nx, nz - 1, t1.data(), wred.data())) != ICON_OK) return rc;
        float *w = &wk[(size_t)k * M];
        for (int i = 0, q = 0; i < nz; ++i) {
            if (i == k) std::fill(w + (size_t)i * nx, w + (size_t)(i + 1) * nx, 0.f);
            else std::memcpy(w + (size_t)i * nx, &wred[(size_t)q++ * nx], sizeof(float) * nx);
        }
    }
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    const int slots = items_per_batch * B > cap ? per_item : items_per_batch * B;
    DevArr rows, Ahwb, m, rp;
    if (cudaMalloc(&rows.p, sizeof(float) * (size_t)slots * nz * nx) != cudaSuccess ||
        cudaMalloc(&Ahwb.p, sizeof(float) * 2 * (size_t)slots * NN) != cudaSuccess ||
        cudaMalloc(&m.p, sizeof(float) * (size_t)slots * NN) != cudaSuccess ||
        cudaMalloc(&rp.p, sizeof(float) * (size_t)slots * nx) != cudaSuccess) {
        cudaGetLastError();
        return loo_fail(ICON_ERR_NOMEM, "icon_loo_sweep: device memory");
    }
    // Work items in tilt-major order.
    struct Item {
        int k, s0, n;
    };
    std::vector<Item> items;
    for (int k = 0; k < nz; ++k)
        for (int s0 = 0; s0 < S; s0 += per_item) items.push_back({k, s0, std::min(per_item, S - s0)});
    std::vector<float> hrows((size_t)slots * nz * nx), hw((size_t)items_per_batch * M), hrp((size_t)slots * nx);
    std::vector<float> rps((size_t)nz * S * nx);
    std::vector<int> iters(nz, 0);
    for (size_t i0 = 0; i0 < items.size(); i0 += items_per_batch) {
        const int ni = (int)std::min<size_t>(items_per_batch, items.size() - i0);
        const int Sb = (ni - 1) * B + items[i0 + ni - 1].n;   // slots up to the last item's last slice
        std::fill(hrows.begin(), hrows.end(), 0.f);          // padding slots solve zero data
        for (int q = 0; q < ni; ++q) {
            const Item &it = items[i0 + q];
            std::memcpy(&hrows[(size_t)q * B * nz * nx], h_rows + (size_t)it.s0 * nz * nx, sizeof(float) * (size_t)it.n * nz * nx);
            std::memcpy(&hw[(size_t)q * M], &wk[(size_t)it.k * M], sizeof(float) * M);
        }
        if ((rc = icon_plan_set_group_weights(P.p, hw.data(), ni)) != ICON_OK) return rc;
        cudaMemcpyAsync(rows.p, hrows.data(), sizeof(float) * (size_t)Sb * nz * nx, cudaMemcpyHostToDevice, st);
        if ((rc = icon_prepare_rhs(P.p, (const float *)rows.p, Ahwb.p, Sb, st)) != ICON_OK) return rc;
        int done = 0;
        if ((rc = icon_solve_until(P.p, cfg, Ahwb.p, (float *)m.p, Sb, 0, tol, 10, &done, nullptr, st)) != ICON_OK) return rc;
        for (int q = 0; q < ni; ++q) {
            const Item &it = items[i0 + q];
            iters[it.k] = std::max(iters[it.k], done);
            if ((rc = icon_reproject(P.p, (const float *)m.p + (size_t)q * B * NN, tilt_deg[it.k],
                                     (float *)rp.p + (size_t)q * B * nx, it.n, st)) != ICON_OK)
                return rc;
        }
        cudaMemcpyAsync(hrp.data(), rp.p, sizeof(float) * (size_t)Sb * nx, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return loo_fail(ICON_ERR_CUDA, "icon_loo_sweep: stream error");
        for (int q = 0; q < ni; ++q) {
            const Item &it = items[i0 + q];
            std::memcpy(&rps[((size_t)it.k * S + it.s0) * nx], &hrp[(size_t)q * B * nx], sizeof(float) * (size_t)it.n * nx);
        }
    }
    // FRC of each omitted tilt's reprojections against its projection (ICONGPU.cu:560-586).
    std::vector<float> gt((size_t)S * nx);
    for (int k = 0; k < nz; ++k) {
        for (int s = 0; s < S; ++s)
            std::memcpy(&gt[(size_t)s * nx], h_rows + ((size_t)s * nz + k) * nx, sizeof(float) * nx);
        if ((rc = icon_frc(gt.data(), &rps[(size_t)k * S * nx], nx, S, 10, h_frc + (size_t)k * (nx / 2))) != ICON_OK)
            return rc;
        if (h_iters) h_iters[k] = iters[k];
    }
    if (h_reproj) std::memcpy(h_reproj, rps.data(), sizeof(float) * rps.size());
    return ICON_OK;
}
