// icon_api.cu -- plans, launch sequences and the C ABI of include/icon_b200.h.
//
// Host-side geometry follows the reference exactly (float arithmetic where it
// uses float); the window tables are evaluated on the device with the same
// float expressions as nufft_Phi2d_1dCU (NU:221-235), so they carry the same
// bits as the reference's tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_internal.h"
#include "icon_kernels.cuh"
#include "icon_launch.h"

using icon::Geo;
using icon::Geo1;
using icon::kTaps;

namespace {

thread_local std::string g_last_error;

icon_status fail(icon_status st, const std::string &msg)
{
    g_last_error = msg;
    return st;
}

#define ICON_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(ICON_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

#define ICON_TRY(expr)                           \
    do {                                         \
        icon_status s_ = (expr);                 \
        if (s_ != ICON_OK) return s_;            \
    } while (0)

constexpr double kRefPi = 3.1415926535898;      // nufft_gpu_v8.cuh:8
constexpr double kRefPiPx2d = 3.14159265;       // px2D.cuh:8

// MainCode.cu:66-71 and NU:471-476 (float where the reference stores float).
void grid_params(int N, float &th, int &n, float &b, float &bf)
{
    float uptop = (float)std::pow(2.0, std::ceil(std::log10((double)N) / std::log10(2.0)));
    th = (float)(2.0 * uptop / (double)N);
    n = (int)std::ceil(th * (float)N);
    b = (float)((double)(2 * th * icon::kHalf) / ((double)(2 * th - 1) * kRefPi));
    bf = (float)(1.0 / std::sqrt(kRefPi * (double)b));
}

// px2D.cu:8-47: s accumulated in float from -1/2 by 1/nx; x = s*cos, s*sin of
// angle*pi/180 in double, stored as float.  Output interleaved (x0, x1).
void px2d(int nx, int nz, const float *th_neg, float *xy)
{
    std::vector<float> s(nx);
    float step = (float)(1.0 / nx);
    s[0] = (float)(-1.0 / 2);
    for (int k = 1; k < nx; ++k) s[k] = s[k - 1] + step;
    for (int i = 0; i < nz; ++i) {
        double a = (double)th_neg[i] * kRefPiPx2d / 180;
        double c = std::cos(a), sn = std::sin(a);
        for (int k = 0; k < nx; ++k) {
            xy[2 * ((size_t)i * nx + k)] = (float)((double)s[k] * c);
            xy[2 * ((size_t)i * nx + k) + 1] = (float)((double)s[k] * sn);
        }
    }
}

// weight.cu:8-41.
void weights(int nx, int nz, const float *t, float *w)
{
    int center = nx / 2;
    for (int i = 0; i < nz; ++i)
        for (int j = 0; j < nx; ++j) {
            float v;
            if (j == center) v = (float)(180.0 / (4 * nz));
            else if (i == 0) v = (float)(2.0 * std::fabs((t[i + 1] - t[i]) * (float)(j - center)));
            else if (i == nz - 1) v = (float)(2.0 * std::fabs((t[i - 1] - t[i]) * (float)(j - center)));
            else v = (float)(1.0 * std::fabs((t[i - 1] - t[i + 1]) * (float)(j - center)));
            w[(size_t)i * nx + j] = v;
        }
}

// Modified Bessel function I0 by its power series sum_k ((x/2)^k / k!)^2
// (positive terms; converges to double precision well within 60 terms for
// the arguments of the Kaiser-Bessel window, x <= 4 * 2 pi).
double bessel_i0(double x)
{
    double term = 1.0, sum = 1.0, q = 0.25 * x * x;
    for (int k = 1; k < 60; ++k) {
        term *= q / ((double)k * (double)k);
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}

// Shape parameter of the Kaiser-Bessel window for oversampling theta:
// kb = pi (2 - 1/theta) (the choice of Potts, Steidl and Tasche's NFFT).
double kb_shape(float theta) { return M_PI * (2.0 - 1.0 / (double)theta); }

// Deapodisation factors (NU:22-42): exp(-b (pi k/n)^2) in double, stored as
// float.  Kaiser-Bessel (kb > 0): the window's Fourier transform
// I0(K sqrt(kb^2 - (2 pi k/n)^2)) / I0(kb K), real for theta >= 1.
std::vector<float> deapod(int N, int n, float b, double kb = 0.0)
{
    std::vector<float> c(N);
    const double i0m = kb > 0.0 ? bessel_i0(kb * icon::kKbHalf) : 1.0;
    for (int X = 0; X < N; ++X) {
        int k = X - N / 2;
        if (kb > 0.0) {
            double w = 2.0 * M_PI * k / (double)n;
            c[X] = (float)(bessel_i0(icon::kKbHalf * std::sqrt(kb * kb - w * w)) / i0m);
        } else {
            c[X] = (float)std::exp(-(double)b * ((kRefPi * k / (double)n) * (kRefPi * k / (double)n)));
        }
    }
    return c;
}

// 1 / (pi I0(kb K)): the Kaiser-Bessel window's scale (0 for the Gaussian).
double kb_inv(double kb) { return kb > 0.0 ? 1.0 / (M_PI * bessel_i0(kb * icon::kKbHalf)) : 0.0; }

std::vector<float2> twiddles(int n)
{
    std::vector<float2> t(n);
    for (int q = 0; q < n; ++q) {
        double a = 2.0 * M_PI * (double)q / (double)n;
        t[q] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    return t;
}

int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

// Owned device allocations of a plan.
struct Arena {
    std::vector<std::unique_ptr<DevBuf>> bufs;
    size_t total = 0;
    template <typename T>
    icon_status alloc(T **out, size_t count)
    {
        auto b = std::make_unique<DevBuf>();
        size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        cudaError_t e = cudaMalloc(&b->p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(ICON_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        }
        b->bytes = bytes;
        total += bytes;
        *out = (T *)b->p;
        bufs.push_back(std::move(b));
        return ICON_OK;
    }
    // Releases one buffer of this arena (reallocation of a grown table).
    void release(void *ptr)
    {
        for (auto it = bufs.begin(); it != bufs.end(); ++it)
            if ((*it)->p == ptr) {
                total -= (*it)->bytes;
                bufs.erase(it);
                return;
            }
    }
    template <typename T>
    icon_status upload(T **out, const T *host, size_t count)
    {
        ICON_TRY(alloc(out, count));
        ICON_CUDA(cudaMemcpy(*out, host, count * sizeof(T), cudaMemcpyHostToDevice));
        return ICON_OK;
    }
};

// Node tables of one geometry (a tilt series or a single reprojection line).
struct NodeTables {
    int M = 0;
    int taps = 0;    // x taps with entries per node (14, or 8 for Kaiser-Bessel)
    float *phix = nullptr, *phiy = nullptr, *w = nullptr;
    int *ix0 = nullptr, *iy0 = nullptr, *row_off = nullptr, *ent_jt = nullptr, *ent_iy0 = nullptr;
    unsigned short *ent_lb = nullptr;
    float *ent_phiy = nullptr, *ent_pxy = nullptr;
};

}  // namespace

struct icon_plan {
    int dev = 0;
    int nx = 0, N0 = 0, N1 = 0, nz = 0, M = 0, n0 = 0, n1 = 0, lg0 = 0, lg1 = 0;
    int window = ICON_WINDOW_GAUSS6;
    int tlo = 0, thi = icon::kTaps - 1;     // taps of the window that can be non-zero
    double kb0 = 0.0, kb1 = 0.0;            // Kaiser-Bessel shape per dimension (0: Gaussian)
    int B = 1, cap = 0, Gcap = 0;
    float th0 = 0, th1 = 0, b0 = 0, bf0 = 0, b1 = 0, bf1 = 0;
    std::vector<float> tlt, th_neg, xy, w;
    int omit_index = 0;
    float reproj_deg = 0.f;   // angle of icon_reconstruct_host's reprojection
    Arena arena;
    NodeTables nodes;
    float *cx = nullptr, *cy = nullptr, *rcx = nullptr, *rcy = nullptr, *phi1 = nullptr;
    int *i10 = nullptr;
    float2 *tw0 = nullptr, *tw0h = nullptr, *tw1 = nullptr;
    // Length of the Toeplitz y-transforms: the smallest 32 R >= 2 N1 - 1 that
    // k_ytoep4 takes (at most n1), else n1; tw1t its twiddles.
    int n1t = 0;
    float2 *tw1t = nullptr;
    // scratch sized for Gcap groups
    float2 *G1 = nullptr, *P = nullptr, *f = nullptr, *rhat = nullptr, *Ahwb = nullptr, *imgc = nullptr;
    float *m = nullptr, *rows = nullptr, *outrp = nullptr, *mout = nullptr;
    float *nodes_xy = nullptr;   // [M][2] node coordinates on the device (Toeplitz kernel)
    double *part_rtr = nullptr, *part_rtar = nullptr, *alpha = nullptr;
    double *step_part = nullptr, *step = nullptr;   // relative update size (icon_solve_until)
    float *wgroup = nullptr;   // [Gcap][M] per-group weights while wgroups > 0
    int wgroups = 0;
    // Distinct weight sets among the groups (Toeplitz kernels are computed
    // once per set): wuniq [kt_unique][M], kidx [Gcap] the set of each group.
    float *wuniq = nullptr;
    int *kidx = nullptr;
    int kt_unique = 0;
    // Normal operator of the iterations: ICON_OPERATOR_NUFFT (the reference's
    // NUFFT pair) or ICON_OPERATOR_TOEPLITZ (A^H W A as a convolution with Kt).
    int op = ICON_OPERATOR_NUFFT;
    // Tolerance stop of the reconstruct calls (icon_plan_set_stop): 0 = the
    // full schedule.
    double stop_tol = 0.0;
    int stop_every = 10;
    float *Kt = nullptr;        // [Gcap][n0][n1] Toeplitz kernels (one used unless per-group weights)
    int kt_groups = 0;          // kernels computed: 1, or one per distinct weight set of the groups
    int kt_cap = 0;             // kernels the Kt table has room for
    bool kt_stale = true;
    float *ones0 = nullptr, *ones1 = nullptr;   // unit deapodisation of the Toeplitz x-passes
    size_t smem_yt = 0;
    int na_rtar = 0;            // partial sums per group of the step length's denominator
    // Toeplitz iterations with the three-step x-kernels (k_xtoep) defer each
    // iteration's update m -= alpha Re r-hat into the next iteration's forward
    // x-pass; flush_update applies a pending one where the loop ends.
    bool xt_ok = false;         // k_xtoep has a variant for n0
    // TMA staging of the x-kernels' columns: tensor maps over G1, Ahwb, r-hat
    // and m (xt_tma), boxes of xt_bh slices; device error flag of their
    // bounded waits.
    // Warm start of the reconstruct calls (icon_plan_set_warm_start): the
    // network, the acceptance test, caller-layout buffers of A^H W b and m,
    // and counts of the slices accepted and redone from zero.
    icon_ws *ws = nullptr;
    icon_warm_cfg wcfg{};
    float2 *ws_A = nullptr;
    float *ws_m = nullptr;
    long long warm_accepted = 0, warm_redone = 0;
    bool xt_tma = false, xt_tma_m = false;
    int xt_bh = 1, xt_box_g1 = 0, xt_box_img = 0;
    CUtensorMap tm_g1, tm_ahwb, tm_rre, tm_m;
    float *rre = nullptr;       // [Gcap][N1][N0][B] Re r-hat of the Toeplitz x-kernels (the deferred update's input)
    int *dev_err = nullptr;
    bool upd_pending = false, upd_clamp = false;
    int upd_dtype = 0, upd_G = 0;
    float upd_thr = 0.f;
    int k3_blocks = 0;
    // reprojection lines, keyed by the .tlt angle
    std::map<float, std::unique_ptr<NodeTables>> lines;
    float2 *fline = nullptr;
    size_t smem_x = 0, smem_y = 0, smem_ya = 0;
    int thr_x = 0, thr_y = 0, ex = 16, ey = 16;   // threads and values per thread of x- and y-pass FFTs
    // tracing: events around every launch while enabled
    bool trace = false;
    long long launches = 0;
    struct Pending {
        int kind;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t ev_get()
    {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    ~icon_plan()
    {
        for (auto &q : pending) {
            cudaEventDestroy(q.a);
            cudaEventDestroy(q.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }

    Geo geo(const NodeTables &t) const
    {
        Geo g;
        g.N0 = N0; g.N1 = N1; g.n0 = n0; g.n1 = n1; g.lg0 = lg0; g.lg1 = lg1;
        g.M = t.M; g.nx = nx; g.nz = nz; g.B = B;
        g.tlo = tlo; g.thi = thi;
        g.w = t.w; g.wstride = 0;
        if (&t == &nodes && wgroups > 0) {   // icon_plan_set_group_weights
            g.w = wgroup;
            g.wstride = (size_t)M;
        }
        g.phix = t.phix; g.phiy = t.phiy; g.ix0 = t.ix0; g.iy0 = t.iy0;
        g.cx = cx; g.cy = cy; g.rcx = rcx; g.rcy = rcy; g.row_off = t.row_off; g.ent_jt = t.ent_jt; g.ent_iy0 = t.ent_iy0;
        g.ent_lb = t.ent_lb; g.ent_phiy = t.ent_phiy; g.ent_pxy = t.ent_pxy;
        g.tw0 = tw0; g.tw0h = tw0h; g.tw1 = tw1;
        g.Kt = Kt;
        g.kstride = kt_groups > 1 ? (size_t)n0 * n1t : 0;
        g.kidx = kt_groups > 1 ? kidx : nullptr;
        return g;
    }
    // The Toeplitz iteration's view: the plan's nodes with unit deapodisation
    // (its x-passes only pad and crop).
    Geo geo_unit() const
    {
        Geo g = geo(nodes);
        g.rcx = ones0;
        g.rcy = ones1;
        g.n1 = n1t;          // the y-transforms of the convolution
        g.tw1 = tw1t;
        return g;
    }
    // The TMA part of the x-kernels' arguments.
    void fill_xt(icon::XtArgs &xa) const
    {
        xa.use_tma = xt_tma ? 1 : 0;
        xa.tma_m = xt_tma_m ? 1 : 0;
        xa.box_g1 = xt_box_g1;
        xa.box_img = xt_box_img;
        xa.err = dev_err;
        if (xt_tma) {
            xa.tm_g1 = tm_g1;
            xa.tm_ahwb = tm_ahwb;
            xa.tm_rre = tm_rre;
            xa.tm_m = tm_m;
        }
    }
    Geo1 geo1() const
    {
        Geo1 g;
        g.phi1 = phi1;
        g.i10 = i10;
        return g;
    }
};

namespace {

enum Kind { K_XF = 0, K_YF, K_FIN, K_YA, K_XA, K_ALPHA, K_UPD, K_ROWS, K_LAYOUT, K_ROWADJ, K_YT, K_YQ, K_XTF, K_XTM };

// Launches one kernel; counts it and, while tracing, brackets it by events
// and records its algorithmic bytes (compulsory reads + writes, see
// algo_bytes below).
#define LAUNCH_B(p, kind, st, bytes, ...)                                 \
    do {                                                                  \
        cudaEvent_t e0_ = nullptr;                                        \
        if ((p)->trace) {                                                 \
            e0_ = (p)->ev_get();                                          \
            cudaEventRecord(e0_, st);                                     \
        }                                                                 \
        __VA_ARGS__;                                                      \
        (p)->launches++;                                                  \
        if ((p)->trace) {                                                 \
            cudaEvent_t e1_ = (p)->ev_get();                              \
            cudaEventRecord(e1_, st);                                     \
            (p)->pending.push_back({kind, e0_, e1_, (double)(bytes)});    \
        }                                                                 \
    } while (0)
#define LAUNCH(p, kind, st, ...) LAUNCH_B(p, kind, st, 0.0, __VA_ARGS__)

// Runs the statement with L = the launcher class of the plan's B.
#define WITH_B(Bv, ...)                                                  \
    switch (Bv) {                                                        \
    case 1: { using L = icon::Launch<1>; __VA_ARGS__; } break;           \
    case 2: { using L = icon::Launch<2>; __VA_ARGS__; } break;           \
    case 4: { using L = icon::Launch<4>; __VA_ARGS__; } break;           \
    default: { using L = icon::Launch<8>; __VA_ARGS__; } break;          \
    }


struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled()
{
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    });
    return fn;
}

// A FP32 tensor map of rank dims (innermost first), strides in bytes of
// dims 1.., box extents; no swizzle, no interleave, zero fill outside.
bool make_map(CUtensorMap *m, void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
              const cuuint32_t *box)
{
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, base, dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps for the x-kernels' TMA staging (k_xtoep): possible when a CTA
// takes at least 2 slices (boxes of 16 bytes or more, every coordinate and
// stride a multiple of 16 bytes); m needs 4.  ICON_XT_TMA=0 keeps the
// per-thread cp.async staging.
void setup_xt_tma(icon_plan *p)
{
    const int n0 = p->n0, B = p->B;
    p->xt_bh = n0 <= 1024 ? B : n0 == 2048 ? std::min(B, 4) : n0 == 4096 ? std::min(B, 2) : 1;
    const char *env = std::getenv("ICON_XT_TMA");
    if (!p->xt_ok || p->xt_bh < 2 || (env && env[0] == '0')) return;
    const int BH = p->xt_bh;
    p->xt_box_g1 = std::min(256, n0);
    p->xt_box_img = std::min(256, n0 / 2);
    const cuuint64_t G = (cuuint64_t)p->Gcap, N0 = (cuuint64_t)p->N0, N1 = (cuuint64_t)p->N1, Bz = (cuuint64_t)B;
    bool ok = true;
    {   // G1 [Gcap n0][N1 B 2] floats
        const cuuint64_t dims[2] = {N1 * Bz * 2, G * (cuuint64_t)n0};
        const cuuint64_t str[1] = {N1 * Bz * 8};
        const cuuint32_t box[2] = {(cuuint32_t)(BH * 2), (cuuint32_t)p->xt_box_g1};
        ok = ok && make_map(&p->tm_g1, p->G1, 2, dims, str, box);
    }
    {   // Ahwb and r-hat [Gcap N1][N0][B 2] floats
        const cuuint64_t dims[3] = {Bz * 2, N0, G * N1};
        const cuuint64_t str[2] = {Bz * 8, N0 * Bz * 8};
        const cuuint32_t box[3] = {(cuuint32_t)(BH * 2), (cuuint32_t)p->xt_box_img, 1};
        ok = ok && make_map(&p->tm_ahwb, p->Ahwb, 3, dims, str, box);

    }
    bool ok_m = BH >= 4;
    if (ok_m) {   // m [Gcap N1][N0][B] floats
        const cuuint64_t dims[3] = {Bz, N0, G * N1};
        const cuuint64_t str[2] = {Bz * 4, N0 * Bz * 4};
        const cuuint32_t box[3] = {(cuuint32_t)BH, (cuuint32_t)p->xt_box_img, 1};
        ok_m = make_map(&p->tm_m, p->m, 3, dims, str, box) && make_map(&p->tm_rre, p->rre, 3, dims, str, box);
    }
    p->xt_tma = ok;
    p->xt_tma_m = ok && ok_m;
}

// Builds window tables and the per-row entry lists of M nodes at xy.
icon_status build_tables(icon_plan *p, const float *xy, const float *w, int M, NodeTables &t)
{
    t.M = M;
    float *xy_d = nullptr;
    ICON_TRY(p->arena.upload(&xy_d, xy, (size_t)2 * M));
    ICON_TRY(p->arena.alloc(&t.phix, (size_t)M * kTaps));
    ICON_TRY(p->arena.alloc(&t.phiy, (size_t)M * icon::kLdPhiy));
    ICON_TRY(p->arena.alloc(&t.ix0, (size_t)M));
    ICON_TRY(p->arena.alloc(&t.iy0, (size_t)M));
    int blk = 256, grd = (M + blk - 1) / blk;
    icon::k_window<<<grd, blk>>>(xy_d, 2, M, p->n0, p->b0, p->bf0, t.phix, kTaps, t.ix0, p->kb0, kb_inv(p->kb0));
    icon::k_window<<<grd, blk>>>(xy_d + 1, 2, M, p->n1, p->b1, p->bf1, t.phiy, icon::kLdPhiy, t.iy0, p->kb1,
                                 kb_inv(p->kb1));
    ICON_CUDA(cudaGetLastError());
    std::vector<int> ix0(M), iy0(M);
    ICON_CUDA(cudaMemcpy(ix0.data(), t.ix0, sizeof(int) * M, cudaMemcpyDeviceToHost));
    ICON_CUDA(cudaMemcpy(iy0.data(), t.iy0, sizeof(int) * M, cudaMemcpyDeviceToHost));
    // Entries (node j, x tap t0) grouped by grid row x = (ix0 + t0) mod n0,
    // sorted within a row by (iy0, j); only the taps tlo..thi the window can
    // make non-zero get entries.
    const int n0 = p->n0, tlo = p->tlo, thi = p->thi;
    t.taps = thi - tlo + 1;
    std::vector<int> cnt(n0 + 1, 0);
    for (int j = 0; j < M; ++j)
        for (int t0 = tlo; t0 <= thi; ++t0) cnt[((ix0[j] + t0) % n0 + n0) % n0 + 1]++;
    for (int x = 0; x < n0; ++x) cnt[x + 1] += cnt[x];
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    size_t E = (size_t)M * t.taps;
    std::vector<int> jt(E), ky(E);
    for (int j = 0; j < M; ++j)
        for (int t0 = tlo; t0 <= thi; ++t0) {
            int x = ((ix0[j] + t0) % n0 + n0) % n0;
            int e = pos[x]++;
            jt[e] = j * 16 + t0;
            ky[e] = iy0[j];
        }
    std::vector<int> order;
    std::vector<int> jt2(E), ky2(E);
    for (int x = 0; x < n0; ++x) {
        int a = cnt[x], c = cnt[x + 1];
        order.resize(c - a);
        for (int i = 0; i < c - a; ++i) order[i] = a + i;
        std::stable_sort(order.begin(), order.end(), [&](int u, int v) {
            return ky[u] != ky[v] ? ky[u] < ky[v] : jt[u] < jt[v];
        });
        for (int i = 0; i < c - a; ++i) {
            jt2[a + i] = jt[order[i]];
            ky2[a + i] = ky[order[i]];
        }
    }
    // Per row, the entries whose first rotated y tap r0 = iy0 + n1/2 + 8 is
    // below v (v = 0..n1+16), relative to the row's first entry.
    const int ldl = icon::lb_ld(p->n1), r0ofs = p->n1 / 2 + icon::kHalo;
    std::vector<unsigned short> lb((size_t)n0 * ldl);
    for (int x = 0; x < n0; ++x) {
        int a = cnt[x], c = cnt[x + 1];
        if (c - a > 65535) return fail(ICON_ERR_INVALID, "more than 65535 window entries on one grid row");
        int e = a;
        for (int v = 0; v < ldl; ++v) {
            while (e < c && ky2[e] + r0ofs < v) ++e;
            lb[(size_t)x * ldl + v] = (unsigned short)(e - a);
        }
        if (c > a && (ky2[a] + r0ofs < 0 || ky2[c - 1] + r0ofs + kTaps > p->n1 + 2 * icon::kHalo))
            return fail(ICON_ERR_INVALID, "window taps outside the rotated y buffer");
        // The mirrored windows of the real-image forward y-pass: buffer rows
        // n1/2 - iy0 + kHalo - 13 .. n1/2 - iy0 + kHalo.
        if (c > a && (p->n1 / 2 - ky2[c - 1] + icon::kHalo - (kTaps - 1) < 0 ||
                      p->n1 / 2 - ky2[a] + icon::kHalo > p->n1 + 2 * icon::kHalo - 1))
            return fail(ICON_ERR_INVALID, "mirrored window taps outside the rotated y buffer");
    }
    ICON_TRY(p->arena.upload(&t.row_off, cnt.data(), (size_t)n0 + 1));
    ICON_TRY(p->arena.upload(&t.ent_jt, jt2.data(), E));
    ICON_TRY(p->arena.upload(&t.ent_iy0, ky2.data(), E));
    ICON_TRY(p->arena.upload(&t.ent_lb, lb.data(), lb.size()));
    ICON_TRY(p->arena.alloc(&t.ent_phiy, E * icon::kLdPhiy));
    ICON_TRY(p->arena.alloc(&t.ent_pxy, E * icon::kLdPhiy));
    icon::k_entry_tables<<<(unsigned)((E + 255) / 256), 256>>>(t.ent_jt, (int)E, t.phiy, t.phix, t.ent_phiy, t.ent_pxy);
    ICON_CUDA(cudaGetLastError());
    ICON_TRY(p->arena.upload(&t.w, w, (size_t)M));
    return ICON_OK;
}

icon_status check_plan(const icon_plan *p, int S)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (S < 1) return fail(ICON_ERR_INVALID, "S must be >= 1");
    if (S > p->cap) return fail(ICON_ERR_CAPACITY, "S = " + std::to_string(S) + " exceeds plan capacity " + std::to_string(p->cap));
    return ICON_OK;
}

inline int groups(const icon_plan *p, int S) { return (S + p->B - 1) / p->B; }

inline int grid1d(size_t total)
{
    size_t b = (total + 255) / 256;
    return (int)std::min<size_t>(std::max<size_t>(b, 1), 148 * 16);
}

// ------------------------------------------------------------- stages ----
// Algorithmic bytes per slot (one slice of a group) of each stage: the data a
// stage must read and write at least once; per-group tables are divided by B.
struct StageBytes {
    double xf_real, xf_cplx, yf, yf_real, fin_store, fin_red, ya, xa_plain, xa_resid, upd;
};
StageBytes stage_bytes(const icon_plan *p, const NodeTables &t)
{
    StageBytes b;
    double NN = (double)p->N0 * p->N1, G1 = (double)p->n0 * p->N1 * 8, MT = (double)t.M * t.taps, B = p->B;
    const double G1h = (double)(p->n0 / 2 + 1) * p->N1 * 8;   // rows 0..n0/2 (real image)
    b.xf_real = NN * 4 + G1h;
    b.xf_cplx = NN * 8 + G1;
    b.yf = G1 + MT * 8 + (MT * 8 + MT * 4) / B;            // G1 row reads, P writes; entries + phiy
    b.yf_real = G1h + MT * 8 + (MT * 8 + MT * 4) / B;
    b.fin_store = MT * 8 + (double)t.M * 8 + (MT * 4 + t.M * 4) / B;
    b.fin_red = MT * 8 + (MT * 4 + t.M * 4) / B;
    b.ya = (double)t.M * 8 + G1 + (MT * 8 + MT * 8) / B;   // f, G1 writes; entries + phix/phiy
    b.xa_plain = G1 + NN * 8;
    b.xa_resid = G1 + NN * 16;
    b.upd = NN * 16;
    return b;
}

icon_status launch_forward(icon_plan *p, const NodeTables &t, const void *img_int, bool real_in, int G, int mode,
                           float2 *f_out, cudaStream_t st)
{
    Geo g = p->geo(t);
    const StageBytes sb = stage_bytes(p, t);
    const double slots = (double)G * p->B;
    // A real image's spectrum is Hermitian: the y-pass takes grid rows
    // 0..n0/2 and interpolates the mirror rows' entries from them.
    dim3 gx(p->N1, G), gy(G, real_in ? p->n0 / 2 + 1 : p->n0);
    WITH_B(p->B,
        LAUNCH_B(p, K_XF, st, (real_in ? sb.xf_real : sb.xf_cplx) * slots,
                 L::xpass_fwd(real_in, p->ex, gx, p->thr_x, p->smem_x, st, g, img_int, p->G1));
        LAUNCH_B(p, K_YF, st, (real_in ? sb.yf_real : sb.yf) * slots,
                 L::ypass_fwd(p->ey, real_in, gy, p->thr_y, p->smem_y, st, g, p->G1, p->P)))
    int kb = (t.M * p->B + 255) / 256;
    dim3 g3(kb, G);
    WITH_B(p->B,
        LAUNCH_B(p, K_FIN, st, (mode == 2 ? sb.fin_red : sb.fin_store) * slots,
                 L::interp_fin(mode, g3, st, g, p->P, mode == 2 ? nullptr : f_out, mode == 2 ? p->part_rtar : nullptr)))
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status launch_adjoint(icon_plan *p, const float2 *f_int, int G, int mode, float2 *out_int, cudaStream_t st)
{
    Geo g = p->geo(p->nodes);
    const StageBytes sb = stage_bytes(p, p->nodes);
    const double slots = (double)G * p->B;
    dim3 gy(G, p->n0), gx(p->N1, G);
    size_t smem = p->smem_x + sizeof(double) * p->thr_x;
    icon::XtArgs xa{};
    p->fill_xt(xa);
    xa.N0 = p->N0; xa.N1 = p->N1; xa.n0 = p->n0; xa.tw0 = p->tw0; xa.G1 = p->G1; xa.rhat = out_int;
    xa.Ahwb = p->Ahwb; xa.part_rtr = p->part_rtr; xa.rcx = p->rcx; xa.rcy = p->rcy; xa.resid = mode == 0 ? 0 : 1;
    WITH_B(p->B,
        LAUNCH_B(p, K_YA, st, sb.ya * slots, L::ypass_adj(p->ey, gy, p->thr_y, p->smem_ya, st, g, f_int, p->G1));
        if (p->xt_ok) {
            LAUNCH_B(p, K_XA, st, (mode == 0 ? sb.xa_plain : sb.xa_resid) * slots, L::xtoep(2, st, G, xa));
        } else {
            LAUNCH_B(p, K_XA, st, (mode == 0 ? sb.xa_plain : sb.xa_resid) * slots,
                     L::xpass_adj(mode, p->ex, gx, p->thr_x, smem, st, g, p->G1, out_int, mode == 0 ? nullptr : p->Ahwb,
                                  mode == 0 ? nullptr : p->part_rtr));
        })
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// Row transform of S slices; the row of slice sl for tilt i starts at
// d_rows + sl*sstride + sec*istride, sec = i, or i + 1 from tilt `skip` on.
icon_status launch_rows_at(icon_plan *p, const float *d_rows, size_t sstride, size_t istride, int skip, int S, int G,
                           float2 *bout, cudaStream_t st)
{
    Geo g = p->geo(p->nodes);
    WITH_B(p->B, LAUNCH(p, K_ROWS, st, L::rows_fwd(p->ex, dim3(p->nz, G), p->thr_x, p->smem_x, st, g, p->geo1(), d_rows,
                                                   sstride, istride, skip, S, p->f, bout)))
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// Rows in the caller layout [S][nz][nx].
icon_status launch_rows(icon_plan *p, const float *d_rows, int S, int G, float2 *bout, cudaStream_t st)
{
    return launch_rows_at(p, d_rows, (size_t)p->nz * p->nx, (size_t)p->nx, INT_MAX, S, G, bout, st);
}

icon_status launch_iteration_toep(icon_plan *p, int G, bool clamp, int data_type, float thr, double *hist_a,
                                  double *hist_r, cudaStream_t st, bool measure_step);

// One ICON iteration over G groups (Iteration2.cu:53-132 with Alpha2).
icon_status launch_iteration(icon_plan *p, int G, bool clamp, int data_type, float thr, double *hist_a, double *hist_r,
                             cudaStream_t st, bool measure_step = false)
{
    if (p->op == ICON_OPERATOR_TOEPLITZ)
        return launch_iteration_toep(p, G, clamp, data_type, thr, hist_a, hist_r, st, measure_step);
    ICON_TRY(launch_forward(p, p->nodes, p->m, true, G, 1, p->f, st));          // f = W A m
    ICON_TRY(launch_adjoint(p, p->f, G, 1, p->rhat, st));                       // rhat = A^H f - Ahwb, ||rhat||^2
    ICON_TRY(launch_forward(p, p->nodes, p->rhat, false, G, 2, nullptr, st));   // r = A rhat, sum w|r|^2
    int kb = (p->M * p->B + 255) / 256;
    LAUNCH(p, K_ALPHA, st, icon::k_alpha<<<G, 32 * p->B, 0, st>>>(p->part_rtr, p->N1, p->part_rtar, kb, p->B, p->alpha, hist_a, hist_r));
    int per_group = p->N1 * p->N0 * p->B;
    dim3 gu((unsigned)std::min<size_t>(((size_t)per_group + 255) / 256, 512), G);
    WITH_B(p->B, LAUNCH_B(p, K_UPD, st, stage_bytes(p, p->nodes).upd * G * p->B,
                          L::update(gu, st, p->m, p->rhat, p->alpha, per_group, clamp ? 1 : 0, data_type, thr,
                                    measure_step ? p->step_part : nullptr)))
    if (measure_step) {                                                          // ||m_new - m_old|| / ||m_new||
        const int slots = G * p->B;
        LAUNCH(p, K_UPD, st, icon::k_step_reduce<<<(slots + 127) / 128, 128, 0, st>>>(p->step_part, (int)gu.x, p->B, slots, p->step));
    }
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// The Toeplitz kernels of the plan's weights (one) or, with per-group
// weights, of every group's (icon_plan_set_group_weights), when stale.
icon_status ensure_toeplitz(icon_plan *p, cudaStream_t st)
{
    if (p->op != ICON_OPERATOR_TOEPLITZ || !p->kt_stale) return ICON_OK;
    const int groups_needed = p->wgroups > 0 ? p->kt_unique : 1;
    if (p->Kt && p->kt_cap < groups_needed) {   // one kernel per group needs a larger table
        p->arena.release(p->Kt);
        p->Kt = nullptr;
    }
    if (!p->Kt) {
        ICON_TRY(p->arena.alloc(&p->Kt, (size_t)groups_needed * p->n0 * p->n1t));
        p->kt_cap = groups_needed;
    }
    float *xy_d = nullptr;
    if (!p->nodes_xy) ICON_TRY(p->arena.upload(&p->nodes_xy, p->xy.data(), p->xy.size()));
    xy_d = p->nodes_xy;
    const float *w = p->wgroups > 0 ? p->wuniq : p->nodes.w;
    dim3 grid((p->n1t + icon::kToepTile - 1) / icon::kToepTile, (p->n0 + icon::kToepTile - 1) / icon::kToepTile,
              groups_needed);
    icon::k_toep_kernel<<<grid, 256, 0, st>>>(xy_d, w, p->wgroups > 0 ? (size_t)p->M : 0, p->M, p->N0, p->N1, p->n0,
                                              p->n1t, icon::ytoep4_fits(p->n1t) ? p->n1t / 32 : 0, p->Kt);
    ICON_CUDA(cudaGetLastError());
    p->kt_groups = groups_needed;
    p->kt_stale = false;
    return ICON_OK;
}

// Applies a deferred update (m -= alpha Re r-hat, clamped as recorded) of
// the last Toeplitz iteration, if one is pending.
icon_status flush_update(icon_plan *p, cudaStream_t st)
{
    if (!p->upd_pending) return ICON_OK;
    p->upd_pending = false;
    const int G = p->upd_G;
    int per_group = p->N1 * p->N0 * p->B;
    dim3 gu((unsigned)std::min<size_t>(((size_t)per_group + 255) / 256, 512), G);
    // m read and written, Re r-hat read
    WITH_B(p->B, LAUNCH_B(p, K_UPD, st, (double)p->N0 * p->N1 * 12 * G * p->B,
                          L::update_re(gu, st, p->m, p->rre, p->alpha, per_group, p->upd_clamp ? 1 : 0, p->upd_dtype,
                                       p->upd_thr)))
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// One Toeplitz iteration with the three-step x-kernels: the forward x-pass of
// m (applying the previous iteration's deferred update first), the Toeplitz
// y-pass, the fused inverse x-pass / r-hat / forward x-pass of r-hat, the
// quadratic form's y-pass and the step length.  This iteration's update is
// left pending (flush_update or the next iteration applies it).
// The kernels of one such iteration with the deferred update given
// explicitly: upd applies the previous iteration's update (clamped when
// clamp_prev) in the forward x-pass.  Changes no host-side state, so it can
// be captured into a CUDA graph and replayed.
icon_status launch_iteration_xt_raw(icon_plan *p, int G, bool upd, bool clamp_prev, int data_type, float thr,
                                    double *hist_a, double *hist_r, cudaStream_t st)
{
    Geo g = p->geo_unit();
    const double slots = (double)G * p->B;
    const double NN = (double)p->N0 * p->N1, G1b = (double)p->n0 * p->N1 * 8, Kb = (double)p->n0 * p->n1t * 4;
    icon::XtArgs xa{};
    p->fill_xt(xa);
    xa.N0 = p->N0; xa.N1 = p->N1; xa.n0 = p->n0; xa.tw0 = p->tw0; xa.G1 = p->G1; xa.m = p->m;
    xa.rre_in = p->rre; xa.alpha = p->alpha; xa.upd = upd ? 1 : 0; xa.clamp = clamp_prev ? 1 : 0;
    xa.data_type = data_type; xa.thr = thr; xa.rre = p->rre; xa.Ahwb = p->Ahwb; xa.part_rtr = p->part_rtr;
    const double xf_bytes = (xa.upd ? NN * 12 : NN * 4) + G1b;   // m (read, written), Re r-hat; G1 written
    dim3 gy(G, p->n0);
    WITH_B(p->B,
        LAUNCH_B(p, K_XTF, st, xf_bytes * slots, L::xtoep(0, st, G, xa));
        LAUNCH_B(p, K_YT, st, (2 * G1b) * slots + Kb * G, L::ypass_toep(p->ey, gy, p->thr_y, p->smem_yt, st, g, p->G1));
        LAUNCH_B(p, K_XTM, st, (2 * G1b + NN * 12) * slots, L::xtoep(1, st, G, xa));
        LAUNCH_B(p, K_YQ, st, G1b * slots + Kb * G,
                 L::ypass_toep_quad(p->ey, gy, p->thr_y, p->smem_yt, st, g, p->G1, p->part_rtar)))
    LAUNCH(p, K_ALPHA, st, icon::k_alpha<<<G, 32 * p->B, 0, st>>>(p->part_rtr, p->N1, p->part_rtar, p->n0, p->B, p->alpha, hist_a, hist_r));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status launch_iteration_xt(icon_plan *p, int G, bool clamp, int data_type, float thr, double *hist_a,
                                double *hist_r, cudaStream_t st)
{
    if (p->upd_pending && p->upd_G != G) ICON_TRY(flush_update(p, st));
    ICON_TRY(launch_iteration_xt_raw(p, G, p->upd_pending, p->upd_clamp, p->upd_dtype, p->upd_thr, hist_a, hist_r, st));
    p->upd_pending = true;
    p->upd_clamp = clamp;
    p->upd_dtype = data_type;
    p->upd_thr = thr;
    p->upd_G = G;
    return ICON_OK;
}

// One ICON iteration with A^H W A as a convolution (k_ypass_toep): the same
// steps as launch_iteration, f-hat = A^H W A m and rtar = r^H A^H W A r
// taken from the Toeplitz form instead of the NUFFT pair.  With the
// three-step x-kernels and no step measurement it is launch_iteration_xt.
icon_status launch_iteration_toep(icon_plan *p, int G, bool clamp, int data_type, float thr, double *hist_a,
                                  double *hist_r, cudaStream_t st, bool measure_step)
{
    if (p->xt_ok && !measure_step) return launch_iteration_xt(p, G, clamp, data_type, thr, hist_a, hist_r, st);
    ICON_TRY(flush_update(p, st));
    Geo g = p->geo_unit();
    const double slots = (double)G * p->B;
    const double NN = (double)p->N0 * p->N1, G1b = (double)p->n0 * p->N1 * 8, Kb = (double)p->n0 * p->n1t * 4;
    dim3 gx(p->N1, G), gy(G, p->n0);
    WITH_B(p->B,
        LAUNCH_B(p, K_XF, st, (NN * 4 + G1b) * slots, L::xpass_fwd_full(p->ex, gx, p->thr_x, p->smem_x, st, g, p->m, p->G1));
        LAUNCH_B(p, K_YT, st, (2 * G1b) * slots + Kb * G, L::ypass_toep(p->ey, gy, p->thr_y, p->smem_yt, st, g, p->G1));
        LAUNCH_B(p, K_XA, st, (G1b + NN * 16) * slots,
                 L::xpass_adj(1, p->ex, gx, p->thr_x, p->smem_x + sizeof(double) * p->thr_x, st, g, p->G1, p->rhat,
                              p->Ahwb, p->part_rtr));
        LAUNCH_B(p, K_XF, st, (NN * 8 + G1b) * slots, L::xpass_fwd(false, p->ex, gx, p->thr_x, p->smem_x, st, g, p->rhat, p->G1));
        LAUNCH_B(p, K_YQ, st, G1b * slots + Kb * G,
                 L::ypass_toep_quad(p->ey, gy, p->thr_y, p->smem_yt, st, g, p->G1, p->part_rtar)))
    LAUNCH(p, K_ALPHA, st, icon::k_alpha<<<G, 32 * p->B, 0, st>>>(p->part_rtr, p->N1, p->part_rtar, p->n0, p->B, p->alpha, hist_a, hist_r));
    int per_group = p->N1 * p->N0 * p->B;
    dim3 gu((unsigned)std::min<size_t>(((size_t)per_group + 255) / 256, 512), G);
    WITH_B(p->B, LAUNCH_B(p, K_UPD, st, stage_bytes(p, p->nodes).upd * G * p->B,
                          L::update(gu, st, p->m, p->rhat, p->alpha, per_group, clamp ? 1 : 0, data_type, thr,
                                    measure_step ? p->step_part : nullptr)))
    if (measure_step) {
        const int slots_i = G * p->B;
        LAUNCH(p, K_UPD, st, icon::k_step_reduce<<<(slots_i + 127) / 128, 128, 0, st>>>(p->step_part, (int)gu.x, p->B, slots_i, p->step));
    }
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// The schedule (Iteration2.cu:129-132) on the plan's m for G groups of which
// the first S slices count, with the ICON phase ended once every one of
// those slices' relative step ||m_new - m_old|| / ||m_new|| is at or below
// tol (checked every check_every ICON iterations and at the phase's last;
// each check synchronises the stream).  *done receives the iterations run
// and h_step (optional) the slices' steps at the last check.
icon_status run_schedule_tol(icon_plan *p, const icon_solve_cfg *cfg, int G, int S, double tol, int check_every,
                             int *done_out, double *h_step, cudaStream_t st)
{
    const int a = cfg->infr_before, b = cfg->icon, c = cfg->infr_after;
    const size_t slots = (size_t)G * p->B;
    std::vector<double> hs(slots);
    icon_status rc = ICON_OK;
    int done = 0;
    p->upd_pending = false;
    auto run = [&](int n, bool clamp, bool checked) {
        for (int k = 0; k < n && rc == ICON_OK; ++k) {
            // tol = 0 never stops: only the phase's last step is measured, for h_step
            const bool check = checked && ((tol > 0.0 && (k + 1) % check_every == 0) || k + 1 == n);
            rc = launch_iteration(p, G, clamp, cfg->data_type, cfg->threshold, nullptr, nullptr, st, check);
            ++done;
            if (rc != ICON_OK || !check) continue;
            cudaError_t e = cudaMemcpyAsync(hs.data(), p->step, sizeof(double) * slots, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
                break;
            }
            bool all = true;
            for (int s = 0; s < S; ++s) {
                if (h_step) h_step[s] = hs[s];
                if (!(hs[s] <= tol)) all = false;
            }
            if (all) break;
        }
    };
    run(a, false, false);      // INFR (Iteration2.cu:129-132)
    run(b, true, tol > 0.0 || h_step != nullptr);   // ICON, stopped once every slice's step is within tol
    run(c, false, false);      // INFR
    if (rc == ICON_OK) rc = flush_update(p, st);
    p->upd_pending = false;
    if (done_out) *done_out = done;
    return rc;
}

// After the row transform of G groups (Sc slices): Ahwb = A^H W b, m = 0,
// the schedule's iterations (MainCode.cu:115-140 with Iteration3), ended at
// the plan's tolerance when one is set (icon_plan_set_stop).
icon_status solve_from_rows_warm(icon_plan *p, const icon_solve_cfg *cfg, int G, int Sc, cudaStream_t st);

icon_status solve_from_rows(icon_plan *p, const icon_solve_cfg *cfg, int G, int Sc, cudaStream_t st)
{
    if (p->ws) return solve_from_rows_warm(p, cfg, G, Sc, st);
    const int a = cfg->infr_before, b = cfg->icon, c = cfg->infr_after, iters = a + b + c;
    ICON_TRY(ensure_toeplitz(p, st));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->Ahwb, st));
    size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    ICON_CUDA(cudaMemsetAsync(p->m, 0, tot * sizeof(float), st));
    if (p->stop_tol > 0.0) return run_schedule_tol(p, cfg, G, Sc, p->stop_tol, p->stop_every, nullptr, nullptr, st);
    p->upd_pending = false;
    for (int it = 0; it < iters; ++it)
        ICON_TRY(launch_iteration(p, G, a <= it && it < iters - c, cfg->data_type, cfg->threshold, nullptr, nullptr, st));
    return flush_update(p, st);
}

// The same with the plan's warm start: A^H W b in the caller layout, the
// network's start, icon_solve_warm (its acceptance test and cold redo), the
// result back in the plan's layout for the output stage.
icon_status solve_from_rows_warm(icon_plan *p, const icon_solve_cfg *cfg, int G, int Sc, cudaStream_t st)
{
    ICON_TRY(ensure_toeplitz(p, st));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->Ahwb, st));
    const size_t NN = (size_t)p->N0 * p->N1;
    LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float2><<<grid1d((size_t)Sc * NN), 256, 0, st>>>(p->Ahwb, p->ws_A, Sc, p->N0, p->N1, p->B));
    ICON_CUDA(cudaGetLastError());
    const int wcap = iconx::ws_capacity(p->ws);
    for (int s0 = 0; s0 < Sc; s0 += wcap)
        ICON_TRY(icon_ws_predict(p->ws, p->ws_A + s0 * NN, p->ws_m + s0 * NN, std::min(wcap, Sc - s0), st));
    std::vector<int> why(Sc, 0);
    int iters = 0;
    ICON_TRY(icon_solve_warm(p, cfg, p->ws_A, p->ws_m, Sc, &p->wcfg, why.data(), &iters, st));
    for (int s = 0; s < Sc; ++s) (why[s] == ICON_WARM_ACCEPTED ? p->warm_accepted : p->warm_redone)++;
    const size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float><<<grid1d(tot), 256, 0, st>>>(p->ws_m, p->m, Sc, p->N0, p->N1, p->B, tot));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status line_tables(icon_plan *p, float tilt_deg, NodeTables **out)
{
    auto it = p->lines.find(tilt_deg);
    if (it != p->lines.end()) {
        *out = it->second.get();
        return ICON_OK;
    }
    auto t = std::make_unique<NodeTables>();
    float thn = -tilt_deg;
    std::vector<float> xy((size_t)2 * p->nx), w((size_t)p->nx, 1.0f);
    px2d(p->nx, 1, &thn, xy.data());
    ICON_TRY(build_tables(p, xy.data(), w.data(), p->nx, *t));
    *out = t.get();
    p->lines[tilt_deg] = std::move(t);
    return ICON_OK;
}

icon_status reproject_internal(icon_plan *p, const float *m_int, float tilt_deg, float *d_out, int S, cudaStream_t st)
{
    NodeTables *lt = nullptr;
    ICON_TRY(line_tables(p, tilt_deg, &lt));
    int G = groups(p, S);
    ICON_TRY(launch_forward(p, *lt, m_int, true, G, 0, p->fline, st));
    Geo g = p->geo(*lt);
    WITH_B(p->B, LAUNCH(p, K_ROWADJ, st, L::row_adj(p->ex, dim3(G), p->thr_x, p->smem_x, st, g, p->geo1(), p->fline, d_out, S)))
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

}  // namespace

// ================================================================ C ABI ====
extern "C" {

const char *icon_last_error(void) { return g_last_error.c_str(); }

icon_status icon_devices(int *h_count, int *h_sm, int max)
{
    if (!h_count) return fail(ICON_ERR_INVALID, "null argument");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *h_count = 0;
        cudaGetLastError();
        return fail(ICON_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    *h_count = n;
    for (int d = 0; h_sm && d < n && d < max; ++d) {
        int sm = 0;
        ICON_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, d));
        h_sm[d] = sm;
    }
    return ICON_OK;
}

static icon_status plan_create_impl(const icon_geometry *geo, int group, icon_plan **out);

icon_status icon_plan_create(const icon_geometry *geo, icon_plan **out) { return plan_create_impl(geo, 0, out); }

// group > 0: slices per group (1, 2, 4 or 8, at most the size's default);
// 0: the default choice.
static icon_status plan_create_impl(const icon_geometry *geo, int group, icon_plan **out)
{
    if (!geo || !out) return fail(ICON_ERR_INVALID, "null argument");
    *out = nullptr;
    int nx = geo->nx, N1 = geo->thickness == 0 ? geo->nx : geo->thickness, nz = geo->ntilt;
    if (nx < 8 || N1 < 8) return fail(ICON_ERR_INVALID, "nx and thickness must be >= 8");
    if (nx > 4096 || N1 > 4096) return fail(ICON_ERR_INVALID, "nx and thickness must be <= 4096");
    if (nz < 2 || !geo->tilt_deg) return fail(ICON_ERR_INVALID, "need at least 2 tilt angles");
    if (geo->capacity < 1) return fail(ICON_ERR_INVALID, "capacity must be >= 1");
    if ((long long)nx * nz * kTaps >= (1LL << 27)) return fail(ICON_ERR_INVALID, "too many nodes");
    int dev = geo->device;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) return fail(ICON_ERR_CUDA, "no CUDA device");
    }
    DeviceGuard guard(dev);
    if (!guard.ok) return fail(ICON_ERR_CUDA, "cudaSetDevice failed");
    auto p = std::make_unique<icon_plan>();
    p->dev = dev;
    p->nx = nx;
    p->N0 = nx;
    p->N1 = N1;
    p->nz = nz;
    p->M = nx * nz;
    grid_params(p->N0, p->th0, p->n0, p->b0, p->bf0);
    grid_params(p->N1, p->th1, p->n1, p->b1, p->bf1);
    if (geo->window != ICON_WINDOW_GAUSS6 && geo->window != ICON_WINDOW_KB4)
        return fail(ICON_ERR_INVALID, "window must be ICON_WINDOW_GAUSS6 or ICON_WINDOW_KB4");
    p->window = geo->window;
    if (p->window == ICON_WINDOW_KB4) {
        p->kb0 = kb_shape(p->th0);
        p->kb1 = kb_shape(p->th1);
        p->tlo = icon::kKbTlo;
        p->thi = icon::kKbThi;
    }
    p->lg0 = ilog2(p->n0);
    p->lg1 = ilog2(p->n1);
    int nmax = std::max(p->n0, p->n1);
    int B = nmax <= 2048 ? 8 : (nmax <= 4096 ? 4 : 2);
    // ICON_BATCH=1|2|4|8 lowers the slices per group, for tuning.
    if (const char *ov = std::getenv("ICON_BATCH")) {
        int v = atoi(ov);
        if ((v == 1 || v == 2 || v == 4 || v == 8) && v < B) B = v;
    }
    if (group > 0) {
        if (group != 1 && group != 2 && group != 4 && group != 8) return fail(ICON_ERR_INVALID, "group must be 1, 2, 4 or 8");
        B = std::min(B, group);
    }
    while (B > 1 && B / 2 >= geo->capacity) B /= 2;
    p->B = B;
    p->cap = geo->capacity;
    p->Gcap = (geo->capacity + B - 1) / B;
    p->tlt.assign(geo->tilt_deg, geo->tilt_deg + nz);
    p->th_neg.resize(nz);
    for (int i = 0; i < nz; ++i) p->th_neg[i] = -p->tlt[i];   // MainCode.cu:42
    float om = p->th_neg[0];
    p->omit_index = 0;
    for (int i = 0; i < nz; ++i)                                // MainCode.cu:46-49
        if (std::fabs(om) > std::fabs(p->th_neg[i])) {
            om = p->th_neg[i];
            p->omit_index = i;
        }
    p->reproj_deg = p->tlt[p->omit_index];
    p->xy.resize((size_t)2 * p->M);
    p->w.resize(p->M);
    px2d(nx, nz, p->th_neg.data(), p->xy.data());
    weights(nx, nz, p->th_neg.data(), p->w.data());
    ICON_TRY(build_tables(p.get(), p->xy.data(), p->w.data(), p->M, p->nodes));
    std::vector<float> cx = deapod(p->N0, p->n0, p->b0, p->kb0), cy = deapod(p->N1, p->n1, p->b1, p->kb1);
    ICON_TRY(p->arena.upload(&p->cx, cx.data(), cx.size()));
    ICON_TRY(p->arena.upload(&p->cy, cy.data(), cy.size()));
    std::vector<float> rcx(cx.size()), rcy(cy.size());
    for (size_t i = 0; i < cx.size(); ++i) rcx[i] = (float)(1.0 / (double)cx[i]);
    for (size_t i = 0; i < cy.size(); ++i) rcy[i] = (float)(1.0 / (double)cy[i]);
    ICON_TRY(p->arena.upload(&p->rcx, rcx.data(), rcx.size()));
    ICON_TRY(p->arena.upload(&p->rcy, rcy.data(), rcy.size()));
    // 1-D row transform nodes (k - nx/2)/nx (MainCode.cu:72-80).
    std::vector<float> px1((size_t)nx);
    for (int k = 0; k < nx; ++k) px1[k] = (float)(((double)(float)k - (double)(float)nx / 2.0) / (double)(float)nx);
    float *px1_d = nullptr;
    ICON_TRY(p->arena.upload(&px1_d, px1.data(), px1.size()));
    ICON_TRY(p->arena.alloc(&p->phi1, (size_t)nx * kTaps));
    ICON_TRY(p->arena.alloc(&p->i10, (size_t)nx));
    icon::k_window<<<(nx + 255) / 256, 256>>>(px1_d, 1, nx, p->n0, p->b0, p->bf0, p->phi1, kTaps, p->i10, p->kb0,
                                              kb_inv(p->kb0));
    ICON_CUDA(cudaGetLastError());
    std::vector<float2> t0 = twiddles(p->n0), t0h = twiddles(p->n0 / 2), t1 = twiddles(p->n1);
    ICON_TRY(p->arena.upload(&p->tw0, t0.data(), t0.size()));
    ICON_TRY(p->arena.upload(&p->tw0h, t0h.data(), t0h.size()));
    ICON_TRY(p->arena.upload(&p->tw1, t1.data(), t1.size()));
    // Launch shapes: an FFT thread owns E values of an [n][B] batch: 32 when
    // radix-32 passes need fewer passes than radix-16 ones and the block still
    // has a full warp, else 16.
    auto pick_e = [&](int lg, int n) {
        bool fewer = (lg + 4) / 5 < (lg + 3) / 4;
        return (fewer && n * B >= 32 * 32) ? 32 : 16;
    };
    p->ex = pick_e(p->lg0, p->n0);
    p->ey = pick_e(p->lg1, p->n1);
    // ICON_FFT_E="ex,ey" (each 16 or 32) overrides the choice, for tuning.
    if (const char *ov = std::getenv("ICON_FFT_E")) {
        int a = 0, c = 0;
        if (sscanf(ov, "%d,%d", &a, &c) == 2) {
            if ((a == 16 || a == 32) && p->n0 * B >= a * 32) p->ex = a;
            if ((c == 16 || c == 32) && p->n1 * B >= c * 32) p->ey = c;
        }
    }
    p->thr_x = p->n0 * B / p->ex;
    p->thr_y = p->n1 * B / p->ey;
    p->smem_x = (size_t)p->n0 * B * sizeof(float2);
    p->smem_y = icon::ypass_fwd_smem(p->n1, B);
    p->smem_ya = icon::ypass_adj_smem(p->n1, B);
    // Toeplitz y-length: a circular convolution of the N1 rows with a kernel
    // of support 2 N1 - 1 needs 2 N1 - 1 points; the four-step kernel takes
    // 32 R for R in {4, 6, 8, 10, 12, 16, 20, 24, 32}.  ICON_TOEP_POW2=1 keeps
    // the power of two n1 (for comparison).
    p->n1t = p->n1;
    if (icon::ytoep4_fits(p->n1) && !std::getenv("ICON_TOEP_POW2")) {
        for (int R : {4, 6, 8, 10, 12, 16, 20, 24, 32})
            if (32 * R >= 2 * N1 - 1 && 32 * R <= p->n1) {
                p->n1t = 32 * R;
                break;
            }
    }
    if (p->n1t == p->n1) {
        p->tw1t = p->tw1;
    } else {
        std::vector<float2> t1t = twiddles(p->n1t);
        ICON_TRY(p->arena.upload(&p->tw1t, t1t.data(), t1t.size()));
    }
    p->smem_yt = icon::ypass_toep_smem(p->n1, B);
    int smem_max = 0;
    ICON_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    size_t need_x = p->smem_x + sizeof(double) * p->thr_x;
    if ((size_t)smem_max < std::max(std::max(need_x, p->smem_yt), std::max(p->smem_y, p->smem_ya)))
        return fail(ICON_ERR_INVALID, "FFT buffer exceeds shared memory");
    {
        cudaError_t e = cudaSuccess;
        WITH_B(B, e = L::set_smem(p->ex, p->ey, p->smem_x, need_x, p->smem_y, p->smem_ya, p->smem_yt))
        if (e != cudaSuccess) return fail(ICON_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        WITH_B(B, e = L::xtoep_prepare(p->n0))
        if (e != cudaSuccess) return fail(ICON_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        p->xt_ok = p->n0 >= 128 && p->n0 <= 8192 && (size_t)smem_max >= icon::xtoep_smem(p->n0, std::min(B, 8192 / p->n0));
    }
    // Scratch for Gcap groups.
    size_t G = p->Gcap, Bz = B;
    ICON_TRY(p->arena.alloc(&p->G1, G * p->n0 * p->N1 * Bz));
    ICON_TRY(p->arena.alloc(&p->P, G * p->M * kTaps * Bz));
    ICON_TRY(p->arena.alloc(&p->f, G * p->M * Bz));
    ICON_TRY(p->arena.alloc(&p->fline, G * p->nx * Bz));
    size_t NN = (size_t)p->N0 * p->N1;
    ICON_TRY(p->arena.alloc(&p->rhat, G * NN * Bz));
    ICON_TRY(p->arena.alloc(&p->rre, G * NN * Bz));
    ICON_TRY(p->arena.alloc(&p->Ahwb, G * NN * Bz));
    ICON_TRY(p->arena.alloc(&p->imgc, G * NN * Bz));
    ICON_TRY(p->arena.alloc(&p->m, G * NN * Bz));
    ICON_TRY(p->arena.alloc(&p->rows, (size_t)p->cap * nz * nx));
    ICON_TRY(p->arena.alloc(&p->outrp, (size_t)p->cap * nx));
    ICON_TRY(p->arena.alloc(&p->mout, (size_t)p->cap * NN));
    p->k3_blocks = (p->M * B + 255) / 256;
    ICON_TRY(p->arena.alloc(&p->part_rtr, G * p->N1 * Bz));
    // rtar partials: one per k_interp_fin block (NUFFT), one per grid row (Toeplitz)
    ICON_TRY(p->arena.alloc(&p->part_rtar, G * std::max(p->k3_blocks, p->n0) * Bz));
    {
        std::vector<float> one((size_t)std::max(p->N0, p->N1), 1.0f);
        ICON_TRY(p->arena.upload(&p->ones0, one.data(), (size_t)p->N0));
        ICON_TRY(p->arena.upload(&p->ones1, one.data(), (size_t)p->N1));
    }
    ICON_TRY(p->arena.alloc(&p->alpha, G * Bz));
    ICON_TRY(p->arena.alloc(&p->step_part, G * 512 * Bz * 2));
    ICON_TRY(p->arena.alloc(&p->step, G * Bz));
    ICON_TRY(p->arena.alloc(&p->dev_err, 1));
    ICON_CUDA(cudaMemset(p->dev_err, 0, sizeof(int)));
    setup_xt_tma(p.get());
    ICON_CUDA(cudaDeviceSynchronize());
    *out = p.release();
    return ICON_OK;
}

icon_status icon_plan_destroy(icon_plan *plan)
{
    if (!plan) return ICON_OK;
    DeviceGuard guard(plan->dev);
    cudaDeviceSynchronize();
    delete plan;
    return ICON_OK;
}

icon_status icon_plan_set_reprojection(icon_plan *p, float tilt_deg)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (!std::isfinite(tilt_deg)) return fail(ICON_ERR_INVALID, "angle must be finite");
    p->reproj_deg = tilt_deg;
    return ICON_OK;
}

icon_status icon_plan_query(const icon_plan *p, int *dims)
{
    if (!p || !dims) return fail(ICON_ERR_INVALID, "null argument");
    dims[0] = p->N0; dims[1] = p->N1; dims[2] = p->n0; dims[3] = p->n1; dims[4] = p->M;
    dims[5] = p->nz; dims[6] = p->B; dims[7] = p->cap;
    dims[8] = (int)std::min<size_t>(p->arena.total >> 20, 0x7fffffff);
    dims[9] = p->omit_index;
    return ICON_OK;
}

icon_status icon_plan_geometry(const icon_plan *p, float *h_xy, float *h_w)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (h_xy) std::memcpy(h_xy, p->xy.data(), sizeof(float) * p->xy.size());
    if (h_w) std::memcpy(h_w, p->w.data(), sizeof(float) * p->w.size());
    return ICON_OK;
}

icon_status icon_weights(int nx, int ntilt, const float *tilt_deg, float *h_w)
{
    if (!tilt_deg || !h_w || nx < 2 || ntilt < 2) return fail(ICON_ERR_INVALID, "icon_weights: bad argument");
    std::vector<float> neg(ntilt);
    for (int i = 0; i < ntilt; ++i) neg[i] = -tilt_deg[i];   // the plan's node angles (MainCode.cu:46-49)
    weights(nx, ntilt, neg.data(), h_w);
    return ICON_OK;
}

icon_status icon_plan_set_group_weights(icon_plan *p, const float *h_w, int ngroups)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (ngroups == 0) {
        if (p->wgroups != 0) p->kt_stale = true;
        p->wgroups = 0;
        return ICON_OK;
    }
    if (!h_w || ngroups < 0 || ngroups > p->Gcap)
        return fail(ICON_ERR_INVALID, "ngroups must be in 0.." + std::to_string(p->Gcap) + " with weights given");
    DeviceGuard guard(p->dev);
    const size_t M = (size_t)p->M;
    if (!p->wgroup) ICON_TRY(p->arena.alloc(&p->wgroup, (size_t)p->Gcap * M));
    ICON_CUDA(cudaMemcpy(p->wgroup, h_w, sizeof(float) * ngroups * M, cudaMemcpyHostToDevice));
    for (int gi = ngroups; gi < p->Gcap; ++gi)   // the remaining groups keep the plan's own weights
        ICON_CUDA(cudaMemcpy(p->wgroup + gi * M, p->nodes.w, sizeof(float) * M, cudaMemcpyDeviceToDevice));
    // Distinct weight sets, in order of first use: group gi uses set kmap[gi].
    std::vector<const float *> sets;
    std::vector<int> kmap(p->Gcap);
    for (int gi = 0; gi < p->Gcap; ++gi) {
        const float *v = gi < ngroups ? h_w + (size_t)gi * M : p->w.data();
        int k = 0;
        while (k < (int)sets.size() && std::memcmp(sets[k], v, sizeof(float) * M) != 0) ++k;
        if (k == (int)sets.size()) sets.push_back(v);
        kmap[gi] = k;
    }
    if (!p->wuniq) ICON_TRY(p->arena.alloc(&p->wuniq, (size_t)p->Gcap * M));
    if (!p->kidx) ICON_TRY(p->arena.alloc(&p->kidx, (size_t)p->Gcap));
    for (size_t k = 0; k < sets.size(); ++k)
        ICON_CUDA(cudaMemcpy(p->wuniq + k * M, sets[k], sizeof(float) * M, cudaMemcpyHostToDevice));
    ICON_CUDA(cudaMemcpy(p->kidx, kmap.data(), sizeof(int) * p->Gcap, cudaMemcpyHostToDevice));
    p->kt_unique = (int)sets.size();
    p->wgroups = ngroups;
    p->kt_stale = true;
    return ICON_OK;
}

icon_status icon_plan_set_warm_start(icon_plan *p, icon_ws *ws, const icon_warm_cfg *wc)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (!ws) {
        p->ws = nullptr;
        return ICON_OK;
    }
    if (!wc || !(wc->tol > 0.0) || wc->check_every < 1 || !(wc->max_dist > 0.0))
        return fail(ICON_ERR_INVALID, "icon_plan_set_warm_start: tol > 0, check_every >= 1 and max_dist > 0 required");
    if (iconx::ws_capacity(ws) < 1) return fail(ICON_ERR_INVALID, "icon_plan_set_warm_start: bad network");
    DeviceGuard guard(p->dev);
    const size_t NN = (size_t)p->N0 * p->N1;
    if (!p->ws_A) ICON_TRY(p->arena.alloc(&p->ws_A, (size_t)p->cap * NN));
    if (!p->ws_m) ICON_TRY(p->arena.alloc(&p->ws_m, (size_t)p->cap * NN));
    p->ws = ws;
    p->wcfg = *wc;
    return ICON_OK;
}

icon_status icon_plan_warm_counts(const icon_plan *p, long long *h_accepted, long long *h_redone)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (h_accepted) *h_accepted = p->warm_accepted;
    if (h_redone) *h_redone = p->warm_redone;
    return ICON_OK;
}

icon_status icon_plan_set_stop(icon_plan *p, double tol, int check_every)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (!(tol >= 0.0) || check_every < 1) return fail(ICON_ERR_INVALID, "tol must be >= 0 and check_every >= 1");
    p->stop_tol = tol;
    p->stop_every = check_every;
    return ICON_OK;
}

icon_status icon_plan_set_operator(icon_plan *p, int op)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (op != ICON_OPERATOR_NUFFT && op != ICON_OPERATOR_TOEPLITZ) return fail(ICON_ERR_INVALID, "unknown operator");
    if (op != p->op) p->kt_stale = true;
    p->op = op;
    return ICON_OK;
}

icon_status icon_nufft_forward(icon_plan *p, const float *d_img, void *d_nodes, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_img || !d_nodes) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float><<<grid1d(tot), 256, 0, st>>>(d_img, p->m, S, p->N0, p->N1, p->B, tot));
    ICON_TRY(launch_forward(p, p->nodes, p->m, true, G, 0, p->f, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_nodes_out<<<grid1d((size_t)S * p->M), 256, 0, st>>>(p->f, (float2 *)d_nodes, S, p->M, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_nufft_forward_complex(icon_plan *p, const void *d_img, void *d_nodes, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_img || !d_nodes) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float2><<<grid1d(tot), 256, 0, st>>>((const float2 *)d_img, p->imgc, S, p->N0, p->N1, p->B, tot));
    ICON_TRY(launch_forward(p, p->nodes, p->imgc, false, G, 0, p->f, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_nodes_out<<<grid1d((size_t)S * p->M), 256, 0, st>>>(p->f, (float2 *)d_nodes, S, p->M, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_nufft_adjoint(icon_plan *p, const void *d_nodes, void *d_img, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_img || !d_nodes) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    size_t tot = (size_t)G * p->M * p->B;
    LAUNCH(p, K_LAYOUT, st, icon::k_nodes_in<<<grid1d(tot), 256, 0, st>>>((const float2 *)d_nodes, p->f, S, p->M, p->B, tot));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->imgc, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float2><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->imgc, (float2 *)d_img, S, p->N0, p->N1, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_rows_forward(icon_plan *p, const float *d_rows, void *d_b, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_rows || !d_b) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    ICON_TRY(launch_rows(p, d_rows, S, G, p->P, st));   // unweighted b into scratch
    LAUNCH(p, K_LAYOUT, st, icon::k_nodes_out<<<grid1d((size_t)S * p->M), 256, 0, st>>>(p->P, (float2 *)d_b, S, p->M, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_prepare_rhs(icon_plan *p, const float *d_rows, void *d_Ahwb, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_rows || !d_Ahwb) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    ICON_TRY(launch_rows(p, d_rows, S, G, nullptr, st));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->imgc, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float2><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->imgc, (float2 *)d_Ahwb, S, p->N0, p->N1, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

// Stack arguments shared by the two stack entry points: the plan's tilts
// read sections 0..nz-1 of the stack, or nz+1 sections with skip_section
// left out.
static icon_status check_stack(const icon_plan *p, const float *d_stack, int ny, int y0, int skip_section, int S)
{
    if (!d_stack) return fail(ICON_ERR_INVALID, "null stack");
    if (ny < 1 || y0 < 0 || S < 1 || (long long)y0 + S > ny)
        return fail(ICON_ERR_INVALID, "slices " + std::to_string(y0) + "..+" + std::to_string(S) + " outside 0.." +
                                          std::to_string(ny - 1));
    if (skip_section > p->nz) return fail(ICON_ERR_INVALID, "skip_section beyond the stack");
    return ICON_OK;
}

icon_status icon_prepare_rhs_stack(icon_plan *p, const float *d_stack, int ny, int y0, int skip_section,
                                   void *d_Ahwb, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    ICON_TRY(check_stack(p, d_stack, ny, y0, skip_section, S));
    if (!d_Ahwb) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    const size_t nx = p->nx;
    ICON_TRY(launch_rows_at(p, d_stack + (size_t)y0 * nx, nx, (size_t)ny * nx, skip_section < 0 ? INT_MAX : skip_section,
                            S, G, nullptr, st));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->imgc, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float2><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->imgc, (float2 *)d_Ahwb, S, p->N0, p->N1, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_reconstruct_stack(icon_plan *p, const icon_solve_cfg *cfg, const float *d_stack, int ny, int y0,
                                   int skip_section, float *d_slices, float *d_reproj, int S, void *stream)
{
    if (!p || !cfg) return fail(ICON_ERR_INVALID, "null argument");
    if (!d_slices && !d_reproj) return fail(ICON_ERR_INVALID, "no output buffer");
    ICON_TRY(check_stack(p, d_stack, ny, y0, skip_section, S));
    if (cfg->infr_before < 0 || cfg->icon < 0 || cfg->infr_after < 0) return fail(ICON_ERR_INVALID, "negative iteration count");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nx = p->nx, NN = (size_t)p->N0 * p->N1;
    const int skip = skip_section < 0 ? INT_MAX : skip_section;
    for (int s0 = 0; s0 < S; s0 += p->cap) {
        const int Sc = std::min(p->cap, S - s0), G = groups(p, Sc);
        ICON_TRY(launch_rows_at(p, d_stack + (size_t)(y0 + s0) * nx, nx, (size_t)ny * nx, skip, Sc, G, nullptr, st));
        ICON_TRY(solve_from_rows(p, cfg, G, Sc, st));
        if (d_slices) {
            dim3 gl((unsigned)std::min<size_t>(((size_t)G * NN + 255) / 256, 4096));
            WITH_B(p->B, LAUNCH(p, K_LAYOUT, st, L::img_out_file(gl, st, p->m, d_slices + (size_t)s0 * NN, Sc, p->N0, p->N1)))
            ICON_CUDA(cudaGetLastError());
        }
        if (d_reproj) ICON_TRY(reproject_internal(p, p->m, p->reproj_deg, d_reproj + (size_t)s0 * nx, Sc, st));
    }
    return ICON_OK;
}

icon_status icon_reconstruct_stack_host(icon_plan *p, const icon_solve_cfg *cfg, const float *d_stack, int ny, int y0,
                                        int skip_section, int S, int outputs, icon_batch_sink sink, void *ctx,
                                        void *stream)
{
    if (!p || !cfg || !sink) return fail(ICON_ERR_INVALID, "null argument");
    if ((outputs & 3) == 0 || (outputs & ~3)) return fail(ICON_ERR_INVALID, "outputs must be a nonempty set of ICON_OUT_* bits");
    ICON_TRY(check_stack(p, d_stack, ny, y0, skip_section, S));
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    bool own = (st == nullptr);
    if (own) ICON_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t NN = (size_t)p->N0 * p->N1, nx = p->nx;
    const bool want_m = outputs & ICON_OUT_SLICES, want_rp = outputs & ICON_OUT_REPROJECTION;
    // Two pinned host buffers (slices, then reprojections) and two events:
    // batch k copies into buffer k % 2 while the sink consumes batch k - 1.
    float *h[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const size_t per = (want_m ? (size_t)p->cap * NN : 0) + (want_rp ? (size_t)p->cap * nx : 0);
    icon_status rc = ICON_OK;
    for (int k = 0; k < 2 && rc == ICON_OK; ++k) {
        cudaError_t e = cudaHostAlloc((void **)&h[k], per * sizeof(float), cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
    }
    auto hm = [&](int k) { return h[k]; };
    auto hr = [&](int k) { return h[k] + (want_m ? (size_t)p->cap * NN : 0); };
    int pend_s0 = -1, pend_n = 0, pend_k = 0;
    auto drain = [&]() -> icon_status {      // waits for the pending batch and hands it to the sink
        if (pend_s0 < 0) return ICON_OK;
        ICON_CUDA(cudaEventSynchronize(ev[pend_k]));
        int r = sink(ctx, pend_s0, pend_n, want_m ? hm(pend_k) : nullptr, want_rp ? hr(pend_k) : nullptr);
        pend_s0 = -1;
        if (r != 0) return fail(ICON_ERR_INVALID, "the batch sink returned " + std::to_string(r));
        return ICON_OK;
    };
    for (int s0 = 0, k = 0; s0 < S && rc == ICON_OK; s0 += p->cap, k ^= 1) {
        const int Sc = std::min(p->cap, S - s0);
        rc = icon_reconstruct_stack(p, cfg, d_stack, ny, y0 + s0, skip_section, want_m ? p->mout : nullptr,
                                    want_rp ? p->outrp : nullptr, Sc, st);
        cudaError_t e = cudaSuccess;
        if (rc == ICON_OK && want_m) e = cudaMemcpyAsync(hm(k), p->mout, sizeof(float) * NN * Sc, cudaMemcpyDeviceToHost, st);
        if (rc == ICON_OK && e == cudaSuccess && want_rp)
            e = cudaMemcpyAsync(hr(k), p->outrp, sizeof(float) * nx * Sc, cudaMemcpyDeviceToHost, st);
        if (rc == ICON_OK && e == cudaSuccess) e = cudaEventRecord(ev[k], st);
        if (rc == ICON_OK && e != cudaSuccess) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
        if (rc == ICON_OK) rc = drain();     // batch k - 1, while batch k runs
        pend_s0 = s0;
        pend_n = Sc;
        pend_k = k;
    }
    if (rc == ICON_OK) rc = drain();
    cudaStreamSynchronize(st);
    for (int k = 0; k < 2; ++k) {
        if (h[k]) cudaFreeHost(h[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
    }
    if (own) cudaStreamDestroy(st);
    return rc;
}

icon_status icon_host_alloc(size_t bytes, void **out)
{
    if (!out) return fail(ICON_ERR_INVALID, "null argument");
    *out = nullptr;
    if (bytes == 0) return fail(ICON_ERR_INVALID, "zero bytes");
    ICON_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
    return ICON_OK;
}

icon_status icon_host_free(void *h)
{
    if (h) ICON_CUDA(cudaFreeHost(h));
    return ICON_OK;
}

icon_status icon_stack_upload(int device, const float *h_stack, int sections, int ny, int nx, int y0, int S,
                              float **d_stack, void *stream)
{
    if (!h_stack || !d_stack) return fail(ICON_ERR_INVALID, "null argument");
    *d_stack = nullptr;
    if (sections < 1 || ny < 1 || nx < 1 || y0 < 0 || S < 1 || (long long)y0 + S > ny)
        return fail(ICON_ERR_INVALID, "stack rows outside the stack");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(ICON_ERR_CUDA, "cannot select device " + std::to_string(device));
    float *d = nullptr;
    ICON_CUDA(cudaMalloc(&d, sizeof(float) * (size_t)sections * S * nx));
    // One 2-D copy: per section, the S rows y0 .. y0+S-1 (contiguous in the
    // file), to a packed [sections][S][nx].
    cudaError_t e = cudaMemcpy2DAsync(d, sizeof(float) * (size_t)S * nx, h_stack + (size_t)y0 * nx,
                                      sizeof(float) * (size_t)ny * nx, sizeof(float) * (size_t)S * nx, sections,
                                      cudaMemcpyHostToDevice, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        return fail(ICON_ERR_CUDA, cudaGetErrorString(e));
    }
    *d_stack = d;
    return ICON_OK;
}

icon_status icon_device_free(int device, void *d)
{
    if (!d) return ICON_OK;
    DeviceGuard guard(device);
    ICON_CUDA(cudaFree(d));
    return ICON_OK;
}

icon_status icon_solve(icon_plan *p, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S, int warm_start,
                       double *h_alpha, double *h_rtr, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!cfg || !d_Ahwb || !d_m) return fail(ICON_ERR_INVALID, "null argument");
    int a = cfg->infr_before, b = cfg->icon, c = cfg->infr_after;
    if (a < 0 || b < 0 || c < 0) return fail(ICON_ERR_INVALID, "negative iteration count");
    int iters = a + b + c;
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    ICON_TRY(ensure_toeplitz(p, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float2><<<grid1d(tot), 256, 0, st>>>((const float2 *)d_Ahwb, p->Ahwb, S, p->N0, p->N1, p->B, tot));
    if (warm_start) LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float><<<grid1d(tot), 256, 0, st>>>(d_m, p->m, S, p->N0, p->N1, p->B, tot));
    else ICON_CUDA(cudaMemsetAsync(p->m, 0, tot * sizeof(float), st));
    double *hist = nullptr;
    size_t slots = (size_t)G * p->B;
    bool want_hist = (h_alpha || h_rtr) && iters > 0;
    if (want_hist) ICON_CUDA(cudaMalloc(&hist, sizeof(double) * 2 * slots * iters));
    icon_status rc = ICON_OK;
    p->upd_pending = false;
    for (int it = 0; it < iters && rc == ICON_OK; ++it) {
        bool clamp = (a <= it && it < iters - c);              // Iteration2.cu:129
        double *ha = want_hist ? hist + (size_t)it * slots : nullptr;
        double *hr = want_hist ? hist + (size_t)(iters + it) * slots : nullptr;
        rc = launch_iteration(p, G, clamp, cfg->data_type, cfg->threshold, ha, hr, st);
    }
    if (rc == ICON_OK) rc = flush_update(p, st);
    p->upd_pending = false;
    if (rc == ICON_OK) {
        LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->m, d_m, S, p->N0, p->N1, p->B));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
    }
    if (want_hist) {
        std::vector<double> hv(2 * slots * iters);
        cudaError_t e = cudaMemcpyAsync(hv.data(), hist, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(hist);
        if (e != cudaSuccess && rc == ICON_OK) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
        if (rc == ICON_OK)
            for (int it = 0; it < iters; ++it)
                for (int s = 0; s < S; ++s) {
                    if (h_alpha) h_alpha[(size_t)it * S + s] = hv[(size_t)it * slots + s];
                    if (h_rtr) h_rtr[(size_t)it * S + s] = hv[(size_t)(iters + it) * slots + s];
                }
    }
    return rc;
}

icon_status icon_solve_until(icon_plan *p, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S,
                            int warm_start, double tol, int check_every, int *h_iters, double *h_step, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!cfg || !d_Ahwb || !d_m) return fail(ICON_ERR_INVALID, "null argument");
    if (!(tol >= 0.0) || check_every < 1) return fail(ICON_ERR_INVALID, "tol must be >= 0 and check_every >= 1");
    const int a = cfg->infr_before, b = cfg->icon, c = cfg->infr_after;
    if (a < 0 || b < 0 || c < 0) return fail(ICON_ERR_INVALID, "negative iteration count");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    const int G = groups(p, S);
    const size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    ICON_TRY(ensure_toeplitz(p, st));
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float2><<<grid1d(tot), 256, 0, st>>>((const float2 *)d_Ahwb, p->Ahwb, S, p->N0, p->N1, p->B, tot));
    if (warm_start) LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float><<<grid1d(tot), 256, 0, st>>>(d_m, p->m, S, p->N0, p->N1, p->B, tot));
    else ICON_CUDA(cudaMemsetAsync(p->m, 0, tot * sizeof(float), st));
    int done = 0;
    icon_status rc = run_schedule_tol(p, cfg, G, S, tol, check_every, &done, h_step, st);
    if (rc == ICON_OK) {
        LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->m, d_m, S, p->N0, p->N1, p->B));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
    }
    if (h_iters) *h_iters = done;
    return rc;
}

icon_status icon_reproject_host(icon_plan *p, const float *h_m, float tilt_deg, float *h_out, int S, void *stream)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    if (!h_m || !h_out) return fail(ICON_ERR_INVALID, "null buffer");
    if (S < 1) return fail(ICON_ERR_INVALID, "S must be >= 1");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t NN = (size_t)p->N0 * p->N1, nx = p->nx;
    for (int s0 = 0; s0 < S; s0 += p->cap) {
        const int Sc = std::min(p->cap, S - s0);
        ICON_CUDA(cudaMemcpyAsync(p->mout, h_m + (size_t)s0 * NN, sizeof(float) * NN * Sc, cudaMemcpyHostToDevice, st));
        ICON_TRY(icon_reproject(p, p->mout, tilt_deg, p->outrp, Sc, st));
        ICON_CUDA(cudaMemcpyAsync(h_out + (size_t)s0 * nx, p->outrp, sizeof(float) * nx * Sc, cudaMemcpyDeviceToHost, st));
        ICON_CUDA(cudaStreamSynchronize(st));
    }
    return ICON_OK;
}

icon_status icon_reproject(icon_plan *p, const float *d_m, float tilt_deg, float *d_out, int S, void *stream)
{
    ICON_TRY(check_plan(p, S));
    if (!d_m || !d_out) return fail(ICON_ERR_INVALID, "null buffer");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    int G = groups(p, S);
    size_t tot = (size_t)G * p->N1 * p->N0 * p->B;
    LAUNCH(p, K_LAYOUT, st, icon::k_img_in<float><<<grid1d(tot), 256, 0, st>>>(d_m, p->m, S, p->N0, p->N1, p->B, tot));
    ICON_CUDA(cudaGetLastError());
    return reproject_internal(p, p->m, tilt_deg, d_out, S, st);
}

icon_status icon_reconstruct_host(icon_plan *p, const icon_solve_cfg *cfg, const float *h_rows, float *h_m,
                                  float *h_reproj, int S, void *stream)
{
    if (!p || !cfg || !h_rows || !h_m) return fail(ICON_ERR_INVALID, "null argument");
    if (S < 1) return fail(ICON_ERR_INVALID, "S must be >= 1");
    DeviceGuard guard(p->dev);
    cudaStream_t st = (cudaStream_t)stream;
    bool own = (st == nullptr);
    if (own) ICON_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    icon_status rc = ICON_OK;
    size_t R = (size_t)p->nz * p->nx, NN = (size_t)p->N0 * p->N1;
    float *d_mo = p->mout;
    if (cfg->infr_before < 0 || cfg->icon < 0 || cfg->infr_after < 0) return fail(ICON_ERR_INVALID, "negative iteration count");
    for (int s0 = 0; s0 < S && rc == ICON_OK; s0 += p->cap) {
        int Sc = std::min(p->cap, S - s0);
        int G = groups(p, Sc);
        cudaError_t e = cudaMemcpyAsync(p->rows, h_rows + (size_t)s0 * R, sizeof(float) * R * Sc, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e)); break; }
        if ((rc = launch_rows(p, p->rows, Sc, G, nullptr, st)) != ICON_OK) break;
        if ((rc = solve_from_rows(p, cfg, G, Sc, st)) != ICON_OK) break;
        LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float><<<grid1d((size_t)Sc * NN), 256, 0, st>>>(p->m, d_mo, Sc, p->N0, p->N1, p->B));
        if (h_reproj && (rc = reproject_internal(p, p->m, p->reproj_deg, p->outrp, Sc, st)) != ICON_OK) break;
        if ((e = cudaMemcpyAsync(h_m + (size_t)s0 * NN, d_mo, sizeof(float) * NN * Sc, cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
            rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
            break;
        }
        if (h_reproj && (e = cudaMemcpyAsync(h_reproj + (size_t)s0 * p->nx, p->outrp, sizeof(float) * p->nx * Sc,
                                             cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
            rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
            break;
        }
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaStreamSynchronize(st);
    if (own) cudaStreamDestroy(st);
    return rc;
}

icon_status icon_trace_enable(icon_plan *p, int enable)
{
    if (!p) return fail(ICON_ERR_INVALID, "null plan");
    p->trace = enable != 0;
    return ICON_OK;
}

icon_status icon_trace_read(icon_plan *p, int *h_count, double *h_ms, double *h_bytes)
{
    if (!p || !h_count || !h_ms) return fail(ICON_ERR_INVALID, "null argument");
    DeviceGuard guard(p->dev);
    for (int k = 0; k < ICON_TRACE_KERNELS; ++k) {
        h_count[k] = 0;
        h_ms[k] = 0.0;
        if (h_bytes) h_bytes[k] = 0.0;
    }
    icon_status rc = ICON_OK;
    for (auto &q : p->pending) {
        float ms = 0.f;
        cudaError_t e = cudaEventSynchronize(q.b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, q.a, q.b);
        if (e != cudaSuccess && rc == ICON_OK) rc = fail(ICON_ERR_CUDA, cudaGetErrorString(e));
        if (q.kind >= 0 && q.kind < ICON_TRACE_KERNELS) {
            h_count[q.kind]++;
            h_ms[q.kind] += ms;
            if (h_bytes) h_bytes[q.kind] += q.bytes;
        }
        p->pool.push_back(q.a);
        p->pool.push_back(q.b);
    }
    p->pending.clear();
    return rc;
}

long long icon_launch_count(const icon_plan *p) { return p ? p->launches : 0; }

icon_status icon_plan_device_error(icon_plan *p, int *h_code)
{
    if (!p || !h_code) return fail(ICON_ERR_INVALID, "null argument");
    DeviceGuard guard(p->dev);
    ICON_CUDA(cudaDeviceSynchronize());
    ICON_CUDA(cudaMemcpy(h_code, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
    ICON_CUDA(cudaMemset(p->dev_err, 0, sizeof(int)));
    return ICON_OK;
}

}  // extern "C"

// ------------------------------------------------ hooks of icon_batch.cu ----
namespace iconx {

icon_status plan_create_group(const icon_geometry *geo, int group, icon_plan **out)
{
    return plan_create_impl(geo, group, out);
}
int plan_group(const icon_plan *p) { return p->B; }
int plan_capacity(const icon_plan *p) { return p->cap; }
int plan_device(const icon_plan *p) { return p->dev; }
float *plan_rows_buffer(icon_plan *p) { return p->rows; }
float *plan_out_buffer(icon_plan *p) { return p->mout; }

static bool clamp_at(const icon_solve_cfg *cfg, int it)
{
    const int a = cfg->infr_before, iters = a + cfg->icon + cfg->infr_after;
    return a <= it && it < iters - cfg->infr_after;                // Iteration2.cu:129
}

icon_status plan_stage_in(icon_plan *p, const float *d_rows, int S, cudaStream_t st)
{
    ICON_TRY(check_plan(p, S));
    DeviceGuard guard(p->dev);
    const int G = groups(p, S);
    ICON_TRY(launch_rows(p, d_rows, S, G, nullptr, st));
    ICON_TRY(ensure_toeplitz(p, st));
    ICON_TRY(launch_adjoint(p, p->f, G, 0, p->Ahwb, st));
    ICON_CUDA(cudaMemsetAsync(p->m, 0, (size_t)G * p->N1 * p->N0 * p->B * sizeof(float), st));
    p->upd_pending = false;
    return ICON_OK;
}

icon_status plan_iteration(icon_plan *p, int S, int it, const icon_solve_cfg *cfg, cudaStream_t st)
{
    const int G = groups(p, S);
    if (p->op == ICON_OPERATOR_TOEPLITZ && p->xt_ok)
        return launch_iteration_xt_raw(p, G, it > 0, it > 0 && clamp_at(cfg, it - 1), cfg->data_type, cfg->threshold,
                                       nullptr, nullptr, st);
    return launch_iteration(p, G, clamp_at(cfg, it), cfg->data_type, cfg->threshold, nullptr, nullptr, st);
}

icon_status plan_stage_out(icon_plan *p, int S, const icon_solve_cfg *cfg, float *d_out, cudaStream_t st)
{
    DeviceGuard guard(p->dev);
    const int iters = cfg->infr_before + cfg->icon + cfg->infr_after;
    if (p->op == ICON_OPERATOR_TOEPLITZ && p->xt_ok && iters > 0) {
        p->upd_pending = true;
        p->upd_clamp = clamp_at(cfg, iters - 1);
        p->upd_dtype = cfg->data_type;
        p->upd_thr = cfg->threshold;
        p->upd_G = groups(p, S);
        ICON_TRY(flush_update(p, st));
    }
    LAUNCH(p, K_LAYOUT, st, icon::k_img_out<float><<<grid1d((size_t)S * p->N0 * p->N1), 256, 0, st>>>(p->m, d_out, S, p->N0, p->N1, p->B));
    ICON_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status fail_msg(icon_status st, const std::string &msg) { return fail(st, msg); }

}  // namespace iconx

extern "C" {

// Lets the other translation units of the library report through
// icon_last_error().
void icon_internal_set_error(const char *msg) { g_last_error = msg ? msg : ""; }

}  // extern "C"
