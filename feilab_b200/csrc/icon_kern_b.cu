// icon_kern_b.cu -- the batched FFT kernels for one slice-group size,
// ICON_KB (1, 2, 4 or 8, set by the build), and their host launchers.
#define ICON_KERNELS_TEMPLATES_ONLY
#include "icon_kernels.cuh"
#include "icon_launch.h"

#ifndef ICON_KB
#error "compile with -DICON_KB=<1|2|4|8>"
#endif

namespace icon {

template <int B>
void Launch<B>::xpass_fwd(bool real_in, int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                          const void *in, float2 *G1)
{
    if (real_in && g.n0 / 2 >= E) {   // half-length FFT per slice: half the threads and buffer
        if (E == 32) k_xpass_fwd_r2c<B, 32><<<grid, threads / 2, smem / 2, st>>>(g, (const float *)in, G1);
        else k_xpass_fwd_r2c<B, 16><<<grid, threads / 2, smem / 2, st>>>(g, (const float *)in, G1);
        return;
    }
    if (E == 32) {
        if (real_in) k_xpass_fwd<true, B, 32><<<grid, threads, smem, st>>>(g, in, G1);
        else k_xpass_fwd<false, B, 32><<<grid, threads, smem, st>>>(g, in, G1);
    } else {
        if (real_in) k_xpass_fwd<true, B, 16><<<grid, threads, smem, st>>>(g, in, G1);
        else k_xpass_fwd<false, B, 16><<<grid, threads, smem, st>>>(g, in, G1);
    }
}

template <int B>
void Launch<B>::xpass_fwd_full(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                               const float *in, float2 *G1)
{
    if (g.n0 / 2 >= E) {   // half-length FFT per slice, as xpass_fwd
        if (E == 32) k_xpass_fwd_r2c<B, 32, true><<<grid, threads / 2, smem / 2, st>>>(g, in, G1);
        else k_xpass_fwd_r2c<B, 16, true><<<grid, threads / 2, smem / 2, st>>>(g, in, G1);
        return;
    }
    if (E == 32) k_xpass_fwd<true, B, 32, true><<<grid, threads, smem, st>>>(g, in, G1);
    else k_xpass_fwd<true, B, 16, true><<<grid, threads, smem, st>>>(g, in, G1);
}

// The four-step register FFT (k_ytoep4) for n1 = 32 R, R in
// {4, 6, 8, 10, 12, 16, 20, 24, 32}; blockDim = n1*B/32, shared memory
// n1*B float2.
template <int B, int MODE>
static void launch_ytoep4(dim3 grid, cudaStream_t st, const Geo &g, float2 *G1, double *part)
{
    const int threads = g.n1 * B / 32;
    const size_t smem = ytoep4_smem(g.n1, B);
    switch (g.n1 / 32) {
    case 4: k_ytoep4<B, 4, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 6: k_ytoep4<B, 6, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 8: k_ytoep4<B, 8, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 10: k_ytoep4<B, 10, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 12: k_ytoep4<B, 12, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 16: k_ytoep4<B, 16, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 20: k_ytoep4<B, 20, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    case 24: k_ytoep4<B, 24, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    default: k_ytoep4<B, 32, MODE><<<grid, threads, smem, st>>>(g, G1, part); break;
    }
}

template <int B>
void Launch<B>::ypass_toep(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, float2 *G1)
{
    if (ytoep4_fits(g.n1)) launch_ytoep4<B, 0>(grid, st, g, G1, nullptr);
    else if (E == 32) k_ypass_toep<B, 32><<<grid, threads, smem, st>>>(g, G1);
    else k_ypass_toep<B, 16><<<grid, threads, smem, st>>>(g, G1);
}

template <int B>
void Launch<B>::ypass_toep_quad(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                                const float2 *G1, double *part)
{
    if (ytoep4_fits(g.n1)) launch_ytoep4<B, 1>(grid, st, g, const_cast<float2 *>(G1), part);
    else if (E == 32) k_ypass_toep_quad<B, 32><<<grid, threads, smem, st>>>(g, G1, part);
    else k_ypass_toep_quad<B, 16><<<grid, threads, smem, st>>>(g, G1, part);
}

// k_xtoep for one (BH, NA, NB) shape: grid (N1 * B/BH, G), half-groups fastest.
template <int B, int BH, int LA, int LNB>
static void xt_go(int mode, cudaStream_t st, int G, const XtArgs &a)
{
    using S = XtShape<BH, LA, LNB>;
    const dim3 grid((unsigned)(a.N1 * (B / BH)), (unsigned)G);
    const size_t smem = xtoep_smem(S::N, BH);
    if (mode == 0) k_xtoep<B, BH, LA, LNB, 0><<<grid, S::T, smem, st>>>(a);
    else if (mode == 1) k_xtoep<B, BH, LA, LNB, 1><<<grid, S::T, smem, st>>>(a);
    else k_xtoep<B, BH, LA, LNB, 2><<<grid, S::T, smem, st>>>(a);
}
template <int B, int BH, int LA, int LNB>
static cudaError_t xt_attr()
{
    const int bytes = (int)xtoep_smem(XtShape<BH, LA, LNB>::N, BH);
    cudaError_t e = cudaFuncSetAttribute((const void *)k_xtoep<B, BH, LA, LNB, 0>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void *)k_xtoep<B, BH, LA, LNB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute((const void *)k_xtoep<B, BH, LA, LNB, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bytes);
}

// Slices per CTA: all B up to n0 = 1024, then at most 8192 / n0 (a CTA's
// transposed values stay at 64 KB, two CTAs per SM).
#define ICON_XT_SHAPES(X)                            \
    X(128, B, 2, 0)                                   \
    X(256, B, 3, 0)                                   \
    X(512, B, 4, 0)                                   \
    X(1024, B, 5, 0)                                  \
    X(2048, (B < 4 ? B : 4), 3, 3)                    \
    X(4096, (B < 2 ? B : 2), 4, 3)                    \
    X(8192, 1, 4, 4)

template <int B>
bool Launch<B>::xtoep(int mode, cudaStream_t st, int G, const XtArgs &a)
{
    switch (a.n0) {
#define X(N, BH, LA, LNB) \
    case N: xt_go<B, BH, LA, LNB>(mode, st, G, a); return true;
        ICON_XT_SHAPES(X)
#undef X
    default: return false;
    }
}

template <int B>
cudaError_t Launch<B>::xtoep_prepare(int n0)
{
    switch (n0) {
#define X(N, BH, LA, LNB) \
    case N: return xt_attr<B, BH, LA, LNB>();
        ICON_XT_SHAPES(X)
#undef X
    default: return cudaSuccess;
    }
}

template <int B>
void Launch<B>::ypass_fwd(int E, bool herm, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                          const float2 *G1, float2 *P)
{
    if (E == 32) {
        if (herm) k_ypass_fwd<B, 32, true><<<grid, threads, smem, st>>>(g, G1, P);
        else k_ypass_fwd<B, 32, false><<<grid, threads, smem, st>>>(g, G1, P);
    } else {
        if (herm) k_ypass_fwd<B, 16, true><<<grid, threads, smem, st>>>(g, G1, P);
        else k_ypass_fwd<B, 16, false><<<grid, threads, smem, st>>>(g, G1, P);
    }
}

template <int B>
void Launch<B>::interp_fin(int mode, dim3 grid, cudaStream_t st, const Geo &g, const float2 *P, float2 *f, double *part)
{
    if (mode == 0) k_interp_fin<0, B><<<grid, 256, 0, st>>>(g, P, f, part);
    else if (mode == 1) k_interp_fin<1, B><<<grid, 256, 0, st>>>(g, P, f, part);
    else k_interp_fin<2, B><<<grid, 256, 0, st>>>(g, P, f, part);
}

template <int B>
void Launch<B>::ypass_adj(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const float2 *f,
                          float2 *G1)
{
    // The band loop needs a full warp; tiny FFTs have fewer threads than that.
    bool guard = threads < 32;
    if (guard) threads = 32;
    if (E == 32) k_ypass_adj<B, 32, false><<<grid, threads, smem, st>>>(g, f, G1);
    else if (!guard) k_ypass_adj<B, 16, false><<<grid, threads, smem, st>>>(g, f, G1);
    else k_ypass_adj<B, 16, true><<<grid, threads, smem, st>>>(g, f, G1);
}

template <int B>
void Launch<B>::xpass_adj(int mode, int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                          const float2 *G1, float2 *out, const float2 *Ahwb, double *part)
{
    if (E == 32) {
        if (mode == 0) k_xpass_adj<0, B, 32><<<grid, threads, smem, st>>>(g, G1, out, Ahwb, part);
        else k_xpass_adj<1, B, 32><<<grid, threads, smem, st>>>(g, G1, out, Ahwb, part);
    } else {
        if (mode == 0) k_xpass_adj<0, B, 16><<<grid, threads, smem, st>>>(g, G1, out, Ahwb, part);
        else k_xpass_adj<1, B, 16><<<grid, threads, smem, st>>>(g, G1, out, Ahwb, part);
    }
}

template <int B>
void Launch<B>::rows_fwd(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const Geo1 &g1,
                         const float *rows, size_t sstride, size_t istride, int skip, int S, float2 *f,
                         float2 *bout)
{
    if (E == 32) k_rows_fwd<B, 32><<<grid, threads, smem, st>>>(g, g1, rows, sstride, istride, skip, S, f, bout);
    else k_rows_fwd<B, 16><<<grid, threads, smem, st>>>(g, g1, rows, sstride, istride, skip, S, f, bout);
}

template <int B>
void Launch<B>::img_out_file(dim3 grid, cudaStream_t st, const float *m, float *out, int S, int N0, int N1)
{
    k_img_out_file<B><<<grid, 256, 0, st>>>(m, out, S, N0, N1);
}

template <int B>
void Launch<B>::row_adj(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const Geo1 &g1,
                        const float2 *f, float *out, int S)
{
    if (E == 32) k_row_adj<B, 32><<<grid, threads, smem, st>>>(g, g1, f, out, S);
    else k_row_adj<B, 16><<<grid, threads, smem, st>>>(g, g1, f, out, S);
}

template <int B>
void Launch<B>::update(dim3 grid, cudaStream_t st, float *m, const float2 *rhat, const double *alpha, int per_group,
                       int clamp, int data_type, float thr, double *step_part)
{
    if (step_part) k_update<B, true><<<grid, 256, 0, st>>>(m, rhat, alpha, per_group, clamp, data_type, thr, step_part);
    else k_update<B, false><<<grid, 256, 0, st>>>(m, rhat, alpha, per_group, clamp, data_type, thr);
}

template <int B>
void Launch<B>::update_re(dim3 grid, cudaStream_t st, float *m, const float *rre, const double *alpha, int per_group,
                          int clamp, int data_type, float thr)
{
    k_update<B, false, float><<<grid, 256, 0, st>>>(m, rre, alpha, per_group, clamp, data_type, thr);
}

// The dynamic shared-memory limit is a property of the kernel function, not
// of a plan: plans of different sizes share the variants of one B, so every
// variant gets the device's opt-in maximum (what a launch actually asks for
// still sets the occupancy).  Lowering it to one plan's size would make a
// larger plan's next launch fail.
template <int B>
cudaError_t Launch<B>::set_smem(int ex, int ey, size_t, size_t, size_t, size_t, size_t)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    auto set = [&](const void *fn) {
        cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        if (r != cudaSuccess && e == cudaSuccess) e = r;
    };
    (void)ex;
    (void)ey;
    set((const void *)k_xpass_fwd<true, B, 32>);
    set((const void *)k_xpass_fwd<false, B, 32>);
    set((const void *)k_xpass_fwd_r2c<B, 32>);
    set((const void *)k_xpass_fwd_r2c<B, 32, true>);
    set((const void *)k_xpass_fwd<true, B, 32, true>);
    set((const void *)k_xpass_adj<0, B, 32>);
    set((const void *)k_xpass_adj<1, B, 32>);
    set((const void *)k_rows_fwd<B, 32>);
    set((const void *)k_row_adj<B, 32>);
    set((const void *)k_xpass_fwd<true, B, 16>);
    set((const void *)k_xpass_fwd<false, B, 16>);
    set((const void *)k_xpass_fwd_r2c<B, 16>);
    set((const void *)k_xpass_fwd_r2c<B, 16, true>);
    set((const void *)k_xpass_fwd<true, B, 16, true>);
    set((const void *)k_xpass_adj<0, B, 16>);
    set((const void *)k_xpass_adj<1, B, 16>);
    set((const void *)k_rows_fwd<B, 16>);
    set((const void *)k_row_adj<B, 16>);
    set((const void *)k_ypass_fwd<B, 32, false>);
    set((const void *)k_ypass_fwd<B, 32, true>);
    set((const void *)k_ypass_adj<B, 32, false>);
    set((const void *)k_ypass_toep<B, 32>);
    set((const void *)k_ypass_toep_quad<B, 32>);
    set((const void *)k_ypass_fwd<B, 16, false>);
    set((const void *)k_ypass_fwd<B, 16, true>);
    set((const void *)k_ypass_adj<B, 16, false>);
    set((const void *)k_ypass_adj<B, 16, true>);
    set((const void *)k_ypass_toep<B, 16>);
    set((const void *)k_ypass_toep_quad<B, 16>);
    set((const void *)k_ytoep4<B, 4, 0>);
    set((const void *)k_ytoep4<B, 6, 0>);
    set((const void *)k_ytoep4<B, 8, 0>);
    set((const void *)k_ytoep4<B, 10, 0>);
    set((const void *)k_ytoep4<B, 12, 0>);
    set((const void *)k_ytoep4<B, 16, 0>);
    set((const void *)k_ytoep4<B, 20, 0>);
    set((const void *)k_ytoep4<B, 24, 0>);
    set((const void *)k_ytoep4<B, 32, 0>);
    set((const void *)k_ytoep4<B, 4, 1>);
    set((const void *)k_ytoep4<B, 6, 1>);
    set((const void *)k_ytoep4<B, 8, 1>);
    set((const void *)k_ytoep4<B, 10, 1>);
    set((const void *)k_ytoep4<B, 12, 1>);
    set((const void *)k_ytoep4<B, 16, 1>);
    set((const void *)k_ytoep4<B, 20, 1>);
    set((const void *)k_ytoep4<B, 24, 1>);
    set((const void *)k_ytoep4<B, 32, 1>);
    return e;
}

template struct Launch<ICON_KB>;

}  // namespace icon
