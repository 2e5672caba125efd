// icon_launch.h -- host launchers of the batched FFT kernels, one explicit
// instantiation per slice-group size B (icon_kern_b.cu is compiled once per B
// so that the kernel variants build in parallel).
#pragma once
#include <cuda_runtime.h>

namespace icon {

struct Geo;
struct Geo1;
struct XtArgs;

template <int B>
struct Launch {
    static void xpass_fwd(bool real_in, int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                          const void *in, float2 *G1);
    // Forward x-pass of a real image with every row written (half-length FFT;
    // rows past n0/2 as conjugates), for the Toeplitz y-pass.
    static void xpass_fwd_full(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                               const float *in, float2 *G1);
    // Toeplitz y-passes: A^H W A on the rows of G1 in place, and the step
    // length's quadratic form into part[G][n0][B].
    static void ypass_toep(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, float2 *G1);
    static void ypass_toep_quad(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                                const float2 *G1, double *part);
    static void ypass_fwd(int E, bool herm, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const float2 *G1,
                          float2 *P);
    static void interp_fin(int mode, dim3 grid, cudaStream_t st, const Geo &g, const float2 *P, float2 *f, double *part);
    static void ypass_adj(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const float2 *f,
                          float2 *G1);
    static void xpass_adj(int mode, int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g,
                          const float2 *G1, float2 *out, const float2 *Ahwb, double *part);
    static void rows_fwd(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const Geo1 &g1,
                         const float *rows, size_t sstride, size_t istride, int skip, int S, float2 *f,
                         float2 *bout);
    static void img_out_file(dim3 grid, cudaStream_t st, const float *m, float *out, int S, int N0, int N1);
    static void row_adj(int E, dim3 grid, int threads, size_t smem, cudaStream_t st, const Geo &g, const Geo1 &g1,
                        const float2 *f, float *out, int S);
    static void update(dim3 grid, cudaStream_t st, float *m, const float2 *rhat, const double *alpha, int per_group,
                       int clamp, int data_type, float thr, double *step_part = nullptr);
    // The same from the real part of r-hat alone (the Toeplitz x-kernels' output).
    static void update_re(dim3 grid, cudaStream_t st, float *m, const float *rre, const double *alpha, int per_group,
                          int clamp, int data_type, float thr);
    // Three-step x-passes (k_xtoep) over G groups: mode 0 the Toeplitz forward
    // of the real image (with the fused update when a.upd), mode 1 the
    // Toeplitz inverse, r-hat and forward of r-hat, mode 2 the NUFFT adjoint's
    // x-pass (deapodised, optionally minus Ahwb with |.|^2 sums).  Returns
    // false when n0 has no variant (the caller then uses the Stockham kernels).
    static bool xtoep(int mode, cudaStream_t st, int G, const XtArgs &a);
    // Raises the shared-memory limit of the k_xtoep variants for n0.
    static cudaError_t xtoep_prepare(int n0);
    // Raises the dynamic shared-memory limit of every kernel variant a plan uses.
    static cudaError_t set_smem(int ex, int ey, size_t smem_x, size_t need_x, size_t smem_y, size_t smem_ya,
                                size_t smem_yt);
};

}  // namespace icon
