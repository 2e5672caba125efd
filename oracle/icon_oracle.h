/*
 * icon_oracle.h -- CPU restatement of the ICON-GPU v1.2.9 reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * feilab_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it; the product never links or calls it.
 *
 * Every routine follows a reference routine and cites it (paths are relative to
 * tomography/ICON_GPU_v1.2.9/sourceCode/ICON-GPU/ in hilbertsun/feilab;
 * NU = nufft_gpu_v8.cu).  The core is compiled twice: once with REAL=double
 * (suffix _f64, the FP64 oracle) and once with REAL=float (suffix _f32, which
 * repeats the reference's float rounding step by step except inside the FFT,
 * where the reference calls cuFFT).
 *
 * Parity pin: the reference ships no test vectors.  The oracle is pinned
 * (a) by known-answer tests against a direct NDFT computed here in double,
 * (b) by the adjoint identity <A x, y> = <x, A^H y>, and
 * (c) against outputs of the reference itself (its own cunfft_* and
 *     Iteration3 routines compiled from the reference sources by
 *     oracle/build_ref.sh and run on a B200), committed as fixtures under
 *     tests/golden/.
 */
#ifndef ICON_ORACLE_H
#define ICON_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Window half-width of the reference (nufft_gpu_v8.cuh:5, NFFTM). */
#define ORA_M 6
/* Taps per dimension, 2m+2 (NU:226). */
#define ORA_T 14
/* Window kinds: the reference's Gaussian of half-width 6, and a Kaiser-Bessel
 * window of half-width 4 (no counterpart in the reference) laid out in the
 * same 14 taps, non-zero on taps 3..10 only. */
#define ORA_WINDOW_GAUSS6 0
#define ORA_WINDOW_KB4 1
#define ORA_KB_M 4

/* Grid parameters for one dimension of size N: theta = 2*2^ceil(log2 N)/N as
 * float, n = ceil(theta*N), window b and bf (MainCode.cu:66-71, NU:471-476). */
void ora_grid_params(int N, float *theta, int *n, float *b, float *bf);

/* Node coordinates of px2D (px2D.cu:8-47): nz lines of nx nodes, interleaved
 * (x0, x1) per node; theta_neg are the already negated tilt angles. */
void ora_px2d(int nx, int nz, const float *theta_neg, float *xy);

/* Density weights of Weight() (weight.cu:8-41). */
void ora_weight(int nx, int nz, const float *theta_neg, float *w);

#ifdef __cplusplus
}
#endif
#endif
