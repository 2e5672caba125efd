/*
 * icon_b200.h -- C ABI of the B200 ICON reconstruction engine.
 *
 * Replaces the internal API of ICON-GPU v1.2.9 (hilbertsun/feilab,
 * tomography/ICON_GPU_v1.2.9/sourceCode/ICON-GPU; NU = nufft_gpu_v8.cu):
 * the reference's routines return void, take plan structs by value, run on
 * the default stream and handle one slice at a time.  Here every call
 * returns an icon_status, plans are opaque handles, work is queued on the
 * caller's stream, and every call processes a batch of S slices of one tilt
 * series (the slices share geometry, which is what makes batching pay).
 *
 * Data layout (all arrays are caller-owned unless stated otherwise):
 *   image   [S][N0][N1]   N0 = detector width nx, N1 = thickness, the
 *                         thickness index fastest -- the reference's device
 *                         layout of m, fhat and Ahwb (NU:763-771, :1111-1115)
 *   nodes   [S][M][2]     M = nx*ntilt complex values, node j = tilt*nx + k
 *                         (px2D.cu:29-47, readSlicePart.cu:21)
 *   rows    [S][ntilt][nx] projection rows: row y of every tilt, per slice y
 *                         (mrc_read_slice(..., 'y', ...), mrcfile3.c:902-951)
 * Pointers named d_* are device pointers on the plan's device; h_* are host
 * pointers.  `stream` is a cudaStream_t passed as void* (NULL = the legacy
 * default stream).  No call synchronises the device except where noted.
 *
 * Errors: a non-zero icon_status; icon_last_error() returns a message for the
 * calling thread.  Nothing here calls exit().
 * Threading: a plan may be used by one host thread at a time; different plans
 * are independent.
 */
#ifndef ICON_B200_H
#define ICON_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    ICON_OK = 0,
    ICON_ERR_INVALID = 1,   /* bad argument or unsupported size            */
    ICON_ERR_CUDA = 2,      /* a CUDA runtime call failed                  */
    ICON_ERR_NOMEM = 3,     /* device or host allocation failed            */
    ICON_ERR_CAPACITY = 4,  /* S larger than the plan's batch capacity     */
    ICON_ERR_IO = 5,        /* file could not be read or written           */
    ICON_ERR_TIMEOUT = 6    /* a bounded device-side wait ran out          */
} icon_status;

typedef struct icon_plan icon_plan;

/* Geometry of one tilt series.  Replaces the set-up of Lib_2D2
 * (MainCode.cu:12-109): .tlt angles, px2D nodes, Weight(), grid sizes
 * n_d = 2*nextpow2(N_d), the Gaussian window of half-width 6 and its
 * deapodisation, cunfft_initPlan_1d / cunfft_initPlan_2d2 (NU:445-556,
 * NU:1298-1391) and initGICONPara2 (NU:1739-1771). */
typedef struct {
    int nx;                  /* detector width, N0 (>= 8)                        */
    int thickness;           /* N1 (>= 8); 0 means nx, as MainCode.cu:14-16     */
    int ntilt;               /* number of tilts (>= 2)                            */
    const float *tilt_deg;   /* h_: angles as written in the .tlt file; they are
                                negated internally as MainCode.cu:42 does          */
    int capacity;            /* most slices any single call will pass            */
    int device;              /* CUDA device ordinal; -1 = the current device     */
    int window;              /* NUFFT window: ICON_WINDOW_GAUSS6 (0, the
                                reference's) or ICON_WINDOW_KB4                  */
} icon_geometry;

/* NUFFT windows.  ICON_WINDOW_GAUSS6 is the reference's Gaussian of
 * half-width m = 6 with 2m+2 = 14 taps per dimension (NU:221-235,
 * NU:471-476) and deapodisation exp(-b (pi k/n)^2) (NU:22-42): the parity
 * mode.  ICON_WINDOW_KB4 (no counterpart in the reference) is the
 * Kaiser-Bessel window of half-width K = 4 grid points, 8 taps per
 * dimension: phi(u) = sinh(kb sqrt(K^2 - u^2)) / (pi sqrt(K^2 - u^2)) for
 * |u| < K (u in grid units), kb = pi (2 - 1/theta), deapodisation
 * I0(K sqrt(kb^2 - (2 pi k/n)^2)), both scaled by 1/I0(kb K).  It
 * approximates the non-uniform DFT about four times more closely than the
 * Gaussian (1.5e-7 against 6.4e-7 relative in float at 64x40) and the
 * y-passes gather 8 x 8 instead of 14 x 14 taps per node.  The
 * iterations' Toeplitz operator has no window, so the window changes only
 * the NUFFT stages (input stage, reprojection, the NUFFT operator). */
#define ICON_WINDOW_GAUSS6 0
#define ICON_WINDOW_KB4 1

/* Iteration schedule and constraint of Iteration3 (Iteration2.cu:3-150):
 * `infr_before` unconstrained steps, `icon` clamped steps, `infr_after`
 * unconstrained steps (the -iter a,b,c flag of ICONGPU.cu:203-211).
 * data_type 1 clamps m <= threshold, 2 clamps m >= threshold
 * (ICONUpdateCU_R, NU:1597-1616). */
typedef struct {
    int infr_before;
    int icon;
    int infr_after;
    int data_type;
    float threshold;
} icon_solve_cfg;

/* icon_plan_create: builds the plan, its device tables and scratch for up to
 * geo->capacity slices.  Replaces cunfft_mallocPlan_2d2 + cunfft_initPlan_2d2
 * (NU:281-324, NU:445-556), cunfft_initPlan_1d (NU:1298-1391) and
 * initGICONPara2 (NU:1739-1771).  Synchronises the device. */
icon_status icon_plan_create(const icon_geometry *geo, icon_plan **out);

/* Frees a plan (cunfft_destroyPlan_2d2 NU:594-628, cunfft_destroyPlan_1d
 * NU:1393-1408, destroyGICONPara NU:1774-1787).  Synchronises the device. */
icon_status icon_plan_destroy(icon_plan *plan);

/* Angle (as in the .tlt file) at which icon_reconstruct_host reprojects. */
icon_status icon_plan_set_reprojection(icon_plan *plan, float tilt_deg);

/* dims[0..9] = N0, N1, n0, n1, M, ntilt, slices per group B, capacity,
 * device bytes held by the plan (low 31 bits in MiB), tilt index of the
 * smallest |angle| (the reprojection tilt of MainCode.cu:46-49). */
icon_status icon_plan_query(const icon_plan *plan, int *dims);

/* h_w[M] <- density weights, h_xy[2M] <- node coordinates (x0, x1), exactly
 * as Weight() and px2D() compute them (weight.cu:8-41, px2D.cu:8-47).
 * Either pointer may be NULL. */
icon_status icon_plan_geometry(const icon_plan *plan, float *h_xy, float *h_w);

/* h_w[ntilt*nx] <- the density weights of a tilt series given as in the
 * .tlt file, as Weight() computes them for the plan's nodes
 * (weight.cu:8-41); tilt i's nodes are h_w[i*nx .. i*nx+nx-1]. */
icon_status icon_weights(int nx, int ntilt, const float *tilt_deg, float *h_w);

/* Per-group density weights: slice group g of every later call (slices
 * g*B .. g*B+B-1, B = icon_plan_query dims[6]) uses h_w[g][M] in place of
 * the plan's own weights, for g < ngroups (<= capacity / B rounded up); the
 * other groups keep the plan's.  ngroups = 0 restores the plan's weights
 * for all.  A node of weight 0 drops out of the data term: with one tilt's
 * nodes at 0 and the others weighted as icon_weights gives for the series
 * without it, a group solves that series (the left-out solves of
 * icon_loo_sweep, all tilts in one batched schedule).  Copies h_w to the
 * device (synchronous).  No counterpart in the reference, whose plans hold
 * one weight vector. */
icon_status icon_plan_set_group_weights(icon_plan *plan, const float *h_w, int ngroups);

/* Normal operator of the iterations of icon_solve, icon_solve_until and the
 * reconstruct calls.  ICON_OPERATOR_NUFFT (the default) evaluates
 * A^H W A m and the step length's w-weighted |A r|^2 with the Gaussian-window
 * NUFFT pair, as Iteration3 does (Iteration2.cu:53-96, alpha_new2.cu:26-114).
 * ICON_OPERATOR_TOEPLITZ uses that A^H W A is a Toeplitz operator: A^H W A m
 * = crop F^-1(K . F(pad m)) on the n0 x n1 grid, and sum_j w_j |(A r)_j|^2 =
 * sum_k K[k] |F(pad r)[k]|^2, with the real kernel
 * K[k] = 1/(n0 n1) sum_j w_j D_N0(x_j0 - k0/n0) D_N1(x_j1 - k1/n1),
 * D_N(u) = sin(pi u (2N-1)) / sin(pi u), computed on the device in double
 * when first needed (and again after the weights change).  It is the exact
 * operator of the node set, without the NUFFT window's approximation (the two
 * differ by ~1e-6 relative per application), and needs no interpolation or
 * gather.  The input stage (A^H W b) and reprojection use the NUFFT either
 * way.  No counterpart in the reference. */
#define ICON_OPERATOR_NUFFT 0
#define ICON_OPERATOR_TOEPLITZ 1
icon_status icon_plan_set_operator(icon_plan *plan, int op);

/* Tolerance stop of the reconstruct calls (icon_reconstruct_host,
 * icon_reconstruct_stack, icon_reconstruct_stack_host): with tol > 0 their
 * ICON phase ends, per batch, once every slice's relative step
 * ||m_new - m_old|| / ||m_new|| is at or below tol, checked every
 * check_every ICON iterations, as icon_solve_until does; tol = 0 (the
 * default) runs the whole schedule, as the reference always does
 * (Iteration2.cu:42-146).  No counterpart in the reference. */
icon_status icon_plan_set_stop(icon_plan *plan, double tol, int check_every);

/* Forward 2-D NUFFT of real images: d_nodes = A d_img.
 * Replaces cunfft_trafo_2d_R2C2 (NU:984-1076). */
icon_status icon_nufft_forward(icon_plan *plan, const float *d_img, void *d_nodes, int S, void *stream);

/* Forward 2-D NUFFT of complex images (cunfft_trafo_2d2, NU:844-949). */
icon_status icon_nufft_forward_complex(icon_plan *plan, const void *d_img, void *d_nodes, int S, void *stream);

/* Adjoint 2-D NUFFT: d_img (complex) = A^H d_nodes.
 * Replaces cunfft_adjoint_2d2 (NU:1167-1238). */
icon_status icon_nufft_adjoint(icon_plan *plan, const void *d_nodes, void *d_img, int S, void *stream);

/* 1-D NUFFT of every projection row: d_b[S][M] complex.
 * Replaces readSlicePart (readSlicePart.cu:3-31) with cunfft_trafo_1d
 * (NU:1479-1516) per row. */
icon_status icon_rows_forward(icon_plan *plan, const float *d_rows, void *d_b, int S, void *stream);

/* Right-hand side A^H W b from projection rows: the input stage of the
 * slice loop of Lib_2D2 (MainCode.cu:115-134: readSlicePart,
 * complexMulDoubleCU, cunfft_adjoint_2d2, complexCopyCU). */
icon_status icon_prepare_rhs(icon_plan *plan, const float *d_rows, void *d_Ahwb, int S, void *stream);

/* icon_prepare_rhs reading the rows straight from a device-resident tilt
 * stack in file order, d_stack[sections][ny][nx] (MRC sections = tilts,
 * y = slice): the rows of slices y0 .. y0+S-1.  With skip_section < 0 the
 * plan's tilt i reads section i; otherwise the stack has one section more
 * than the plan has tilts, section skip_section is left out and tilt i reads
 * section i + (i >= skip_section) -- the cross-validation input of
 * readSlicePart_crossV (readSlicePart_crossV.cu:3-34).  Replaces the per-row
 * file reads of readSlicePart (readSlicePart.cu:3-31 over mrc_read_slice,
 * mrcfile3.c:902-951, one fread per pixel) with one upload of the stack. */
icon_status icon_prepare_rhs_stack(icon_plan *plan, const float *d_stack, int ny, int y0, int skip_section,
                                   void *d_Ahwb, int S, void *stream);

/* The per-slice pipeline of Lib_2D2 (MainCode.cu:113-142) on the device,
 * from a tilt stack as in icon_prepare_rhs_stack to outputs in file layout:
 * d_slices[S][N1][N0] with X fastest, the order saveMRC_real_inv writes a
 * slice in (saveMRC_real.cu:49-53), and, when d_reproj is not NULL,
 * d_reproj[S][nx], the reprojection at the plan's reprojection angle
 * (icon_plan_set_reprojection).  The schedule starts from m = 0.  S may
 * exceed the capacity (processed in chunks).  Asynchronous on `stream`. */
icon_status icon_reconstruct_stack(icon_plan *plan, const icon_solve_cfg *cfg, const float *d_stack, int ny, int y0,
                                   int skip_section, float *d_slices, float *d_reproj, int S, void *stream);

/* icon_reconstruct_stack with the results streamed to host memory: slices
 * y0 .. y0+S-1 in batches of the plan's capacity; each batch's outputs are
 * copied into one of two pinned host buffers and handed to `sink` while the
 * next batch runs on the GPU (the reference writes each slice's file after
 * its solve, MainCode.cu:142-160, with the GPU idle meanwhile).  The sink
 * receives the batch's first slice index (relative to y0), its slice count
 * and the host arrays h_slices[count][N1][N0] (X fastest) and
 * h_reproj[count][nx] -- NULL unless requested in `outputs` -- which stay
 * valid until it returns; a nonzero return stops the run with an error.
 * The sink runs on the calling thread.  Returns after the last batch's sink. */
#define ICON_OUT_SLICES 1
#define ICON_OUT_REPROJECTION 2
typedef int (*icon_batch_sink)(void *ctx, int s0, int count, const float *h_slices, const float *h_reproj);
icon_status icon_reconstruct_stack_host(icon_plan *plan, const icon_solve_cfg *cfg, const float *d_stack, int ny,
                                        int y0, int skip_section, int S, int outputs, icon_batch_sink sink, void *ctx,
                                        void *stream);

/* Pinned (page-locked, portable) host memory for a stack read from a file,
 * so that icon_stack_upload copies at full speed, and its release. */
icon_status icon_host_alloc(size_t bytes, void **out);
icon_status icon_host_free(void *h_ptr);

/* One upload of the rows y0 .. y0+S-1 of every section of a host tilt stack
 * h_stack[sections][ny][nx] (file order) to new device memory on `device`,
 * packed as d_stack[sections][S][nx] (so ny = S, y0 = 0 in the stack calls).
 * A single 2-D copy; synchronises `stream`.  Free with icon_device_free. */
icon_status icon_stack_upload(int device, const float *h_stack, int sections, int ny, int nx, int y0, int S,
                              float **d_stack, void *stream);
icon_status icon_device_free(int device, void *d_ptr);

/* ICON iterations on S slices: replaces Iteration3 (Iteration2.cu:3-150)
 * with Alpha2 (alpha_new2.cu:3-119).  d_m is the start value when
 * warm_start != 0 and is zeroed first otherwise (Iteration2.cu:33); it
 * receives the result.  h_alpha and h_rtr, when not NULL, receive the step
 * length alpha and ||rhat||^2 of every iteration and slice, [iters][S]
 * (this synchronises the stream at the end). */
icon_status icon_solve(icon_plan *plan, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S,
                       int warm_start, double *h_alpha, double *h_rtr, void *stream);

/* icon_solve whose ICON phase stops at a tolerance.  The schedule is the
 * reference's (INFR for infr_before iterations, ICON with the threshold
 * clamp for at most `icon`, INFR for infr_after; Iteration2.cu:129-132),
 * but every check_every ICON iterations (and at the phase's last) the size
 * of that iteration's update relative to the new image,
 * ||m_new - m_old|| / ||m_new|| (summed in double), is read for every slice,
 * and the ICON phase ends once all slices are at or below tol; the final
 * INFR iterations then run as usual.  For the clamped iteration this step,
 * not ||rhat||, goes to zero at a fixed point.  tol = 0 runs the whole
 * schedule (the result is icon_solve's).  *h_iters receives the iterations
 * done and h_step[S] (optional) each slice's relative step at the last
 * check.  Synchronises the stream at every check.  The reference has no
 * such stop: it always runs the full count. */
icon_status icon_solve_until(icon_plan *plan, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S,
                             int warm_start, double tol, int check_every, int *h_iters, double *h_step, void *stream);

/* Acceptance test of a warm-started solve (icon_solve_warm). */
typedef struct {
    double tol;          /* relative-step tolerance of the ICON phase (> 0), as icon_solve_until */
    int check_every;     /* ICON iterations between checks (>= 1)                               */
    double max_dist;     /* largest accepted ||m - m_infr|| / ||m_infr|| (> 0), m_infr the cold
                            start's iterate after the first INFR phase; the cold result itself
                            lies 1.0-1.3 from it on synthetic series (the clamped ICON phase adds
                            the missing-wedge content), so 2 is a working bound                  */
} icon_warm_cfg;

/* Reasons icon_solve_warm redid a slice from m = 0 (h_redone[s]). */
#define ICON_WARM_ACCEPTED 0
#define ICON_WARM_NOT_FINITE 1      /* the warm result holds a NaN or an infinity       */
#define ICON_WARM_NOT_CONVERGED 2   /* its relative step stayed above tol               */
#define ICON_WARM_TOO_FAR 3         /* farther than max_dist from the cold INFR iterate */

/* Warm-started solve with the plain cold-start solve as fallback.  d_m
 * [S][N0][N1] holds each slice's start on entry (e.g. icon_ws_predict's
 * output) and its result on return.  The schedule runs from those starts
 * with the ICON phase stopped at wc->tol (icon_solve_until).  The cold
 * start's first INFR phase (cfg->infr_before iterations from m = 0, a few
 * percent of the schedule) gives m_infr.  A slice is accepted when its
 * result is finite, its last relative step is at most tol, and
 * ||m - m_infr|| <= max_dist ||m_infr||; every other slice is solved again
 * from m = 0 with the full schedule (icon_solve with warm_start = 0) and its
 * result replaced by that cold one, which is bit for bit what icon_solve
 * gives for the slice (slices do not interact).  h_redone[S] (optional)
 * receives ICON_WARM_* per slice, *h_iters (optional) the iterations of the
 * warm solve.  Allocates device scratch for the slices it redoes;
 * synchronises the stream.  The redone slices run as slices 0.. of a new
 * batch, so a plan with per-group weights (icon_plan_set_group_weights)
 * would solve them with other groups' weights: use one without.  No counterpart in the reference, which always
 * starts from m = 0 (Iteration2.cu:33). */
icon_status icon_solve_warm(icon_plan *plan, const icon_solve_cfg *cfg, const void *d_Ahwb, float *d_m, int S,
                            const icon_warm_cfg *wc, int *h_redone, int *h_iters, void *stream);

/* Reprojection of S solved slices at one tilt angle (given as in the .tlt
 * file): forward 2-D NUFFT at the nodes of that single tilt, then the 1-D
 * adjoint NUFFT, real part (reProject_NFFT2, reProject_NFFT.cu:25-42, with
 * cunfft_adjoint_1d NU:1518-1536).  d_out[S][nx]. */
icon_status icon_reproject(icon_plan *plan, const float *d_m, float tilt_deg, float *d_out, int S, void *stream);

/* icon_reproject from and to host memory: h_m [S][N0][N1] (Y fastest),
 * h_out [S][nx]; S may exceed the capacity (processed in chunks through the
 * plan's buffers).  Returns when h_out is filled.  Used by icon-gpu --resume
 * for slices whose files a previous run wrote (the reference recomputes
 * every slice, MainCode.cu:113-162). */
icon_status icon_reproject_host(icon_plan *plan, const float *h_m, float tilt_deg, float *h_out, int S, void *stream);

/* The whole per-slice pipeline of Lib_2D2 (MainCode.cu:113-142) for S
 * slices from host memory: rows in, reconstructed slices out, plus the
 * reprojection when h_reproj is not NULL -- at the smallest-|angle| tilt of
 * the plan (MainCode.cu:46-49, :142) unless icon_plan_set_reprojection chose
 * another angle (the cross-validation solve of MainCode_crossV.cu:153
 * reprojects at the tilt it left out).
 * Host buffers should be pinned for full copy speed.  Work is queued on
 * `stream` (NULL: a stream of its own); the call returns after the results
 * are in host memory.  S may exceed the capacity: it is processed in chunks. */
icon_status icon_reconstruct_host(icon_plan *plan, const icon_solve_cfg *cfg, const float *h_rows, float *h_m,
                                  float *h_reproj, int S, void *stream);

/* Kernel tracing (no reference counterpart; the reference's cudaEvent timing
 * blocks are commented out, e.g. Iteration2.cu:36-40).  While enabled, every
 * kernel launch of the solver is bracketed by CUDA events on its stream.
 * icon_trace_read synchronises, and for each of the ICON_TRACE_KERNELS kernel
 * kinds returns the number of launches, their summed device time in ms and,
 * when h_bytes is not NULL, their summed algorithmic bytes (the data each
 * launch must read and write at least once), then clears the record.  Kinds, in order: xpass_fwd, ypass_fwd, interp_fin,
 * ypass_adj, xpass_adj, alpha, update, rows_fwd, layout, row_adj, ypass_toep, ypass_toep_quad,
 * xtoep_fwd (the Toeplitz forward x-pass of m, with the previous iteration's
 * update), xtoep_mid (the Toeplitz inverse x-pass, r-hat and forward x-pass
 * of r-hat in one kernel). */
#define ICON_TRACE_KERNELS 14
icon_status icon_trace_enable(icon_plan *plan, int enable);
icon_status icon_trace_read(icon_plan *plan, int *h_count, double *h_ms, double *h_bytes);

/* Number of kernels this plan has launched since it was created. */
long long icon_launch_count(const icon_plan *plan);

/* Reads and clears the plan's device error flag: 0, or 1 when a bounded wait
 * of the x-kernels for their TMA column loads ran out (the kernel then
 * skipped its output, so results since the last read are not valid).
 * Synchronises the device.  No counterpart in the reference. */
icon_status icon_plan_device_error(icon_plan *plan, int *h_code);

/* icon_rows_forward_noalloc: the work of icon_rows_forward (the 1-D NUFFT of
 * every projection row, d_b[S][ntilt*nx] complex) for callers that cannot
 * allocate device memory -- a process whose own pool allocator owns all
 * device memory, or a real-time loop that must not call cudaMalloc because it
 * can block on the device -- and so cannot create a plan.  No counterpart in
 * the reference.  It calls no cudaMalloc, cudaFree or allocating library
 * routine: its tables live in one file-scope __device__ array of
 * ICON_NOALLOC_SCRATCH_BYTES, part of this library's device code.  That code
 * is loaded on a device, the array with it, at the first use of the library
 * there under lazy module loading (the CUDA default since 12.2; with
 * CUDA_MODULE_LOADING=EAGER, at context creation), and the load allocates
 * device memory and may synchronise: make the first call on each device
 * before a pool allocator takes its memory, before any real-time region and
 * before any stream capture.  The array then stays until the process exits;
 * later calls allocate nothing.  Every call looks up the array's device
 * address and sets the row kernel's shared-memory limit (cheap host calls).
 * nx must be in [8, ICON_NOALLOC_MAX_NX] (larger sizes return
 * ICON_ERR_INVALID).  Runs on the current device and on `stream`.  All calls
 * share the array: calls that overlap on one GPU (other streams or host
 * threads) race on it and must be serialised by the caller. */
#define ICON_NOALLOC_MAX_NX 4096
#define ICON_NOALLOC_SCRATCH_BYTES (512 * 1024)
icon_status icon_rows_forward_noalloc(const float *d_rows, int nx, int ntilt, int S, void *d_b, void *stream);

/* Message for the last failed call on this thread ("" if none). */
const char *icon_last_error(void);

/* Number of CUDA devices and, for the first `max` of them, their
 * multiprocessor counts (h_sm may be NULL).  The reference queries the same to
 * split slices across GPUs in proportion to SM count (ICONGPU.cu:153-160,
 * :398-430). */
icon_status icon_devices(int *h_count, int *h_sm, int max);

#ifdef __cplusplus
}
#endif
#endif
