/* icon_tools.h -- the steps either side of the ICON solve that the
 * reference does in companion tools, on the GPU.
 *
 * All device pointers are caller-owned; stream arguments are cudaStream_t
 * passed as void *.  Functions return icon_status (icon_b200.h) and leave a
 * message for icon_last_error() on failure.
 */
#ifndef ICON_TOOLS_H
#define ICON_TOOLS_H

#include "icon_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Tilt-stack pre-processing: replaces ICONPreProcess
 * (sourceCode/ICONPreProcess/ICONPreProcess.c:29-85, 216-300).  d_in and
 * d_out are [nz][ny][nx] float (may be the same array; nz <= 1024).  Every
 * projection has the mode of a 256-bin histogram of its central 80 %
 * subtracted; when h_tilt_deg (nz angles, host memory) is not NULL and
 * thickness > 0, each is then scaled to variance 0.33 * thickness /
 * cos(tilt).  Needs no device memory of its own. */
icon_status icon_preprocess(const float *d_in, float *d_out, int nx, int ny, int nz, const float *h_tilt_deg,
                            int thickness, void *stream);

/* The same on a stack in host memory (h_in may equal h_out); allocates and
 * frees device memory for the stack and synchronises. */
icon_status icon_preprocess_host(const float *h_in, float *h_out, int nx, int ny, int nz, const float *h_tilt_deg,
                                 int thickness);

/* Volume assembly with the cross-validation mask: replaces ICONMask3
 * (sourceCode/ICONMask3/ICONCrossVMaskIn2D_weightOnlyOnSampled.cu, MK).
 *
 * icon_mask_radius: the mask radius as rates of n/2, from the
 * cross-validation and full-reconstruction FRC curves (frc_len values each,
 * the second column of crossV.frc / fullRec.frc) when radius < 0 -- the last
 * frequencies where crossV/fullRec >= 0.5 and >= 0.3 (MK:1033-1100) -- or
 * from an explicit radius in pixels; invalid curves fall back to the radius
 * the tilt span fills (MK:996-1005), as the reference does.  *explicit_radius
 * tells the filter which rule set its Gaussian width (MK:391-411). */
icon_status icon_mask_radius(int n, const float *tilts, int ntilt, int radius, const float *crossv,
                             const float *fullrec, int frc_len, float *rate05, float *rate03, int *explicit_radius);

/* Filter for n x n slices (n a power of two, 16..8192): the sampling mask of
 * the tilts (MK:1107-1139), 1 inside the radius, a Gaussian roll-off of
 * gauss_width pixels (<= 0: the reference's default) blended with the mask
 * beyond, times rr / r_full on sampled frequencies (MK:369-468); work space
 * for `capacity` slices per call on the current device. */
typedef struct icon_mask icon_mask;
icon_status icon_mask_create(int n, const float *tilts, int ntilt, float rate05, float rate03, int explicit_radius,
                             int gauss_width, int capacity, icon_mask **out);
icon_status icon_mask_destroy(icon_mask *mask);

/* The filter on the half spectrum, [n][n/2+1] floats, into host memory. */
icon_status icon_mask_filter(const icon_mask *mask, float *h_filter);

/* d_slices [S][n][n] (rows along the thickness) -> d_out [S][thickness][n]:
 * each slice filtered (R2C, times the filter, C2R, / n^2; MK:479-600) and
 * rows ystart .. ystart+thickness-1 kept (ystart = n/2 - thickness/2 +
 * zshift in ICONMask3, MK:1162). */
icon_status icon_mask_apply(icon_mask *mask, const float *d_slices, int S, int ystart, int thickness, float *d_out,
                            void *stream);

/* The same on slices in host memory, in batches of the filter's capacity;
 * allocates and frees device memory and synchronises. */
icon_status icon_mask_apply_host(icon_mask *mask, const float *h_slices, int S, int ystart, int thickness,
                                 float *h_out);

/* Assembly without the mask (ICONMask3 -noMask 1, MK:43-368): rows
 * ystart .. ystart+thickness-1 of every n x n slice. */
icon_status icon_volume_crop(const float *d_slices, int n, int S, int ystart, int thickness, float *d_out,
                             void *stream);

/* Fourier ring correlation of two nx-by-ny images (host memory, nx fastest)
 * as the reference's cross validation computes it: calFRC_nonsqure
 * (calFRC.cu:93-174; rings with the y frequency scaled by (nx/ny)^2,
 * frc[0] = 1) and, with smooth_overlap > 0, frcSmooth (ICONGPU.cu:59-91).
 * frc_out receives nx/2 values.  Host computation in double. */
icon_status icon_frc(const float *a, const float *b, int nx, int ny, int smooth_overlap, float *frc_out);

/* Leave-one-out cross validation over every tilt.  The reference validates
 * one tilt (the smallest |angle|): Lib_2D_crossV2 (MainCode_crossV.cu:3-189)
 * reconstructs without it, reprojects at its angle and compares with the
 * omitted projection by FRC.  This call does that for each of the nz tilts
 * in turn: h_rows [S][nz][nx] (host; rows of every tilt per slice),
 * thickness, tilt_deg[nz], the solve schedule cfg, on `device`.  All nz*S
 * left-out solves run as one batched schedule on one plan over all tilts of
 * `capacity` slots: each slice group is (omitted tilt, B slices) with that
 * tilt's nodes weighted 0 and the rest weighted for the series without it
 * (icon_plan_set_group_weights), which solves the reduced series.  tol > 0
 * ends each batch's ICON phase at that relative step (icon_solve_until);
 * tol = 0 is the reference's solve for every tilt.
 * Solves start from m = 0: a start holding the omitted projection (the
 * reconstruction from all tilts, say) would leak it into the validation.
 * h_frc [nz][nx/2] receives the
 * smoothed FRC of each omitted tilt; h_reproj [nz][S][nx] (optional) the
 * reprojections; h_iters[nz] (optional) the iterations of each tilt's
 * longest batch.  op is the iterations' normal operator
 * (ICON_OPERATOR_NUFFT or ICON_OPERATOR_TOEPLITZ, icon_plan_set_operator);
 * with the Toeplitz operator the groups of a batch that leave out the same
 * tilt share one kernel.  Synchronous. */
icon_status icon_loo_sweep(const float *h_rows, int nx, int thickness, int nz, const float *tilt_deg,
                           const icon_solve_cfg *cfg, int S, int capacity, double tol, int device, float *h_frc,
                           float *h_reproj, int *h_iters, int op);

#ifdef __cplusplus
}
#endif

#endif /* ICON_TOOLS_H */
