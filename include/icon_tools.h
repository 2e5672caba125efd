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

#ifdef __cplusplus
}
#endif

#endif /* ICON_TOOLS_H */
