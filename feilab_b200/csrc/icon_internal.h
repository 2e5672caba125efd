// icon_internal.h -- C++ hooks of icon_api.cu for the other translation
// units of the library (not part of the C ABI).  They drive one plan's
// pipeline in pieces, so that icon_batch.cu can capture the iterations of
// many plans into CUDA graphs.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "icon_b200.h"
#include "icon_warmstart.h"

namespace iconx {

// icon_plan_create with a given number of slices per group (1, 2, 4 or 8,
// capped at the size's default; 0 = the default).
icon_status plan_create_group(const icon_geometry *geo, int group, icon_plan **out);
int plan_group(const icon_plan *p);
int plan_capacity(const icon_plan *p);
int plan_device(const icon_plan *p);
// Device buffers of the plan: rows [capacity][ntilt][nx], images
// [capacity][N0][N1].
float *plan_rows_buffer(icon_plan *p);
float *plan_out_buffer(icon_plan *p);

// Input stage of S slices whose rows are at d_rows (device, [S][ntilt][nx]):
// the row transform, A^H W b and m = 0 (MainCode.cu:115-134); also computes
// the Toeplitz kernel if the plan uses it and it is stale.
icon_status plan_stage_in(icon_plan *p, const float *d_rows, int S, cudaStream_t st);
// Iteration `it` of cfg's schedule (Iteration2.cu:42-146) for S slices.
// Touches no host-side state: it may be captured into a CUDA graph, and a
// replay does what a direct call does.  With the Toeplitz operator and the
// three-step x-kernels the update of iteration it - 1 is applied inside
// iteration it (plan_stage_out applies the last one).
icon_status plan_iteration(icon_plan *p, int S, int it, const icon_solve_cfg *cfg, cudaStream_t st);
// After the last iteration: any deferred update, then m as [S][N0][N1]
// (Y fastest) into d_out.
icon_status plan_stage_out(icon_plan *p, int S, const icon_solve_cfg *cfg, float *d_out, cudaStream_t st);

// Slices a warm-start network takes per call (icon_ws_create's capacity).
int ws_capacity(const icon_ws *w);

// Sets icon_last_error() and returns st.
icon_status fail_msg(icon_status st, const std::string &msg);

}  // namespace iconx
