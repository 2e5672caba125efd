/* icon_warmstart.h -- learned warm start for the ICON solve.
 *
 * The reference (ICON-GPU v1.2.9) starts every solve from m = 0
 * (cudaMemset of m before the loop, IG/Iteration2.cu:33).  This library adds
 * a start predicted by a small U-Net from the slice's back-projection
 * Re(A^H W b): 4 levels of 16/32/64/128 channels, 3x3 convolutions with ReLU,
 * 2x2 average pooling, nearest upsampling and skip connections, BF16
 * activations and weights with FP32 accumulation on the sm_100a tensor cores
 * (tcgen05.mma fed by TMA).  None of this has a reference counterpart; the
 * solve that follows is the reference's algorithm unchanged (icon_solve with
 * warm_start = 1).
 *
 * All device pointers are caller-owned; stream arguments are cudaStream_t
 * passed as void *.  Functions return icon_status (icon_b200.h) and leave a
 * message for icon_last_error() on failure.
 */
#ifndef ICON_WARMSTART_H
#define ICON_WARMSTART_H

#include <stddef.h>

#include "icon_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One 3x3 convolution (stride 1, zero padding 1) on the tensor cores, the
 * building block of the network, exported for tests and other callers.
 * in0 [nimg][H][W][cin0] and, when in1 is not NULL, in1 [nimg][H][W][cin1]
 * are BF16 NHWC tensors read as one input of cin0 + cin1 channels (each a
 * multiple of 16).  w: BF16 [9][N][cin0 + cin1] with tap = 3*dy + dx;
 * bias: FP32 [N] or NULL; relu: 0 or 1.  Output channels [0, nsplit) go to
 * out0 [nimg][H][W][nsplit] and [nsplit, N) to out1 [nimg][H][W][N - nsplit];
 * acc0 / acc1 = 1 add to the output's values instead of overwriting them.
 * N and nsplit are multiples of 16, N <= 256. */
icon_status icon_ws_conv3x3(const void *in0, int cin0, const void *in1, int cin1, int nimg, int H, int W,
                            const void *w, const float *bias, int N, int relu, void *out0, int nsplit, int acc0,
                            void *out1, int acc1, void *stream);

/* The network.  Slices are in the layout of icon_prepare_rhs / icon_solve:
 * Ahwb [S][N0][N1] complex (pairs of float), m [S][N0][N1] float, Y
 * fastest.  The network image of a slice is Re(Ahwb) as N1 rows of N0
 * pixels, padded to multiples of 8 and divided by its RMS; its output times
 * the same RMS and a fixed gain is the predicted start.  Parameters are FP32
 * masters (BF16 copies feed the tensor cores); training uses Adam (beta
 * 0.9 / 0.999, eps 1e-8) on the mean squared error over the valid pixels in
 * network units. */
typedef struct icon_ws icon_ws;

/* Network for the geometry (N0, N1) of `plan`, on the current device, for
 * up to `capacity` slices per call (at most the plan's capacity). */
icon_status icon_ws_create(icon_plan *plan, int capacity, icon_ws **out);
icon_status icon_ws_destroy(icon_ws *ws);

/* Number of FP32 parameters. */
size_t icon_ws_param_count(void);

/* He-normal initialisation from a seed; resets the optimiser. */
icon_status icon_ws_init(icon_ws *ws, unsigned long long seed);

/* Copies all parameters and the output gain (> 0) in or out. */
icon_status icon_ws_set_params(icon_ws *ws, const float *h_params, size_t count, float gain);
icon_status icon_ws_get_params(icon_ws *ws, float *h_params, size_t count, float *h_gain);
icon_status icon_ws_set_gain(icon_ws *ws, float gain);

/* m0 [S][N0][N1] = network(Ahwb): the warm start for icon_solve. */
icon_status icon_ws_predict(icon_ws *ws, const void *d_Ahwb, float *d_m0, int S, void *stream);

/* Forward pass, mean squared error against d_target [S][N0][N1] (both in
 * network units: divided by RMS * gain), and the gradients of every
 * parameter, kept in the network (icon_ws_get_grads copies them out).
 * *h_loss (optional; synchronises) receives the loss. */
icon_status icon_ws_backprop(icon_ws *ws, const void *d_Ahwb, const float *d_target, int S, double *h_loss,
                             void *stream);
icon_status icon_ws_get_grads(icon_ws *ws, float *h_grads, size_t count);

/* One Adam step with learning rate lr from the last gradients. */
icon_status icon_ws_update(icon_ws *ws, float lr, void *stream);

/* icon_ws_backprop followed by icon_ws_update. */
icon_status icon_ws_train_step(icon_ws *ws, const void *d_Ahwb, const float *d_target, int S, float lr,
                               double *h_loss, void *stream);

/* Loads parameters and output gain from a weights file: the 8 bytes
 * "ICONWSB1", the parameter count (uint64, little-endian), the gain (float32)
 * and the FP32 parameters (as written by feilab_b200.warmstart.save_raw from a
 * trained network's .npz).  Fails with ICON_ERR_IO when the file does not
 * hold this network's parameter count. */
icon_status icon_ws_load(icon_ws *ws, const char *path);

/* Warm start of the plan's reconstruct calls (icon_reconstruct_host,
 * icon_reconstruct_stack, icon_reconstruct_stack_host): after the input
 * stage, the network `ws` (made for this plan; it must outlive the use)
 * predicts each slice's start and icon_solve_warm with `wc` solves from it,
 * redoing from m = 0 every slice its acceptance test rejects.  ws = NULL
 * turns it off (the reference's cold start, Iteration2.cu:33).  Allocates
 * two image buffers of the plan's capacity on first use.  No counterpart in
 * the reference. */
icon_status icon_plan_set_warm_start(icon_plan *plan, icon_ws *ws, const icon_warm_cfg *wc);

/* Slices the plan's warm-started reconstruct calls have accepted and redone
 * from m = 0 since the plan was made. */
icon_status icon_plan_warm_counts(const icon_plan *plan, long long *h_accepted, long long *h_redone);

/* Test of the convolution's bounded waits (no reference counterpart): one
 * convolution as icon_ws_conv3x3 (one input, no bias, no ReLU, one output)
 * whose first pipeline stage waits for 16 bytes more than its loads deliver,
 * so that the wait for it ends only by running out after wait_us
 * microseconds (1 .. 1000000).  The kernel then records error code 1, lets
 * the loads it issued land (within 2 s), skips its output, releases its
 * tensor memory and returns; icon_ws_device_error reports the code and the
 * device stays usable. */
icon_status icon_ws_conv3x3_wait_test(const void *in0, int cin0, int nimg, int H, int W, const void *w, int N,
                                      void *out0, unsigned wait_us, void *stream);

/* Reads and clears the current device's error flag of the tensor-core
 * kernels (0: none; 1, 2, 3: a bounded wait for a TMA load, for the MMAs of
 * a stage, or for the accumulator ran out; the kernel then skipped its
 * output).  Synchronises with the device. */
icon_status icon_ws_device_error(int *h_code);

#ifdef __cplusplus
}
#endif

#endif /* ICON_WARMSTART_H */
