// ws_conv.cuh -- 3x3 convolution (stride 1, zero padding 1) of NHWC BF16
// activations as an implicit GEMM on the sm_100a tensor cores.
//
// One CTA computes a tile of 128 output pixels (one image row, w0..w0+127)
// by N output channels: D[128][N] = sum over K of A[128][K] * B[N][K]^T with
// K = taps x input channels.  For every (input tensor, chunk of cc channels,
// tap) step, TMA loads the 128 x cc input box shifted by the tap (zero fill
// outside the image gives the padding) and the N x cc weight box, both into
// swizzled K-major shared-memory tiles; one thread issues cc/16
// tcgen05.mma (M = 128, K = 16) per step into an FP32 accumulator in tensor
// memory.  A ring of kStages stages keeps the loads ahead of the MMAs.  The
// epilogue (four warps, one pixel per thread) reads the accumulator with
// tcgen05.ld, adds the bias, applies ReLU, rounds to BF16 and stores the
// pixel's channels; the channels can be split over two outputs (the gradient
// of a concatenated input) and added to what an output holds.
//
// Two input tensors are read as one concatenated input (the decoder's skip
// connections), so the concatenation is never stored.  Weights are
// [tap][N][Cin] BF16 with tap = 3*dy + dx.
#pragma once
#include "ws_tc.cuh"

namespace ws {

constexpr int kConvStages = 4;
constexpr int kConvThreads = 128;
constexpr int kTileM = 128;

struct ConvArgs {
    int nin;                 // input tensors (1 or 2), concatenated along channels
    int cin0, cin1;          // their channels
    int H, W;                // image size (output = input size)
    int cc;                  // channels per K step (16, 32 or 64; divides cin0 and cin1)
    int N;                   // output channels (multiple of 16, <= 256)
    int nsplit;              // out0 takes channels [0, nsplit), out1 [nsplit, N)
    __nv_bfloat16 *out0, *out1;
    int acc0, acc1;          // 1: add to the output's values
    const float *bias;       // [N] or null
    int relu;
    int *err;                // device error flag
    // Limit of the pipeline's load and MMA waits (normally kWaitNs).  The
    // waits that drain copies and MMAs before the CTA exits always use
    // kWaitNs, so nothing is left in flight.
    unsigned long long wait_ns;
    // Test of the bounded waits: the first stage's barrier expects 16 bytes
    // more than its loads deliver, so the wait for it can only run out.
    int hold;
};

__host__ __device__ inline size_t conv_stage_a_bytes(int cc) { return (size_t)kTileM * cc * 2; }
__host__ __device__ inline size_t conv_stage_b_bytes(int N, int cc) { return (((size_t)N * cc * 2) + 1023) & ~(size_t)1023; }
__host__ __device__ inline size_t conv_smem_bytes(int N, int cc)
{
    return 1024 /* alignment slack */ + kConvStages * (conv_stage_a_bytes(cc) + conv_stage_b_bytes(N, cc)) +
           (2 * kConvStages + 1) * 8 + 16 + (size_t)N * 4;
}
__host__ __device__ inline uint32_t conv_tmem_cols(int N)
{
    uint32_t c = 32;
    while ((int)c < N) c <<= 1;
    return c;
}

__global__ void __launch_bounds__(kConvThreads, 1)
k_conv3x3_tc(const __grid_constant__ CUtensorMap in0, const __grid_constant__ CUtensorMap in1,
             const __grid_constant__ CUtensorMap wmap, ConvArgs a)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const size_t abytes = conv_stage_a_bytes(a.cc), bbytes = conv_stage_b_bytes(a.N, a.cc);
    unsigned char *sa = base;
    unsigned char *sb = base + kConvStages * abytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(sb + kConvStages * bbytes);
    uint64_t *empty = full + kConvStages;
    uint64_t *done = empty + kConvStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    float *sbias = reinterpret_cast<float *>(tslot + 4);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int w0 = blockIdx.x * kTileM, h = blockIdx.y, img = blockIdx.z;
    const uint32_t ncols = conv_tmem_cols(a.N);
    const int sw = a.cc * 2;                       // swizzle span = row bytes of a tile
    const int chunks0 = a.cin0 / a.cc, chunks = chunks0 + (a.nin > 1 ? a.cin1 / a.cc : 0);
    const int steps = 9 * chunks;
    const uint32_t tx = (uint32_t)(kTileM * a.cc * 2 + a.N * a.cc * 2);
    const uint32_t idesc = idesc_bf16(kTileM, a.N);

    if (tid == 0) {
        for (int s = 0; s < kConvStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_fence_init();
        tma_prefetch_desc(&in0);
        if (a.nin > 1) tma_prefetch_desc(&in1);
        tma_prefetch_desc(&wmap);
    }
    for (int i = tid; i < a.N; i += kConvThreads) sbias[i] = a.bias ? a.bias[i] : 0.f;
    if (warp == 0) tmem_alloc(tslot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    bool ok = true;
    if (warp == 0) {
        if (lane == 0) {
            // Step k: global chunk g = k / 9 (tensor 0's chunks, then tensor
            // 1's), tap = k % 9.
            auto issue = [&](int k) {
                const int s = k % kConvStages, g = k / 9, tap = k - 9 * g, dy = tap / 3, dx = tap - 3 * dy;
                const bool second = g >= chunks0;
                const int c0 = (second ? g - chunks0 : g) * a.cc;
                const int wc0 = (second ? a.cin0 : 0) + c0;
                mbar_expect_tx(&full[s], tx + ((a.hold && k == 0) ? 16u : 0u));
                tma_load_4d(sa + s * abytes, second ? &in1 : &in0, c0, w0 + dx - 1, h + dy - 1, img, &full[s]);
                tma_load_3d(sb + s * bbytes, &wmap, wc0, 0, tap, &full[s]);
            };
            const int pre = steps < kConvStages ? steps : kConvStages;
            for (int k = 0; k < pre; ++k) issue(k);
            int issued = pre;
            for (int k = 0; k < steps && ok; ++k) {
                const int s = k % kConvStages;
                if (!mbar_wait(&full[s], (uint32_t)((k / kConvStages) & 1), a.err, kErrLoadWait, a.wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(sa + s * abytes), b0 = smem_u32(sb + s * bbytes);
                for (int kk = 0; kk < a.cc / 16; ++kk) {
                    const uint64_t ad = smem_desc_kmajor(a0 + kk * 32, sw);
                    const uint64_t bd = smem_desc_kmajor(b0 + kk * 32, sw);
                    mma_bf16(tmem, ad, bd, idesc, (k > 0) || (kk > 0));
                }
                mma_commit(&empty[s]);
                // Refill the stage of step k-1 once its MMAs are done (step
                // k's MMAs stay queued meanwhile).
                if (k >= 1 && issued < steps) {
                    const int kp = k - 1, sp = kp % kConvStages;
                    if (!mbar_wait(&empty[sp], (uint32_t)((kp / kConvStages) & 1), a.err, kErrMmaWait, a.wait_ns)) {
                        ok = false;
                        break;
                    }
                    issue(issued++);
                }
            }
            mma_commit(done);
            if (!ok) {
                // Let the copies already issued land before the CTA exits.
                for (int k = 0; k < issued; ++k) {
                    const int s = k % kConvStages;
                    mbar_wait(&full[s], (uint32_t)((k / kConvStages) & 1), a.err, kErrLoadWait);
                }
            }
        }
        __syncwarp();
    }
    const bool fin = mbar_wait(done, 0, a.err, kErrDoneWait);
    tc_fence_after();
    if (fin && *a.err == kErrNone) {
        const int px = w0 + tid;
        const bool valid = px < a.W;
        const size_t pix = ((size_t)img * a.H + h) * a.W + px;
        for (int c = 0; c < a.N; c += 16) {
            float v[16];
            __syncwarp();
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            if (!valid) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] += sbias[c + i];
                if (a.relu) v[i] = fmaxf(v[i], 0.f);
            }
            const bool first = c < a.nsplit;
            const int C = first ? a.nsplit : a.N - a.nsplit;
            __nv_bfloat16 *dst = (first ? a.out0 : a.out1) + pix * C + (first ? c : c - a.nsplit);
            if (first ? a.acc0 : a.acc1) {
                const __nv_bfloat162 *old = reinterpret_cast<const __nv_bfloat162 *>(dst);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float2 o = __bfloat1622float2(old[i]);
                    v[2 * i] += o.x;
                    v[2 * i + 1] += o.y;
                }
            }
            uint4 pk[2];
            uint32_t *pw = reinterpret_cast<uint32_t *>(pk);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                pw[i] = *reinterpret_cast<uint32_t *>(&t);
            }
            uint4 *d4 = reinterpret_cast<uint4 *>(dst);
            d4[0] = pk[0];
            d4[1] = pk[1];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace ws
