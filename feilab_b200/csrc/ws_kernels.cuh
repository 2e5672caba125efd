// ws_kernels.cuh -- SIMT kernels of the warm-start U-Net: everything but the
// 3x3 tensor-core convolutions (ws_conv.cuh).  Activations are NHWC BF16
// images [n][H][W][C]; arithmetic is FP32; every reduction is two-level with
// a fixed order (partial sums per block, then one pass over the partials), so
// results do not depend on scheduling.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace ws {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ __nv_bfloat16 tobf(float v) { return __float2bfloat16_rn(v); }

// ------------------------------------------------------------ slice layout
// Slices in the layout of the C ABI: [S][N0][N1], Y (N1) fastest, as the
// reference's images (X*N1 + Y).  The network image of slice s is
// [Hp][Wp] with h = Y, w = X (Hp, Wp: N1, N0 rounded up to multiples of 8).

// Per-slice sums of squares of Re(Ahwb); block s writes ss[s].
__global__ void k_slice_sumsq(const float2 *__restrict__ Ahwb, int N0, int N1, double *__restrict__ ss)
{
    __shared__ double red[256];
    const int s = blockIdx.x;
    const float2 *base = Ahwb + (size_t)s * N0 * N1;
    double acc = 0.0;
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
        double v = base[i].x;
        acc += v * v;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) ss[s] = red[0];
}

// Network input x[s][h][w] = Re(Ahwb[s][w][h]) / scale_s for h < N1, w < N0,
// zero in the padding; scale_s = sqrt(ss/(N0 N1)), or 1 when zero.
__global__ void k_net_input(const float2 *__restrict__ Ahwb, const double *__restrict__ ss, int N0, int N1, int Hp,
                            int Wp, int S, float *__restrict__ x, float *__restrict__ scale)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)S * Hp * Wp;
    if (i >= total) return;
    const int w = (int)(i % Wp), h = (int)((i / Wp) % Hp), s = (int)(i / ((size_t)Wp * Hp));
    const double q = ss[s] / ((double)N0 * N1);
    const float sc = q > 0 ? (float)sqrt(q) : 1.f;
    if (h == 0 && w == 0) scale[s] = sc;
    x[i] = (h < N1 && w < N0) ? Ahwb[((size_t)s * N0 + w) * N1 + h].x / sc : 0.f;
}

// Training target t[s][h][w] = m[s][w][h] / (scale_s * gain), zero in the padding.
__global__ void k_net_target(const float *__restrict__ m, const float *__restrict__ scale, float gain, int N0, int N1,
                             int Hp, int Wp, int S, float *__restrict__ t)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)S * Hp * Wp;
    if (i >= total) return;
    const int w = (int)(i % Wp), h = (int)((i / Wp) % Hp), s = (int)(i / ((size_t)Wp * Hp));
    t[i] = (h < N1 && w < N0) ? m[((size_t)s * N0 + w) * N1 + h] / (scale[s] * gain) : 0.f;
}

// m0[s][X][Y] = scale_s * gain * y[s][Y][X].
__global__ void k_net_output(const float *__restrict__ y, const float *__restrict__ scale, float gain, int N0, int N1,
                             int Hp, int Wp, int S, float *__restrict__ m)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)S * N0 * N1;
    if (i >= total) return;
    const int Y = (int)(i % N1), X = (int)((i / N1) % N0), s = (int)(i / ((size_t)N1 * N0));
    m[i] = (scale[s] * gain) * y[((size_t)s * Hp + Y) * Wp + X];
}

// ------------------------------------------------------------ first layer
// 3x3 convolution of the one-channel input to 16 channels, bias, ReLU.
// w: [9][16] FP32, tap = 3*dy + dx.
__global__ void k_conv_in(const float *__restrict__ x, const float *__restrict__ w, const float *__restrict__ bias,
                          int n, int H, int W, __nv_bfloat16 *__restrict__ y)
{
    __shared__ float sw[9 * 16 + 16];
    for (int i = threadIdx.x; i < 9 * 16; i += blockDim.x) sw[i] = w[i];
    for (int i = threadIdx.x; i < 16; i += blockDim.x) sw[144 + i] = bias[i];
    __syncthreads();
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)n * H * W) return;
    const int xw = (int)(p % W), xh = (int)((p / W) % H), im = (int)(p / ((size_t)W * H));
    float in[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        const int hh = xh + t / 3 - 1, ww = xw + t % 3 - 1;
        in[t] = (hh >= 0 && hh < H && ww >= 0 && ww < W) ? x[((size_t)im * H + hh) * W + ww] : 0.f;
    }
    __align__(16) __nv_bfloat16 o[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        float a = sw[144 + c];
#pragma unroll
        for (int t = 0; t < 9; ++t) a = fmaf(sw[t * 16 + c], in[t], a);
        o[c] = tobf(fmaxf(a, 0.f));
    }
    uint4 *d = reinterpret_cast<uint4 *>(y + p * 16);
    d[0] = reinterpret_cast<uint4 *>(o)[0];
    d[1] = reinterpret_cast<uint4 *>(o)[1];
}

// Weight and bias gradients of the first layer: block = 160 threads, one per
// output (tap*16 + c, or 144 + c for the bias); each block sums over its
// strip of per_block pixels into part[blk][160].
__global__ void k_conv_in_wgrad(const float *__restrict__ x, const __nv_bfloat16 *__restrict__ gz, int n, int H,
                                int W, int per_block, float *__restrict__ part)
{
    const int o = threadIdx.x, c = o % 16, t = o / 16;
    const size_t p0 = (size_t)blockIdx.x * per_block, total = (size_t)n * H * W;
    float acc = 0.f;
    for (int k = 0; k < per_block; ++k) {
        const size_t p = p0 + k;
        if (p >= total) break;
        const float g = bf(gz[p * 16 + c]);
        if (t == 9) {
            acc += g;
        } else {
            const int xw = (int)(p % W), xh = (int)((p / W) % H), im = (int)(p / ((size_t)W * H));
            const int hh = xh + t / 3 - 1, ww = xw + t % 3 - 1;
            if (hh >= 0 && hh < H && ww >= 0 && ww < W) acc = fmaf(g, x[((size_t)im * H + hh) * W + ww], acc);
        }
    }
    part[(size_t)blockIdx.x * 160 + o] = acc;
}

// ------------------------------------------------------------ pool / upsample
// 2x2 average pooling; C a multiple of 8 (8 channels per thread).
__global__ void k_pool2(const __nv_bfloat16 *__restrict__ in, int n, int H, int W, int C, __nv_bfloat16 *__restrict__ out)
{
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * Ho * Wo * C8) return;
    const int c8 = (int)(i % C8);
    const size_t q = i / C8;
    const int wo = (int)(q % Wo), ho = (int)((q / Wo) % Ho), im = (int)(q / ((size_t)Wo * Ho));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
            const uint4 v =
                *reinterpret_cast<const uint4 *>(in + (((size_t)im * H + 2 * ho + dy) * W + 2 * wo + dx) * C + 8 * c8);
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += bf(e[k]);
        }
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = tobf(0.25f * acc[k]);
    *reinterpret_cast<uint4 *>(out + (((size_t)im * Ho + ho) * Wo + wo) * C + 8 * c8) = *reinterpret_cast<uint4 *>(o);
}

// Gradient of the pooling: gin[2h+dy][2w+dx] (+)= gout[h][w] / 4 (H, W = input size).
__global__ void k_pool2_bwd(const __nv_bfloat16 *__restrict__ gout, int n, int H, int W, int C, int accumulate,
                            __nv_bfloat16 *__restrict__ gin)
{
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * H * W * C8) return;
    const int c8 = (int)(i % C8);
    const size_t q = i / C8;
    const int w = (int)(q % W), h = (int)((q / W) % H), im = (int)(q / ((size_t)W * H));
    const uint4 g = *reinterpret_cast<const uint4 *>(gout + (((size_t)im * Ho + h / 2) * Wo + w / 2) * C + 8 * c8);
    const __nv_bfloat16 *ge = reinterpret_cast<const __nv_bfloat16 *>(&g);
    uint4 *dst = reinterpret_cast<uint4 *>(gin + q * C + 8 * c8);
    __align__(16) __nv_bfloat16 o[8];
    if (accumulate) {
        const uint4 old = *dst;
        const __nv_bfloat16 *oe = reinterpret_cast<const __nv_bfloat16 *>(&old);
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = tobf(bf(oe[k]) + 0.25f * bf(ge[k]));
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = tobf(0.25f * bf(ge[k]));
    }
    *dst = *reinterpret_cast<uint4 *>(o);
}

// Nearest 2x upsampling: out[h][w] = in[h/2][w/2] (H, W = output size).
__global__ void k_up2(const __nv_bfloat16 *__restrict__ in, int n, int H, int W, int C, __nv_bfloat16 *__restrict__ out)
{
    const int C8 = C / 8;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * H * W * C8) return;
    const int c8 = (int)(i % C8);
    const size_t q = i / C8;
    const int w = (int)(q % W), h = (int)((q / W) % H), im = (int)(q / ((size_t)W * H));
    *reinterpret_cast<uint4 *>(out + q * C + 8 * c8) =
        *reinterpret_cast<const uint4 *>(in + (((size_t)im * (H / 2) + h / 2) * (W / 2) + w / 2) * C + 8 * c8);
}

// Gradient of the upsampling: gin[h][w] = sum of gout over its 2x2 block
// (H, W = input size).
__global__ void k_up2_bwd(const __nv_bfloat16 *__restrict__ gout, int n, int H, int W, int C,
                          __nv_bfloat16 *__restrict__ gin)
{
    const int C8 = C / 8;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * H * W * C8) return;
    const int c8 = (int)(i % C8);
    const size_t q = i / C8;
    const int w = (int)(q % W), h = (int)((q / W) % H), im = (int)(q / ((size_t)W * H));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
            const uint4 v = *reinterpret_cast<const uint4 *>(
                gout + (((size_t)im * 2 * H + 2 * h + dy) * (2 * W) + 2 * w + dx) * C + 8 * c8);
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += bf(e[k]);
        }
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = tobf(acc[k]);
    *reinterpret_cast<uint4 *>(gin + q * C + 8 * c8) = *reinterpret_cast<uint4 *>(o);
}

// ReLU gradient in place: g = g where y > 0, else 0 (y is the ReLU output).
__global__ void k_relu_bwd(__nv_bfloat16 *__restrict__ g, const __nv_bfloat16 *__restrict__ y, size_t count8)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count8) return;
    uint4 gv = reinterpret_cast<uint4 *>(g)[i];
    const uint4 yv = reinterpret_cast<const uint4 *>(y)[i];
    __nv_bfloat16 *ge = reinterpret_cast<__nv_bfloat16 *>(&gv);
    const __nv_bfloat16 *ye = reinterpret_cast<const __nv_bfloat16 *>(&yv);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (!(bf(ye[k]) > 0.f)) ge[k] = tobf(0.f);
    reinterpret_cast<uint4 *>(g)[i] = gv;
}

// ------------------------------------------------------------ weight gradients
// dW[tap][co][ci] = sum over pixels of gz[p][co] * X[p shifted by tap][ci] for
// a 3x3 convolution whose input is X0 (c0 channels) concatenated with X1 (c1
// channels), and db[co] = sum gz[p][co].  Block = 16 x 16 threads over one
// (16 co, 16 ci) tile; it walks the 64-pixel row segments item = split +
// k*nsplit and writes its sums to part[split][tap][co][ci] (bias sums to
// bpart[split][co] from the ci-tile 0 blocks).
constexpr int kWgSeg = 64;

__global__ void __launch_bounds__(256) k_wgrad3x3(const __nv_bfloat16 *__restrict__ X0, int c0,
                                                   const __nv_bfloat16 *__restrict__ X1, int c1,
                                                   const __nv_bfloat16 *__restrict__ gz, int N, int n, int H, int W,
                                                   int nsplit, float *__restrict__ part, float *__restrict__ bpart)
{
    __shared__ float sg[kWgSeg][17];
    __shared__ float sx[3][kWgSeg + 2][17];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // ci, co within the tile
    const int co0 = blockIdx.y * 16, ci0 = blockIdx.z * 16;
    const int Cin = c0 + c1;
    const bool second = ci0 >= c0;
    const __nv_bfloat16 *X = second ? X1 : X0;
    const int CX = second ? c1 : c0, cx0 = second ? ci0 - c0 : ci0;
    const int segs = (W + kWgSeg - 1) / kWgSeg;
    const long long items = (long long)n * H * segs;
    float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float bacc = 0.f;
    for (long long it = blockIdx.x; it < items; it += nsplit) {
        const int seg = (int)(it % segs);
        const long long r = it / segs;
        const int h = (int)(r % H), im = (int)(r / H), w0 = seg * kWgSeg;
        __syncthreads();
        for (int i = threadIdx.x; i < kWgSeg * 16; i += 256) {
            const int px = i / 16, c = i % 16, w = w0 + px;
            sg[px][c] = (w < W) ? bf(gz[(((size_t)im * H + h) * W + w) * N + co0 + c]) : 0.f;
        }
        for (int i = threadIdx.x; i < 3 * (kWgSeg + 2) * 16; i += 256) {
            const int c = i % 16, px = (i / 16) % (kWgSeg + 2), dy = i / (16 * (kWgSeg + 2));
            const int hh = h + dy - 1, ww = w0 + px - 1;
            sx[dy][px][c] = (hh >= 0 && hh < H && ww >= 0 && ww < W)
                                ? bf(X[(((size_t)im * H + hh) * W + ww) * CX + cx0 + c])
                                : 0.f;
        }
        __syncthreads();
        for (int px = 0; px < kWgSeg; ++px) {
            const float g = sg[px][ty];
            bacc += g;
#pragma unroll
            for (int t = 0; t < 9; ++t) acc[t] = fmaf(g, sx[t / 3][px + t % 3][tx], acc[t]);
        }
    }
    const size_t base = (size_t)blockIdx.x * 9 * N * Cin;
#pragma unroll
    for (int t = 0; t < 9; ++t) part[base + ((size_t)t * N + co0 + ty) * Cin + ci0 + tx] = acc[t];
    if (blockIdx.z == 0 && tx == 0) bpart[(size_t)blockIdx.x * N + co0 + ty] = bacc;
}

// out[i] = sum over s < nsplit of part[s][i], in order of s.
__global__ void k_sum_parts(const float *__restrict__ part, int nsplit, size_t len, float *__restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len) return;
    float a = 0.f;
    for (int s = 0; s < nsplit; ++s) a += part[(size_t)s * len + i];
    out[i] = a;
}

// ------------------------------------------------------------ output layer
// y[p] = b + sum_c w[c] * d[p][c] (1x1 convolution of 16 channels to one).
__global__ void k_conv_out(const __nv_bfloat16 *__restrict__ d, const float *__restrict__ w, const float *__restrict__ b,
                           size_t npix, float *__restrict__ y)
{
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    const uint4 *v = reinterpret_cast<const uint4 *>(d + p * 16);
    float a = b[0];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const uint4 u = v[q];
        const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
        for (int k = 0; k < 8; ++k) a = fmaf(w[8 * q + k], bf(e[k]), a);
    }
    y[p] = a;
}

// Mean squared error over the valid pixels (h < Hv, w < Wv) of S images
// [S][Hp][Wp]: dy = 2 (y - t) / count (zero in the padding); per-block partial
// sums of (y - t)^2 in double to lpart[blockIdx.x].  blockDim = 256.
__global__ void k_mse(const float *__restrict__ y, const float *__restrict__ t, int S, int Hp, int Wp, int Hv, int Wv,
                      float *__restrict__ dy, double *__restrict__ lpart)
{
    __shared__ double red[256];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)S * Hp * Wp;
    double l = 0.0;
    if (i < total) {
        const int w = (int)(i % Wp), h = (int)((i / Wp) % Hp);
        float g = 0.f;
        if (h < Hv && w < Wv) {
            const float e = y[i] - t[i];
            l = (double)e * e;
            g = 2.f * e / ((float)S * Hv * Wv);
        }
        dy[i] = g;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}

// Backward of the output layer: gd[p][c] = dy[p] * w[c] (BF16), and per-block
// partial sums of dw[c] = sum dy[p] d[p][c] and db = sum dy[p]
// (part[blk][17]).  blockDim = 256.
__global__ void k_conv_out_bwd(const __nv_bfloat16 *__restrict__ d, const float *__restrict__ dy,
                               const float *__restrict__ w, size_t npix, __nv_bfloat16 *__restrict__ gd,
                               float *__restrict__ part)
{
    __shared__ float red[17][257];
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float loc[17];
#pragma unroll
    for (int k = 0; k < 17; ++k) loc[k] = 0.f;
    if (p < npix) {
        const float g = dy[p];
        const uint4 *v = reinterpret_cast<const uint4 *>(d + p * 16);
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const uint4 u = v[q];
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                loc[8 * q + k] = g * bf(e[k]);
                o[8 * q + k] = tobf(g * w[8 * q + k]);
            }
        }
        loc[16] = g;
        uint4 *dst = reinterpret_cast<uint4 *>(gd + p * 16);
        dst[0] = reinterpret_cast<uint4 *>(o)[0];
        dst[1] = reinterpret_cast<uint4 *>(o)[1];
    }
#pragma unroll
    for (int k = 0; k < 17; ++k) red[k][threadIdx.x] = loc[k];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 17; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 17) part[(size_t)blockIdx.x * 17 + threadIdx.x] = red[threadIdx.x][0];
}

// ------------------------------------------------------------ optimiser
// Adam on the FP32 master parameters (bias-corrected, no weight decay).
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of a 3x3 layer's weights: wb[tap][N][Cin] = w, and the weights
// of its input gradient wt[tap][Cin][N] = w[8 - tap][N][Cin] (flipped taps,
// swapped channels).
__global__ void k_weights_bf16(const float *__restrict__ w, int N, int Cin, __nv_bfloat16 *__restrict__ wb,
                               __nv_bfloat16 *__restrict__ wt)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)9 * N * Cin) return;
    const int ci = (int)(i % Cin), co = (int)((i / Cin) % N), tap = (int)(i / ((size_t)Cin * N));
    const __nv_bfloat16 v = tobf(w[i]);
    wb[i] = v;
    wt[((size_t)(8 - tap) * Cin + ci) * N + co] = v;
}

}  // namespace ws
