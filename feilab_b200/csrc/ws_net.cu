// ws_net.cu -- the warm-start U-Net: parameters, activations, forward and
// backward passes, Adam, and the network part of include/icon_warmstart.h.
//
// Layers (channels; level l works on the image downsampled 2^l times):
//   level 0  in: 1 -> 16 (SIMT), c0b: 16 -> 16                 -> e0
//   level 1  pool(e0), c1a: 16 -> 32, c1b: 32 -> 32            -> e1
//   level 2  pool(e1), c2a: 32 -> 64, c2b: 64 -> 64            -> e2
//   level 3  pool(e2), c3a: 64 -> 128, c3b: 128 -> 128         -> b
//   decoder  up(b) ++ e2: 192 -> 64, 64 -> 64                  -> d2
//            up(d2) ++ e1: 96 -> 32, 32 -> 32                  -> d1
//            up(d1) ++ e0: 48 -> 16, 16 -> 16                  -> d0
//   out      1x1: 16 -> 1 (no ReLU)
// All 3x3 layers but the first run on the tensor cores (ws_conv.cuh), their
// input gradients too (the same convolution with flipped weights); weight
// gradients, pooling, upsampling and the first and last layers are SIMT
// (ws_kernels.cuh).  The image is the slice's N1 x N0 back-projection padded
// to multiples of 8, divided by its RMS; the output is scaled back by the
// same RMS times a fixed gain.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "icon_b200.h"
#include "icon_internal.h"
#include "icon_warmstart.h"
#include "ws_kernels.cuh"

extern "C" void icon_internal_set_error(const char *msg);
icon_status ws_conv3x3_launch(const void *in0, int cin0, const void *in1, int cin1, int nimg, int H, int W,
                              const void *w, const float *bias, int N, int relu, void *out0, int nsplit, int acc0,
                              void *out1, int acc1, cudaStream_t st, unsigned long long wait_ns = 2000000000ull,
                              int hold = 0);

namespace {

icon_status net_fail(icon_status st, const std::string &msg)
{
    icon_internal_set_error(msg.c_str());
    return st;
}

#define NET_CUDA(call)                                                                                          \
    do {                                                                                                        \
        cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess) return net_fail(ICON_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define NET_TRY(x)                         \
    do {                                   \
        icon_status s_ = (x);              \
        if (s_ != ICON_OK) return s_;      \
    } while (0)

using bf16 = __nv_bfloat16;

struct TcLayer {
    int cin0, cin1, N;
    size_t w_off, b_off;
    bf16 *wb = nullptr, *wt = nullptr;
};

// 3x3 tensor-core layers {cin0, cin1, N} in the order of the header comment.
const int kLayerShape[13][3] = {{16, 0, 16},  {16, 0, 32},   {32, 0, 32},  {32, 0, 64}, {64, 0, 64},
                                {64, 0, 128}, {128, 0, 128}, {128, 64, 64}, {64, 0, 64}, {64, 32, 32},
                                {32, 0, 32},  {32, 16, 16},  {16, 0, 16}};
enum { C0B, C1A, C1B, C2A, C2B, C3A, C3B, D2A, D2B, D1A, D1B, D0A, D0B };

// Parameter layout: first layer w [9][16], b [16]; then per 3x3 layer
// w [9][N][Cin], b [N]; then the output layer w [16], b [1].
constexpr size_t kInW = 0, kInB = 144;

size_t layout_params(std::vector<TcLayer> *layers, size_t *out_w)
{
    size_t off = 160;
    std::vector<TcLayer> L;
    for (auto &s : kLayerShape) {
        TcLayer t;
        t.cin0 = s[0];
        t.cin1 = s[1];
        t.N = s[2];
        t.w_off = off;
        off += (size_t)9 * t.N * (t.cin0 + t.cin1);
        t.b_off = off;
        off += t.N;
        L.push_back(t);
    }
    if (out_w) *out_w = off;
    off += 17;
    if (layers) *layers = L;
    return off;
}

// Scratch sizes of the weight-gradient reduction (splits per layer).
int wgrad_splits(int N, int Cin) { return std::max(1, std::min(256, 1184 / ((N / 16) * (Cin / 16)))); }

struct Img {
    bf16 *p = nullptr;
    int H = 0, W = 0, C = 0;
};

struct DevMem {
    std::vector<void *> ptrs;
    ~DevMem()
    {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    icon_status alloc(T **out, size_t count)
    {
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 256));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return net_fail(ICON_ERR_NOMEM, "warm start: cudaMalloc failed");
        }
        ptrs.push_back(p);
        *out = static_cast<T *>(p);
        return ICON_OK;
    }
};

unsigned long long splitmix(unsigned long long &s)
{
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double gauss(unsigned long long &s)
{
    double u1 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    double u2 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

unsigned grid1(size_t n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

struct icon_ws {
    int dev = 0, N0 = 0, N1 = 0, cap = 0, Hp = 0, Wp = 0;
    float gain = 1.f;
    int step = 0;
    DevMem mem;
    std::vector<TcLayer> layers;
    size_t nparam = 0, out_off = 0;
    float *params = nullptr, *grads = nullptr, *am = nullptr, *av = nullptr;
    float *x = nullptr, *t = nullptr, *y = nullptr, *dy = nullptr, *in_scale = nullptr;
    double *ss = nullptr, *lpart = nullptr;
    float *part = nullptr, *bpart = nullptr;
    size_t part_len = 0, bpart_len = 0;
    // activations and their gradients
    Img e0a, e0, u0, d0a, d0, p0, e1a, e1, u1, d1a, d1, p1, e2a, e2, u2, d2a, d2, p2, ba, b;
    Img g_e0a, g_e0, g_u0, g_d0a, g_d0, g_p0, g_e1a, g_e1, g_u1, g_d1a, g_d1, g_p1, g_e2a, g_e2, g_u2, g_d2a, g_d2,
        g_p2, g_ba, g_b;

    icon_status img(Img &m, int level, int C)
    {
        m.H = Hp >> level;
        m.W = Wp >> level;
        m.C = C;
        return mem.alloc(&m.p, (size_t)cap * m.H * m.W * C);
    }

    icon_status refresh_bf16(cudaStream_t st)
    {
        for (auto &L : layers) {
            const size_t n = (size_t)9 * L.N * (L.cin0 + L.cin1);
            ws::k_weights_bf16<<<grid1(n, 256), 256, 0, st>>>(params + L.w_off, L.N, L.cin0 + L.cin1, L.wb, L.wt);
        }
        NET_CUDA(cudaGetLastError());
        return ICON_OK;
    }

    icon_status conv(int li, const Img &in0, const Img *in1, Img &out, int S, cudaStream_t st)
    {
        const TcLayer &L = layers[li];
        return ws_conv3x3_launch(in0.p, in0.C, in1 ? in1->p : nullptr, in1 ? in1->C : 0, S, out.H, out.W, L.wb,
                                 params + L.b_off, L.N, 1, out.p, L.N, 0, nullptr, 0, st);
    }

    void pool(const Img &in, Img &out, int S, cudaStream_t st)
    {
        size_t n = (size_t)S * out.H * out.W * (in.C / 8);
        ws::k_pool2<<<grid1(n, 256), 256, 0, st>>>(in.p, S, in.H, in.W, in.C, out.p);
    }

    void up(const Img &in, Img &out, int S, cudaStream_t st)
    {
        size_t n = (size_t)S * out.H * out.W * (out.C / 8);
        ws::k_up2<<<grid1(n, 256), 256, 0, st>>>(in.p, S, out.H, out.W, out.C, out.p);
    }

    icon_status forward(const float2 *Ahwb, int S, cudaStream_t st)
    {
        ws::k_slice_sumsq<<<S, 256, 0, st>>>(Ahwb, N0, N1, ss);
        const size_t npix = (size_t)S * Hp * Wp;
        ws::k_net_input<<<grid1(npix, 256), 256, 0, st>>>(Ahwb, ss, N0, N1, Hp, Wp, S, x, in_scale);
        ws::k_conv_in<<<grid1(npix, 128), 128, 0, st>>>(x, params + kInW, params + kInB, S, Hp, Wp, e0a.p);
        NET_CUDA(cudaGetLastError());
        NET_TRY(conv(C0B, e0a, nullptr, e0, S, st));
        pool(e0, p0, S, st);
        NET_TRY(conv(C1A, p0, nullptr, e1a, S, st));
        NET_TRY(conv(C1B, e1a, nullptr, e1, S, st));
        pool(e1, p1, S, st);
        NET_TRY(conv(C2A, p1, nullptr, e2a, S, st));
        NET_TRY(conv(C2B, e2a, nullptr, e2, S, st));
        pool(e2, p2, S, st);
        NET_TRY(conv(C3A, p2, nullptr, ba, S, st));
        NET_TRY(conv(C3B, ba, nullptr, b, S, st));
        up(b, u2, S, st);
        NET_TRY(conv(D2A, u2, &e2, d2a, S, st));
        NET_TRY(conv(D2B, d2a, nullptr, d2, S, st));
        up(d2, u1, S, st);
        NET_TRY(conv(D1A, u1, &e1, d1a, S, st));
        NET_TRY(conv(D1B, d1a, nullptr, d1, S, st));
        up(d1, u0, S, st);
        NET_TRY(conv(D0A, u0, &e0, d0a, S, st));
        NET_TRY(conv(D0B, d0a, nullptr, d0, S, st));
        ws::k_conv_out<<<grid1(npix, 256), 256, 0, st>>>(d0.p, params + out_off, params + out_off + 16, npix, y);
        NET_CUDA(cudaGetLastError());
        return ICON_OK;
    }

    // Gradients of one 3x3 layer: ReLU backward of gout in place, weight and
    // bias gradients, and (when gin0) the input gradient split over gin0 /
    // gin1 (acc0: add to gin0).
    icon_status layer_bwd(int li, Img &gout, const Img &out, const Img &in0, const Img *in1, Img *gin0, int acc0,
                          Img *gin1, int S, cudaStream_t st)
    {
        const TcLayer &L = layers[li];
        const size_t cnt8 = (size_t)S * out.H * out.W * out.C / 8;
        ws::k_relu_bwd<<<grid1(cnt8, 256), 256, 0, st>>>(gout.p, out.p, cnt8);
        const int Cin = L.cin0 + L.cin1;
        const int segs = (out.W + ws::kWgSeg - 1) / ws::kWgSeg;
        const long long items = (long long)S * out.H * segs;
        int nsplit = wgrad_splits(L.N, Cin);
        if (nsplit > items) nsplit = (int)items;
        const size_t wlen = (size_t)9 * L.N * Cin;
        if ((size_t)nsplit * wlen > part_len || (size_t)nsplit * L.N > bpart_len)
            return net_fail(ICON_ERR_INVALID, "warm start: weight-gradient scratch too small");
        dim3 g(nsplit, L.N / 16, Cin / 16);
        ws::k_wgrad3x3<<<g, 256, 0, st>>>(in0.p, L.cin0, in1 ? in1->p : nullptr, L.cin1, gout.p, L.N, S, out.H,
                                           out.W, nsplit, part, bpart);
        ws::k_sum_parts<<<grid1(wlen, 256), 256, 0, st>>>(part, nsplit, wlen, grads + L.w_off);
        ws::k_sum_parts<<<grid1(L.N, 256), 256, 0, st>>>(bpart, nsplit, L.N, grads + L.b_off);
        NET_CUDA(cudaGetLastError());
        if (gin0)
            NET_TRY(ws_conv3x3_launch(gout.p, L.N, nullptr, 0, S, out.H, out.W, L.wt, nullptr, Cin, 0, gin0->p,
                                      L.cin0, acc0, gin1 ? gin1->p : nullptr, 0, st));
        return ICON_OK;
    }

    void pool_bwd(const Img &gout, Img &gin, int S, cudaStream_t st)
    {
        size_t n = (size_t)S * gin.H * gin.W * (gin.C / 8);
        ws::k_pool2_bwd<<<grid1(n, 256), 256, 0, st>>>(gout.p, S, gin.H, gin.W, gin.C, 1, gin.p);
    }

    void up_bwd(const Img &gout, Img &gin, int S, cudaStream_t st)
    {
        size_t n = (size_t)S * gin.H * gin.W * (gin.C / 8);
        ws::k_up2_bwd<<<grid1(n, 256), 256, 0, st>>>(gout.p, S, gin.H, gin.W, gin.C, gin.p);
    }

    icon_status backward(int S, cudaStream_t st)
    {
        const size_t npix = (size_t)S * Hp * Wp;
        {
            const unsigned nb = grid1(npix, 256);
            if ((size_t)nb * 17 > part_len) return net_fail(ICON_ERR_INVALID, "warm start: output scratch too small");
            ws::k_conv_out_bwd<<<nb, 256, 0, st>>>(d0.p, dy, params + out_off, npix, g_d0.p, part);
            ws::k_sum_parts<<<1, 32, 0, st>>>(part, (int)nb, 17, grads + out_off);
        }
        NET_TRY(layer_bwd(D0B, g_d0, d0, d0a, nullptr, &g_d0a, 0, nullptr, S, st));
        NET_TRY(layer_bwd(D0A, g_d0a, d0a, u0, &e0, &g_u0, 0, &g_e0, S, st));
        up_bwd(g_u0, g_d1, S, st);
        NET_TRY(layer_bwd(D1B, g_d1, d1, d1a, nullptr, &g_d1a, 0, nullptr, S, st));
        NET_TRY(layer_bwd(D1A, g_d1a, d1a, u1, &e1, &g_u1, 0, &g_e1, S, st));
        up_bwd(g_u1, g_d2, S, st);
        NET_TRY(layer_bwd(D2B, g_d2, d2, d2a, nullptr, &g_d2a, 0, nullptr, S, st));
        NET_TRY(layer_bwd(D2A, g_d2a, d2a, u2, &e2, &g_u2, 0, &g_e2, S, st));
        up_bwd(g_u2, g_b, S, st);
        NET_TRY(layer_bwd(C3B, g_b, b, ba, nullptr, &g_ba, 0, nullptr, S, st));
        NET_TRY(layer_bwd(C3A, g_ba, ba, p2, nullptr, &g_p2, 0, nullptr, S, st));
        pool_bwd(g_p2, g_e2, S, st);
        NET_TRY(layer_bwd(C2B, g_e2, e2, e2a, nullptr, &g_e2a, 0, nullptr, S, st));
        NET_TRY(layer_bwd(C2A, g_e2a, e2a, p1, nullptr, &g_p1, 0, nullptr, S, st));
        pool_bwd(g_p1, g_e1, S, st);
        NET_TRY(layer_bwd(C1B, g_e1, e1, e1a, nullptr, &g_e1a, 0, nullptr, S, st));
        NET_TRY(layer_bwd(C1A, g_e1a, e1a, p0, nullptr, &g_p0, 0, nullptr, S, st));
        pool_bwd(g_p0, g_e0, S, st);
        NET_TRY(layer_bwd(C0B, g_e0, e0, e0a, nullptr, &g_e0a, 0, nullptr, S, st));
        {
            const size_t cnt8 = (size_t)S * Hp * Wp * 16 / 8;
            ws::k_relu_bwd<<<grid1(cnt8, 256), 256, 0, st>>>(g_e0a.p, e0a.p, cnt8);
            const int per = 2048;
            const unsigned nb = grid1(npix, per);
            if ((size_t)nb * 160 > part_len)
                return net_fail(ICON_ERR_INVALID, "warm start: input-layer scratch too small");
            ws::k_conv_in_wgrad<<<nb, 160, 0, st>>>(x, g_e0a.p, S, Hp, Wp, per, part);
            ws::k_sum_parts<<<1, 160, 0, st>>>(part, (int)nb, 160, grads + kInW);
        }
        NET_CUDA(cudaGetLastError());
        return ICON_OK;
    }
};

namespace {

icon_status check_ws(const icon_ws *w, int S)
{
    if (!w) return net_fail(ICON_ERR_INVALID, "null warm-start network");
    if (S < 1 || S > w->cap) return net_fail(ICON_ERR_CAPACITY, "S outside 1..capacity of the warm-start network");
    return ICON_OK;
}

struct DevGuard {
    int old = -1;
    explicit DevGuard(int dev)
    {
        if (cudaGetDevice(&old) != cudaSuccess) old = -1;
        cudaSetDevice(dev);
    }
    ~DevGuard()
    {
        if (old >= 0) cudaSetDevice(old);
    }
};

}  // namespace

extern "C" {

size_t icon_ws_param_count(void) { return layout_params(nullptr, nullptr); }

icon_status icon_ws_create(icon_plan *plan, int capacity, icon_ws **out)
{
    if (!plan || !out || capacity < 1) return net_fail(ICON_ERR_INVALID, "icon_ws_create: bad argument");
    *out = nullptr;
    int dims[10];
    NET_TRY(icon_plan_query(plan, dims));
    auto w = std::make_unique<icon_ws>();
    w->dev = iconx::plan_device(plan);
    DevGuard dg(w->dev);
    w->N0 = dims[0];
    w->N1 = dims[1];
    if (capacity > dims[7]) return net_fail(ICON_ERR_CAPACITY, "warm-start capacity above the plan's");
    w->cap = capacity;
    w->Hp = (w->N1 + 7) & ~7;
    w->Wp = (w->N0 + 7) & ~7;
    w->nparam = layout_params(&w->layers, &w->out_off);
    auto &M = w->mem;
    NET_TRY(M.alloc(&w->params, w->nparam));
    NET_TRY(M.alloc(&w->grads, w->nparam));
    NET_TRY(M.alloc(&w->am, w->nparam));
    NET_TRY(M.alloc(&w->av, w->nparam));
    NET_CUDA(cudaMemset(w->params, 0, w->nparam * sizeof(float)));
    NET_CUDA(cudaMemset(w->grads, 0, w->nparam * sizeof(float)));
    NET_CUDA(cudaMemset(w->am, 0, w->nparam * sizeof(float)));
    NET_CUDA(cudaMemset(w->av, 0, w->nparam * sizeof(float)));
    for (auto &L : w->layers) {
        const size_t n = (size_t)9 * L.N * (L.cin0 + L.cin1);
        NET_TRY(M.alloc(&L.wb, n));
        NET_TRY(M.alloc(&L.wt, n));
    }
    const size_t npix = (size_t)capacity * w->Hp * w->Wp;
    NET_TRY(M.alloc(&w->x, npix));
    NET_TRY(M.alloc(&w->t, npix));
    NET_TRY(M.alloc(&w->y, npix));
    NET_TRY(M.alloc(&w->dy, npix));
    NET_TRY(M.alloc(&w->in_scale, capacity));
    NET_TRY(M.alloc(&w->ss, capacity));
    NET_TRY(M.alloc(&w->lpart, grid1(npix, 256)));
    size_t need = std::max<size_t>((size_t)grid1(npix, 256) * 17, (size_t)grid1(npix, 2048) * 160), bneed = 0;
    for (auto &L : w->layers) {
        const int Cin = L.cin0 + L.cin1, ns = wgrad_splits(L.N, Cin);
        need = std::max(need, (size_t)ns * 9 * L.N * Cin);
        bneed = std::max(bneed, (size_t)ns * L.N);
    }
    w->part_len = need;
    w->bpart_len = bneed;
    NET_TRY(M.alloc(&w->part, need));
    NET_TRY(M.alloc(&w->bpart, bneed));
    struct A {
        Img *m, *g;
        int level, C;
    } acts[] = {{&w->e0a, &w->g_e0a, 0, 16}, {&w->e0, &w->g_e0, 0, 16},  {&w->u0, &w->g_u0, 0, 32},
                {&w->d0a, &w->g_d0a, 0, 16}, {&w->d0, &w->g_d0, 0, 16},  {&w->p0, &w->g_p0, 1, 16},
                {&w->e1a, &w->g_e1a, 1, 32}, {&w->e1, &w->g_e1, 1, 32},  {&w->u1, &w->g_u1, 1, 64},
                {&w->d1a, &w->g_d1a, 1, 32}, {&w->d1, &w->g_d1, 1, 32},  {&w->p1, &w->g_p1, 2, 32},
                {&w->e2a, &w->g_e2a, 2, 64}, {&w->e2, &w->g_e2, 2, 64},  {&w->u2, &w->g_u2, 2, 128},
                {&w->d2a, &w->g_d2a, 2, 64}, {&w->d2, &w->g_d2, 2, 64},  {&w->p2, &w->g_p2, 3, 64},
                {&w->ba, &w->g_ba, 3, 128},  {&w->b, &w->g_b, 3, 128}};
    for (auto &a : acts) {
        NET_TRY(w->img(*a.m, a.level, a.C));
        NET_TRY(w->img(*a.g, a.level, a.C));
    }
    *out = w.release();
    return ICON_OK;
}

icon_status icon_ws_destroy(icon_ws *w)
{
    if (!w) return ICON_OK;
    DevGuard g(w->dev);
    cudaDeviceSynchronize();
    delete w;
    return ICON_OK;
}

icon_status icon_ws_init(icon_ws *w, unsigned long long seed)
{
    if (!w) return net_fail(ICON_ERR_INVALID, "null warm-start network");
    DevGuard g(w->dev);
    std::vector<float> h(w->nparam, 0.f);
    unsigned long long s = seed;
    const double sd_in = std::sqrt(2.0 / 9.0);
    for (size_t i = kInW; i < kInB; ++i) h[i] = (float)(sd_in * gauss(s));
    for (auto &L : w->layers) {
        const double sd = std::sqrt(2.0 / (9.0 * (L.cin0 + L.cin1)));
        for (size_t i = 0; i < (size_t)9 * L.N * (L.cin0 + L.cin1); ++i) h[L.w_off + i] = (float)(sd * gauss(s));
    }
    for (int i = 0; i < 16; ++i) h[w->out_off + i] = (float)(0.25 * gauss(s));
    NET_CUDA(cudaMemcpy(w->params, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
    NET_CUDA(cudaMemset(w->am, 0, w->nparam * sizeof(float)));
    NET_CUDA(cudaMemset(w->av, 0, w->nparam * sizeof(float)));
    w->step = 0;
    NET_TRY(w->refresh_bf16(0));
    NET_CUDA(cudaDeviceSynchronize());
    return ICON_OK;
}

icon_status icon_ws_set_params(icon_ws *w, const float *h_params, size_t count, float gain)
{
    if (!w || !h_params) return net_fail(ICON_ERR_INVALID, "icon_ws_set_params: null argument");
    if (count != w->nparam) return net_fail(ICON_ERR_INVALID, "icon_ws_set_params: wrong parameter count");
    if (!(gain > 0.f)) return net_fail(ICON_ERR_INVALID, "icon_ws_set_params: gain must be positive");
    DevGuard g(w->dev);
    NET_CUDA(cudaMemcpy(w->params, h_params, count * sizeof(float), cudaMemcpyHostToDevice));
    w->gain = gain;
    NET_TRY(w->refresh_bf16(0));
    NET_CUDA(cudaDeviceSynchronize());
    return ICON_OK;
}

icon_status icon_ws_get_params(icon_ws *w, float *h_params, size_t count, float *h_gain)
{
    if (!w || !h_params) return net_fail(ICON_ERR_INVALID, "icon_ws_get_params: null argument");
    if (count != w->nparam) return net_fail(ICON_ERR_INVALID, "icon_ws_get_params: wrong parameter count");
    DevGuard g(w->dev);
    NET_CUDA(cudaDeviceSynchronize());
    NET_CUDA(cudaMemcpy(h_params, w->params, count * sizeof(float), cudaMemcpyDeviceToHost));
    if (h_gain) *h_gain = w->gain;
    return ICON_OK;
}

icon_status icon_ws_set_gain(icon_ws *w, float gain)
{
    if (!w || !(gain > 0.f)) return net_fail(ICON_ERR_INVALID, "icon_ws_set_gain: bad argument");
    w->gain = gain;
    return ICON_OK;
}

icon_status icon_ws_load(icon_ws *w, const char *path)
{
    if (!w || !path) return net_fail(ICON_ERR_INVALID, "icon_ws_load: null argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return net_fail(ICON_ERR_IO, std::string("icon_ws_load: cannot open ") + path);
    char magic[8];
    unsigned long long count = 0;
    float gain = 0.f;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "ICONWSB1", 8) == 0 &&
              std::fread(&count, sizeof(count), 1, f) == 1 && std::fread(&gain, sizeof(gain), 1, f) == 1;
    std::vector<float> p;
    if (ok && count == w->nparam) {
        p.resize(count);
        ok = std::fread(p.data(), sizeof(float), count, f) == count;
    } else {
        ok = false;
    }
    std::fclose(f);
    if (!ok)
        return net_fail(ICON_ERR_IO, std::string("icon_ws_load: ") + path + " is not a weights file of " +
                                         std::to_string(w->nparam) + " parameters");
    return icon_ws_set_params(w, p.data(), p.size(), gain);
}

icon_status icon_ws_predict(icon_ws *w, const void *d_Ahwb, float *d_m0, int S, void *stream)
{
    NET_TRY(check_ws(w, S));
    if (!d_Ahwb || !d_m0) return net_fail(ICON_ERR_INVALID, "icon_ws_predict: null pointer");
    DevGuard g(w->dev);
    cudaStream_t st = (cudaStream_t)stream;
    NET_TRY(w->forward((const float2 *)d_Ahwb, S, st));
    const size_t nout = (size_t)S * w->N1 * w->N0;
    ws::k_net_output<<<grid1(nout, 256), 256, 0, st>>>(w->y, w->in_scale, w->gain, w->N0, w->N1, w->Hp, w->Wp, S,
                                                         d_m0);
    NET_CUDA(cudaGetLastError());
    return ICON_OK;
}

icon_status icon_ws_backprop(icon_ws *w, const void *d_Ahwb, const float *d_target, int S, double *h_loss,
                             void *stream)
{
    NET_TRY(check_ws(w, S));
    if (!d_Ahwb || !d_target) return net_fail(ICON_ERR_INVALID, "icon_ws_backprop: null pointer");
    DevGuard g(w->dev);
    cudaStream_t st = (cudaStream_t)stream;
    NET_TRY(w->forward((const float2 *)d_Ahwb, S, st));
    const size_t npix = (size_t)S * w->Hp * w->Wp;
    ws::k_net_target<<<grid1(npix, 256), 256, 0, st>>>(d_target, w->in_scale, w->gain, w->N0, w->N1, w->Hp, w->Wp, S,
                                                         w->t);
    const unsigned nb = grid1(npix, 256);
    ws::k_mse<<<nb, 256, 0, st>>>(w->y, w->t, S, w->Hp, w->Wp, w->N1, w->N0, w->dy, w->lpart);
    NET_CUDA(cudaGetLastError());
    NET_TRY(w->backward(S, st));
    if (h_loss) {
        std::vector<double> lp(nb);
        NET_CUDA(cudaMemcpyAsync(lp.data(), w->lpart, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        NET_CUDA(cudaStreamSynchronize(st));
        double l = 0.0;
        for (double v : lp) l += v;
        *h_loss = l / ((double)S * w->N1 * w->N0);
    }
    return ICON_OK;
}

icon_status icon_ws_update(icon_ws *w, float lr, void *stream)
{
    if (!w) return net_fail(ICON_ERR_INVALID, "null warm-start network");
    if (!(lr > 0.f)) return net_fail(ICON_ERR_INVALID, "icon_ws_update: lr must be positive");
    DevGuard g(w->dev);
    cudaStream_t st = (cudaStream_t)stream;
    w->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)w->step), c2 = 1.f - std::pow(b2, (float)w->step);
    ws::k_adam<<<grid1(w->nparam, 256), 256, 0, st>>>(w->params, w->grads, w->am, w->av, w->nparam, lr, b1, b2, 1e-8f,
                                                      c1, c2);
    NET_CUDA(cudaGetLastError());
    return w->refresh_bf16(st);
}

icon_status icon_ws_train_step(icon_ws *w, const void *d_Ahwb, const float *d_target, int S, float lr,
                               double *h_loss, void *stream)
{
    NET_TRY(icon_ws_backprop(w, d_Ahwb, d_target, S, h_loss, stream));
    return icon_ws_update(w, lr, stream);
}

icon_status icon_ws_get_grads(icon_ws *w, float *h_grads, size_t count)
{
    if (!w || !h_grads) return net_fail(ICON_ERR_INVALID, "icon_ws_get_grads: null argument");
    if (count != w->nparam) return net_fail(ICON_ERR_INVALID, "icon_ws_get_grads: wrong parameter count");
    DevGuard g(w->dev);
    NET_CUDA(cudaDeviceSynchronize());
    NET_CUDA(cudaMemcpy(h_grads, w->grads, count * sizeof(float), cudaMemcpyDeviceToHost));
    return ICON_OK;
}

}  // extern "C"

int iconx::ws_capacity(const icon_ws *w) { return w ? w->cap : 0; }
