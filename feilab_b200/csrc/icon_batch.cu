// icon_batch.cu -- uneven multi-series batches (include/icon_batch.h): one
// tuned plan per series, each series' iteration captured into CUDA graphs,
// all series replayed round-robin on their own streams; and the autotuner of
// slices per group and per launch with its cache file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "icon_batch.h"
#include "icon_internal.h"

namespace {

using iconx::fail_msg;

#define B_CUDA(call)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) return fail_msg(ICON_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
#define B_TRY(call)                        \
    do {                                   \
        icon_status s_ = (call);           \
        if (s_ != ICON_OK) return s_;      \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int thickness_of(const icon_series &s) { return s.thickness == 0 ? s.nx : s.thickness; }

// Cache key of a series shape; slice counts of 256 and more share a key
// (the chunk candidates are the same for them).
std::string shape_key(const icon_series &s, int op)
{
    std::ostringstream k;
    k << s.nx << ' ' << thickness_of(s) << ' ' << s.ntilt << ' ' << std::min(s.slices, 256) << ' ' << op;
    return k.str();
}

std::map<std::string, icon_tuning> read_cache(const char *path)
{
    std::map<std::string, icon_tuning> m;
    if (!path) return m;
    FILE *f = fopen(path, "r");
    if (!f) return m;
    char line[512];
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        int nx, th, nz, sl, op, g, c;
        double us;
        if (sscanf(line, "%d %d %d %d %d %d %d %lf", &nx, &th, &nz, &sl, &op, &g, &c, &us) == 8) {
            std::ostringstream k;
            k << nx << ' ' << th << ' ' << nz << ' ' << sl << ' ' << op;
            m[k.str()] = icon_tuning{g, c, us, 2};
        }
    }
    fclose(f);
    return m;
}

// Times `iters` iterations of one candidate plan on `S` slices of constant
// rows (the FFT work does not depend on the values): device microseconds
// per slice and iteration, or a negative value when the plan cannot be made.
double time_candidate(const icon_series &s, int device, int op, int group, int chunk)
{
    std::vector<float> tilts(s.tilt_deg, s.tilt_deg + s.ntilt);
    icon_geometry g{s.nx, thickness_of(s), s.ntilt, tilts.data(), chunk, device};
    icon_plan *p = nullptr;
    if (iconx::plan_create_group(&g, group, &p) != ICON_OK) return -1.0;
    if (iconx::plan_group(p) != group || icon_plan_set_operator(p, op) != ICON_OK) {
        icon_plan_destroy(p);
        return -1.0;
    }
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double us = -1.0;
    const icon_solve_cfg cfg{0, 16, 0, 2, 0.0f};
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
        cudaEventCreate(&e1) == cudaSuccess &&
        cudaMemsetAsync(iconx::plan_rows_buffer(p), 0x3c, sizeof(float) * (size_t)chunk * s.ntilt * s.nx, st) ==
            cudaSuccess &&
        iconx::plan_stage_in(p, iconx::plan_rows_buffer(p), chunk, st) == ICON_OK) {
        bool ok = true;
        for (int it = 0; it < 3 && ok; ++it) ok = iconx::plan_iteration(p, chunk, it, &cfg, st) == ICON_OK;
        const int n = 8;
        ok = ok && cudaEventRecord(e0, st) == cudaSuccess;
        for (int it = 3; it < 3 + n && ok; ++it) ok = iconx::plan_iteration(p, chunk, it, &cfg, st) == ICON_OK;
        ok = ok && cudaEventRecord(e1, st) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
        float ms = 0.f;
        if (ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) us = 1e3 * ms / ((double)n * chunk);
    }
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    icon_plan_destroy(p);
    return us;
}

// Candidates: every group size up to the size's default, times chunk sizes
// of 64, 128 and 256 slices (capped at the series' slices).
icon_tuning tune_series(const icon_series &s, int device, int op)
{
    const int n0 = 2 * (1 << (int)std::ceil(std::log2((double)s.nx)));
    const int th = thickness_of(s);
    const int n1 = 2 * (1 << (int)std::ceil(std::log2((double)th)));
    const int nmax = std::max(n0, n1);
    const int gmax = nmax <= 2048 ? 8 : (nmax <= 4096 ? 4 : 2);
    icon_tuning best{0, 0, 0.0, 1};
    std::vector<int> chunks;
    for (int c : {64, 128, 256}) {
        const int cc = std::min(c, s.slices);
        if (std::find(chunks.begin(), chunks.end(), cc) == chunks.end()) chunks.push_back(cc);
    }
    for (int g = gmax; g >= 2; g /= 2)
        for (int c : chunks) {
            if (g > c && g != gmax) continue;
            const double us = time_candidate(s, device, op, g, c);
            if (us > 0 && (best.group == 0 || us < best.us_per_slice_iteration)) best = icon_tuning{g, c, us, 1};
        }
    return best;
}

// Graph key of an iteration: slices, whether it applies the previous
// update, the previous and the current iteration's clamp.
long long graph_key(int S, bool upd, bool clamp_prev, bool clamp_cur)
{
    return (long long)S * 8 + (upd ? 4 : 0) + (clamp_prev ? 2 : 0) + (clamp_cur ? 1 : 0);
}

}  // namespace

struct icon_batch {
    int device = 0, op = ICON_OPERATOR_TOEPLITZ;
    std::vector<icon_series> series;
    std::vector<std::vector<float>> tilts;
    std::vector<icon_tuning> tuning;
    std::vector<icon_plan *> plans;
    std::vector<cudaStream_t> streams;
    cudaStream_t capture = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<std::map<long long, cudaGraphExec_t>> graphs;
    int g_dtype = -1;        // data type and threshold the graphs were captured with
    float g_thr = 0.f;
    void drop_graphs()
    {
        for (auto &m : graphs) {
            for (auto &kv : m) cudaGraphExecDestroy(kv.second);
            m.clear();
        }
    }
    ~icon_batch()
    {
        DevGuard g(device);
        for (auto &m : graphs)
            for (auto &kv : m) cudaGraphExecDestroy(kv.second);
        for (auto s : streams)
            if (s) cudaStreamDestroy(s);
        if (capture) cudaStreamDestroy(capture);
        if (done) cudaEventDestroy(done);
        for (auto p : plans)
            if (p) icon_plan_destroy(p);
    }
    // The graph of one iteration of series k (captured on first use).
    icon_status graph(int k, int S, int it, const icon_solve_cfg *cfg, cudaGraphExec_t *out)
    {
        const int a = cfg->infr_before, iters = a + cfg->icon + cfg->infr_after;
        auto clamp_at = [&](int i) { return a <= i && i < iters - cfg->infr_after; };
        const long long key = graph_key(S, it > 0, it > 0 && clamp_at(it - 1), clamp_at(it));
        auto f = graphs[k].find(key);
        if (f != graphs[k].end()) {
            *out = f->second;
            return ICON_OK;
        }
        B_CUDA(cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal));
        icon_status rc = iconx::plan_iteration(plans[k], S, it, cfg, capture);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(capture, &g);
        if (rc != ICON_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail_msg(ICON_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t x = nullptr;
        e = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail_msg(ICON_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        graphs[k][key] = x;
        *out = x;
        return ICON_OK;
    }
};

extern "C" {

icon_status icon_batch_create(const icon_series *series, int nseries, int device, int op, const char *tune_cache,
                              int tune, icon_batch **out)
{
    if (!series || nseries < 1 || !out) return fail_msg(ICON_ERR_INVALID, "need at least one series");
    if (op != ICON_OPERATOR_NUFFT && op != ICON_OPERATOR_TOEPLITZ) return fail_msg(ICON_ERR_INVALID, "unknown operator");
    *out = nullptr;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail_msg(ICON_ERR_CUDA, "no CUDA device");
    for (int k = 0; k < nseries; ++k)
        if (series[k].slices < 1 || !series[k].tilt_deg || series[k].ntilt < 2)
            return fail_msg(ICON_ERR_INVALID, "series " + std::to_string(k) + ": bad slices or tilts");
    DevGuard guard(device);
    std::unique_ptr<icon_batch> b(new icon_batch);
    b->device = device;
    b->op = op;
    b->series.assign(series, series + nseries);
    b->tilts.resize(nseries);
    for (int k = 0; k < nseries; ++k) {
        b->tilts[k].assign(series[k].tilt_deg, series[k].tilt_deg + series[k].ntilt);
        b->series[k].tilt_deg = b->tilts[k].data();
    }
    auto cache = read_cache(tune_cache);
    FILE *append = nullptr;
    for (int k = 0; k < nseries; ++k) {
        const icon_series &s = b->series[k];
        const std::string key = shape_key(s, op);
        icon_tuning t{0, std::min(s.slices, 128), 0.0, 0};
        auto f = cache.find(key);
        if (f != cache.end()) {
            t = f->second;
        } else if (tune) {
            icon_tuning r = tune_series(s, device, op);
            if (r.group > 0) {
                t = r;
                cache[key] = r;
                if (tune == 2 && tune_cache) {
                    if (!append) append = fopen(tune_cache, "a");
                    if (append)
                        fprintf(append, "%s %d %d %.4f\n", key.c_str(), r.group, r.chunk, r.us_per_slice_iteration);
                }
            }
        }
        t.chunk = std::max(1, std::min(t.chunk, s.slices));
        b->tuning.push_back(t);
    }
    if (append) fclose(append);
    b->plans.assign(nseries, nullptr);
    b->streams.assign(nseries, nullptr);
    b->graphs.resize(nseries);
    for (int k = 0; k < nseries; ++k) {
        const icon_series &s = b->series[k];
        icon_geometry g{s.nx, thickness_of(s), s.ntilt, s.tilt_deg, b->tuning[k].chunk, device};
        B_TRY(iconx::plan_create_group(&g, b->tuning[k].group, &b->plans[k]));
        B_TRY(icon_plan_set_operator(b->plans[k], op));
        b->tuning[k].group = iconx::plan_group(b->plans[k]);
        B_CUDA(cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking));
    }
    B_CUDA(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
    B_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    *out = b.release();
    return ICON_OK;
}

icon_status icon_batch_destroy(icon_batch *b)
{
    delete b;
    return ICON_OK;
}

icon_status icon_batch_tuning(const icon_batch *b, int k, icon_tuning *out)
{
    if (!b || !out || k < 0 || k >= (int)b->series.size()) return fail_msg(ICON_ERR_INVALID, "bad series index");
    *out = b->tuning[k];
    return ICON_OK;
}

static icon_status batch_run(icon_batch *b, const icon_solve_cfg *cfg, const float *const *h_rows, float *const *h_m,
                             int concurrent, int *where);

icon_status icon_batch_reconstruct_host(icon_batch *b, const icon_solve_cfg *cfg, const float *const *h_rows,
                                        float *const *h_m, int concurrent)
{
    int where = -1;
    icon_status rc = batch_run(b, cfg, h_rows, h_m, concurrent, &where);
    if (rc != ICON_OK && where >= 0) {
        const icon_series &s = b->series[where];
        std::ostringstream m;
        m << "series " << where << " (nx " << s.nx << ", thickness " << thickness_of(s) << ", " << s.ntilt
          << " tilts, " << s.slices << " slices, group " << b->tuning[where].group << ", chunk "
          << b->tuning[where].chunk << "): " << icon_last_error();
        return fail_msg(rc, m.str());
    }
    return rc;
}

static icon_status batch_run(icon_batch *b, const icon_solve_cfg *cfg, const float *const *h_rows, float *const *h_m,
                             int concurrent, int *where)
{
    if (!b || !cfg || !h_rows || !h_m) return fail_msg(ICON_ERR_INVALID, "null argument");
    if (cfg->infr_before < 0 || cfg->icon < 0 || cfg->infr_after < 0)
        return fail_msg(ICON_ERR_INVALID, "negative iteration count");
    const int ns = (int)b->series.size();
    for (int k = 0; k < ns; ++k)
        if (!h_rows[k] || !h_m[k]) return fail_msg(ICON_ERR_INVALID, "null buffer of series " + std::to_string(k));
    DevGuard guard(b->device);
    const int iters = cfg->infr_before + cfg->icon + cfg->infr_after;
    if (cfg->data_type != b->g_dtype || cfg->threshold != b->g_thr) {   // the graphs hold these as kernel arguments
        b->drop_graphs();
        b->g_dtype = cfg->data_type;
        b->g_thr = cfg->threshold;
    }
    // Per series: next slice, slices of the current chunk, next iteration.
    struct State {
        int s0 = 0, S = 0, it = 0;
        bool active = true;
    };
    std::vector<State> st(ns);
    auto begin_chunk = [&](int k) -> icon_status {
        *where = k;
        const icon_series &s = b->series[k];
        State &q = st[k];
        q.S = std::min(b->tuning[k].chunk, s.slices - q.s0);
        q.it = 0;
        const size_t R = (size_t)s.ntilt * s.nx;
        float *rows = iconx::plan_rows_buffer(b->plans[k]);
        B_CUDA(cudaMemcpyAsync(rows, h_rows[k] + (size_t)q.s0 * R, sizeof(float) * R * q.S, cudaMemcpyHostToDevice,
                               b->streams[k]));
        return iconx::plan_stage_in(b->plans[k], rows, q.S, b->streams[k]);
    };
    auto end_chunk = [&](int k) -> icon_status {
        *where = k;
        const icon_series &s = b->series[k];
        State &q = st[k];
        const size_t NN = (size_t)s.nx * thickness_of(s);
        float *outb = iconx::plan_out_buffer(b->plans[k]);
        B_TRY(iconx::plan_stage_out(b->plans[k], q.S, cfg, outb, b->streams[k]));
        B_CUDA(cudaMemcpyAsync(h_m[k] + (size_t)q.s0 * NN, outb, sizeof(float) * NN * q.S, cudaMemcpyDeviceToHost,
                               b->streams[k]));
        q.s0 += q.S;
        q.active = q.s0 < s.slices;
        return ICON_OK;
    };
    if (!concurrent) {
        // One series after another, direct launches on its stream.
        for (int k = 0; k < ns; ++k) {
            while (st[k].active) {
                *where = k;
                B_TRY(begin_chunk(k));
                for (int it = 0; it < iters; ++it)
                    B_TRY(iconx::plan_iteration(b->plans[k], st[k].S, it, cfg, b->streams[k]));
                B_TRY(end_chunk(k));
            }
            B_CUDA(cudaStreamSynchronize(b->streams[k]));
        }
        *where = -1;
        return ICON_OK;
    }
    // Round-robin: every active series gets its next iteration (one graph
    // launch) in turn, so all series' streams have work queued at once.
    int left = ns;
    for (int k = 0; k < ns; ++k) B_TRY(begin_chunk(k));
    while (left > 0) {
        for (int k = 0; k < ns; ++k) {
            State &q = st[k];
            if (!q.active) continue;
            if (q.it < iters) {
                *where = k;
                cudaGraphExec_t x = nullptr;
                B_TRY(b->graph(k, q.S, q.it, cfg, &x));
                B_CUDA(cudaGraphLaunch(x, b->streams[k]));
                ++q.it;
            }
            if (q.it == iters) {
                B_TRY(end_chunk(k));
                if (q.active) B_TRY(begin_chunk(k));
                else --left;
            }
        }
    }
    for (int k = 0; k < ns; ++k) {
        *where = k;
        B_CUDA(cudaStreamSynchronize(b->streams[k]));
    }
    *where = -1;
    return ICON_OK;
}

}  // extern "C"
