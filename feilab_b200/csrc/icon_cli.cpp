// icon_cli.cpp -- icon-gpu, a drop-in for the ICON-GPU v1.2.9 command-line
// tool (ICON-GPU/ICONGPU.cu:93-609) on the B200 engine of libicon_b200.
//
// Same flags, spellings, defaults and exit behaviour (-1 on -help or a missing
// parameter, ICONGPU.cu:283-316), same output files:
//   <o>/reconstruction/mid%05d.mrc        one xz-slice per file, X fastest
//                                         (saveMRC_real_inv, saveMRC_real.cu:33-56)
//   <o>/crossValidation/GroundTruth.mrc, fullRec_reProjection.mrc,
//   crossV_reprojection.mrc, fullRec.frc, crossV.frc   (ICONGPU.cu:468-592)
// plus, with --volume FILE, the slices stacked into one MRC volume.
// Slices are reconstructed in batches on each listed GPU; slice ranges are
// split across GPUs in proportion to their SM counts (ICONGPU.cu:393-466).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "icon_b200.h"
#include "icon_tools.h"
#include "icon_warmstart.h"
#include "mrc_io.h"

namespace {

void help()
{
    printf("ICON parameter\n######\n");
    printf("-input (-i) : the aligned tilt series.\n######\n");
    printf("-tiltfile (-t) : the aligned tilt file.\n######\n");
    printf("-outputPath (-o) : the folder for the results; \"crossValidation\" and \"reconstruction\" are created inside.\n######\n");
    printf("-slice (-s) : first and last slice, split by ','. For example 0,511 reconstructs slices 0 to 511.\n######\n");
    printf("-ICONIteration (-iter) : iterations a,b,c: a INFR iterations, b ICON iterations, c INFR iterations.\n######\n");
    printf("-dataType (-d) : 1 for cryoET or plastic embedded ET (signal black), 2 for negative stain (signal white); default 1.\n######\n");
    printf("-threshold (-thr) : the threshold used in ICON, default 0.03 (-0.03 for data type 2).\n######\n");
    printf("-skipCrossValidation (-skipCV) : 1 skips the cross validation and its frc files; default 0.\n######\n");
    printf("-gpu (-g) : the GPUs to use, e.g. 0,2,4,6; default -1, all GPUs.\n######\n");
    printf("-help (-h) : for help.\n");
    printf("long options: --volume FILE (write the slices as one MRC volume), --batch N (slices per GPU batch, default 128),\n"
           "  --loo (cross-validate every tilt in turn: crossValidation/loo/tiltNNN.frc and loo_summary.txt),\n"
           "  --operator nufft|toeplitz (normal operator of the iterations: the Gaussian-window NUFFT pair, default,\n"
           "    or its Toeplitz form, the exact operator as one convolution: faster, within 1e-4 of the default),\n"
           "  --tol T (end the ICON iterations of a batch once every slice's relative step is at most T; default 0,\n"
           "    the full -iter schedule), --resume (keep the slices whose reconstruction/mid%%05d.mrc already exists\n"
           "    with this run's sizes; they are read back, not recomputed),\n"
           "  --window gauss6|kb4 (NUFFT window of the input stage, the reprojections and the NUFFT operator: the\n"
           "    Gaussian of half-width 6, default, or the Kaiser-Bessel window of half-width 4, 8 taps instead of 14;\n"
           "    the leave-one-out sweep of --loo keeps the Gaussian),\n"
           "  --warm-start FILE (start each slice of the reconstruction from the learned network's prediction, weights\n"
           "    file as python -m feilab_b200.warmstart export writes it; the ICON phase ends at --tol, default 0.02,\n"
           "    and every slice whose warm result fails the acceptance test is solved again from zero; the\n"
           "    cross-validation solve always starts from zero)\n");
}

struct Args {
    std::string input, tilt, out, volume;
    int ystart = 0, yend = -1;
    int iters[3] = {0, 0, 0};
    int data_type = 1;
    float threshold = 520.0f;
    int thickness = 0;
    int skip_cv = 0;
    std::vector<int> gpus;
    int batch = 128;
    bool loo = false;
    int op = ICON_OPERATOR_NUFFT;
    double tol = 0.0;
    bool resume = false;
    int window = ICON_WINDOW_GAUSS6;
    std::string warm;   // --warm-start weights file
};

// Per-GPU work: a contiguous slice range.
struct Job {
    int device = 0;
    int y0 = 0, y1 = 0;   // [y0, y1)
    int rc = 0;
    std::string err;
    long long warm_accepted = 0, warm_redone = 0;
};

std::string join(const std::string &a, const std::string &b) { return a + "/" + b; }

// Output side of one GPU's full reconstruction: the batch sink of
// icon_reconstruct_stack_host.  Slices arrive X fastest, so each file is
// written straight from the pinned buffer while the GPU solves the next batch.
struct FullSink {
    const Job *job;
    int ybase;   // slice index of the stack row the batches count from
    const Args *A;
    const MrcHeader *inh;
    int thickness;
    const std::string *recdir;
    std::vector<float> *volume, *rp_full;
    std::chrono::steady_clock::time_point last;
    std::string err;
};

int full_sink(void *ctx, int s0, int count, const float *h_slices, const float *h_reproj)
{
    FullSink &c = *static_cast<FullSink *>(ctx);
    const int nx = c.inh->nx;
    const size_t NN = (size_t)nx * c.thickness;
    auto now = std::chrono::steady_clock::now();
    double dt = std::chrono::duration<double>(now - c.last).count() / count;
    c.last = now;
    for (int s = 0; s < count; ++s) {
        const int y = c.ybase + s0 + s;
        const float *slice = h_slices + (size_t)s * NN;
        MrcHeader oh = *c.inh;                           // saveMRC_real.cu:37-46
        oh.mz = c.inh->mx;
        oh.zlen = c.inh->xlen;
        oh.nx = nx;
        oh.ny = c.thickness;
        oh.nz = 1;
        char name[64];
        snprintf(name, sizeof name, "mid%05d.mrc", y);
        if (!mrc_write_float(join(*c.recdir, name), oh, slice, c.err)) return 1;
        if (c.volume) std::memcpy(&(*c.volume)[(size_t)(y - c.A->ystart) * NN], slice, sizeof(float) * NN);
        std::memcpy(&(*c.rp_full)[(size_t)(y - c.A->ystart) * nx], h_reproj + (size_t)s * nx, sizeof(float) * nx);
        printf("slice %d finished, time %lf\n", y, dt);
    }
    return 0;
}

struct CvSink {
    const Job *job;
    const Args *A;
    int nx;
    std::vector<float> *rp_cv;
};

int cv_sink(void *ctx, int s0, int count, const float *, const float *h_reproj)
{
    CvSink &c = *static_cast<CvSink *>(ctx);
    std::memcpy(&(*c.rp_cv)[(size_t)(c.job->y0 + s0 - c.A->ystart) * c.nx], h_reproj, sizeof(float) * c.nx * count);
    return 0;
}

// One GPU's share: reconstruct slices [y0, y1) (and, unless skipped, the
// cross-validation solve), write the slice files, fill the reprojections.
// The GPU gets the share's rows of every section in one copy (the reference
// reads each slice's rows from the file pixel by pixel, readSlicePart.cu:3-31
// over mrcfile3.c:902-951) and both solves read them from there.
void run_job(Job &job, const Args &A, const MrcHeader &inh, const std::vector<float> &tilts, int thickness,
             const float *stack, int omit, std::vector<float> &rp_full, std::vector<float> &rp_cv,
             std::vector<float> *volume, const std::string &recdir)
{
    const int nx = inh.nx, ny = inh.ny, nz = inh.nz;
    const int S = job.y1 - job.y0;
    if (S <= 0) return;
    icon_solve_cfg cfg{A.iters[0], A.iters[1], A.iters[2], A.data_type, A.threshold};
    const int cap = std::min(A.batch, S);
    auto fail = [&](const std::string &m) {
        job.rc = 1;
        job.err = m + ": " + icon_last_error();
    };
    float *d_stack = nullptr;
    if (icon_stack_upload(job.device, stack, nz, ny, nx, job.y0, S, &d_stack, nullptr) != ICON_OK)
        return fail("stack upload");
    struct Free {
        int dev;
        float *p;
        ~Free() { icon_device_free(dev, p); }
    } free_stack{job.device, d_stack};
    // Full reconstruction (Lib_2D2, MainCode.cu:3-177), in runs of slices
    // still to do (all of them unless --resume found finished ones).
    {
        icon_geometry g{nx, thickness, nz, tilts.data(), cap, job.device, A.window};
        icon_plan *plan = nullptr;
        if (icon_plan_create(&g, &plan) != ICON_OK) return fail("plan");
        struct Destroy {
            icon_plan *p;
            ~Destroy() { icon_plan_destroy(p); }
        } destroy{plan};
        if (icon_plan_set_operator(plan, A.op) != ICON_OK || icon_plan_set_stop(plan, A.tol, 10) != ICON_OK)
            return fail("plan options");
        // --warm-start: the network for this plan (destroyed before the plan).
        struct Net {
            icon_ws *w = nullptr;
            ~Net() { icon_ws_destroy(w); }
        } net;
        if (!A.warm.empty()) {
            icon_warm_cfg wc{A.tol > 0.0 ? A.tol : 0.02, 10, 2.0};
            if (icon_ws_create(plan, std::min(cap, 32), &net.w) != ICON_OK || icon_ws_load(net.w, A.warm.c_str()) != ICON_OK ||
                icon_plan_set_warm_start(plan, net.w, &wc) != ICON_OK)
                return fail("warm start");
        }
        std::vector<char> done(S, 0);
        if (A.resume) {
            // A finished slice: its file exists with this run's sizes; its
            // data fills the volume and its reprojection is recomputed.
            std::vector<float> mine;   // finished slices, [k][N0][N1] (Y fastest)
            std::vector<int> ys;
            const size_t NN = (size_t)nx * thickness;
            std::vector<float> buf;
            for (int s = 0; s < S; ++s) {
                char name[64];
                snprintf(name, sizeof name, "mid%05d.mrc", job.y0 + s);
                MrcHeader h;
                std::string e;
                if (!mrc_read_header(join(recdir, name), h, e) || h.nx != nx || h.ny != thickness || h.nz != 1 ||
                    h.mode != 2)
                    continue;
                buf.resize(NN);
                if (!mrc_read_sections_into(join(recdir, name), h, 0, 1, buf.data(), e)) continue;
                done[s] = 1;
                ys.push_back(job.y0 + s);
                if (volume) std::memcpy(&(*volume)[(size_t)(job.y0 + s - A.ystart) * NN], buf.data(), sizeof(float) * NN);
                const size_t k = mine.size() / NN;
                mine.resize(mine.size() + NN);
                for (int X = 0; X < nx; ++X)
                    for (int Y = 0; Y < thickness; ++Y) mine[k * NN + (size_t)X * thickness + Y] = buf[(size_t)Y * nx + X];
            }
            if (!ys.empty()) {
                // Their reprojections at the smallest-|angle| tilt, as the solve's own.
                std::vector<float> rp(ys.size() * (size_t)nx);
                if (icon_reproject_host(plan, mine.data(), tilts[omit], rp.data(), (int)ys.size(), nullptr) != ICON_OK)
                    return fail("reprojection of finished slices");
                for (size_t k = 0; k < ys.size(); ++k)
                    std::memcpy(&rp_full[(size_t)(ys[k] - A.ystart) * nx], &rp[k * nx], sizeof(float) * nx);
                printf("resume: %zu of %d slices on GPU %d already reconstructed\n", ys.size(), S, job.device);
            }
        }
        FullSink sink{&job, job.y0, &A, &inh, thickness, &recdir, volume, &rp_full, std::chrono::steady_clock::now(), {}};
        for (int r0 = 0; r0 < S;) {
            if (done[r0]) {
                ++r0;
                continue;
            }
            int r1 = r0;
            while (r1 < S && !done[r1]) ++r1;
            sink.ybase = job.y0 + r0;
            icon_status rc = icon_reconstruct_stack_host(plan, &cfg, d_stack, S, r0, -1, r1 - r0,
                                                         ICON_OUT_SLICES | ICON_OUT_REPROJECTION, full_sink, &sink,
                                                         nullptr);
            if (rc != ICON_OK) {
                job.rc = 1;
                job.err = sink.err.empty() ? std::string("reconstruction: ") + icon_last_error() : sink.err;
                return;
            }
            r0 = r1;
        }
        if (net.w) icon_plan_warm_counts(plan, &job.warm_accepted, &job.warm_redone);
    }
    if (A.skip_cv) return;
    // Cross-validation solve without the smallest-|angle| tilt, reprojected
    // at that tilt (Lib_2D_crossV2, MainCode_crossV.cu:3-189); the stack's
    // section `omit` is skipped on the device.
    std::vector<float> t2;
    for (int i = 0; i < nz; ++i)
        if (i != omit) t2.push_back(tilts[i]);
    icon_geometry g{nx, thickness, nz - 1, t2.data(), cap, job.device, A.window};
    icon_plan *plan = nullptr;
    if (icon_plan_create(&g, &plan) != ICON_OK) return fail("cross-validation plan");
    if (icon_plan_set_reprojection(plan, tilts[omit]) != ICON_OK || icon_plan_set_operator(plan, A.op) != ICON_OK ||
        icon_plan_set_stop(plan, A.tol, 10) != ICON_OK) {
        icon_plan_destroy(plan);
        return fail("cross-validation reprojection angle");
    }
    CvSink sink{&job, &A, nx, &rp_cv};
    icon_status rc = icon_reconstruct_stack_host(plan, &cfg, d_stack, S, 0, omit, S, ICON_OUT_REPROJECTION, cv_sink,
                                                 &sink, nullptr);
    icon_plan_destroy(plan);
    if (rc != ICON_OK) fail("cross-validation reconstruction");
}

bool next_arg(int argc, char **argv, int &i, std::string &v)
{
    if (i + 1 >= argc) return false;
    v = argv[++i];
    ++i;
    return true;
}

}  // namespace

int main(int argc, char **argv)
{
    Args A;
    bool mark[10] = {false, false, false, false, false, true, true, true, true, true};   // ICONGPU.cu:142-149
    int ndev = 0;
    std::vector<int> sm(256, 0);
    icon_devices(&ndev, sm.data(), 256);
    printf("##################\n%d GPU(s) are detected in the system!\n", ndev);
    for (int d = 0; d < ndev; ++d) A.gpus.push_back(d);
    int i = 1;
    while (i < argc) {
        std::string a = argv[i], v;
        if (a.size() > 2 && a[0] == '-' && a[1] == '-') {               // long options of this tool
            if (a == "--volume" && next_arg(argc, argv, i, v)) A.volume = v;
            else if (a == "--batch" && next_arg(argc, argv, i, v)) A.batch = std::max(1, atoi(v.c_str()));
            else if (a == "--loo") { A.loo = true; ++i; }
            else if (a == "--resume") { A.resume = true; ++i; }
            else if (a == "--tol" && next_arg(argc, argv, i, v)) A.tol = std::max(0.0, atof(v.c_str()));
            else if (a == "--operator" && next_arg(argc, argv, i, v) && (v == "nufft" || v == "toeplitz"))
                A.op = v == "toeplitz" ? ICON_OPERATOR_TOEPLITZ : ICON_OPERATOR_NUFFT;
            else if (a == "--warm-start" && next_arg(argc, argv, i, v)) A.warm = v;
            else if (a == "--window" && next_arg(argc, argv, i, v) && (v == "gauss6" || v == "kb4"))
                A.window = v == "kb4" ? ICON_WINDOW_KB4 : ICON_WINDOW_GAUSS6;
            else if (a == "--help") { help(); return -1; }
            else { printf("parameter error!\n Please use -help to see the manual\n"); return -1; }
            continue;
        }
        if (a[0] != '-') { ++i; continue; }
        std::string k = a.substr(1);
        bool needs = (k == "input" || k == "i" || k == "tiltfile" || k == "t" || k == "outputPath" || k == "o" ||
                      k == "slice" || k == "s" || k == "ICONIteration" || k == "iter" || k == "dataType" ||
                      k == "d" || k == "threshold" || k == "thr" || k == "gpu" || k == "g" || k == "thickness" ||
                      k == "thi" || k == "skipCrossValidation" || k == "skipCV");
        if (k == "help" || k == "h") {
            help();
            return -1;
        }
        if (!needs) { ++i; continue; }
        if (!next_arg(argc, argv, i, v)) { printf("parameter error!\n Please use -help to see the manual\n"); return -1; }
        if (k == "input" || k == "i") { A.input = v; mark[0] = true; }
        else if (k == "tiltfile" || k == "t") { A.tilt = v; mark[1] = true; }
        else if (k == "outputPath" || k == "o") { A.out = v; mark[2] = true; }
        else if (k == "slice" || k == "s") { if (sscanf(v.c_str(), "%d,%d", &A.ystart, &A.yend) == 2) mark[3] = true; }
        else if (k == "ICONIteration" || k == "iter") {
            if (sscanf(v.c_str(), "%d,%d,%d", &A.iters[0], &A.iters[1], &A.iters[2]) == 3) mark[4] = true;
        }
        else if (k == "dataType" || k == "d") A.data_type = atoi(v.c_str());
        else if (k == "threshold" || k == "thr") A.threshold = (float)atof(v.c_str());
        else if (k == "thickness" || k == "thi") A.thickness = atoi(v.c_str());
        else if (k == "skipCrossValidation" || k == "skipCV") A.skip_cv = atoi(v.c_str());
        else if (k == "gpu" || k == "g") {                             // ICONGPU.cu:231-263
            std::vector<int> list;
            size_t p = 0;
            while (p <= v.size()) {
                size_t q = v.find(',', p);
                std::string tok = v.substr(p, q == std::string::npos ? std::string::npos : q - p);
                int d = atoi(tok.c_str());
                if (d == -1) break;
                list.push_back(d);
                if (q == std::string::npos) break;
                p = q + 1;
            }
            if (!list.empty()) A.gpus = list;
        }
    }
    for (bool m : mark)
        if (!m) {
            printf("parameter error!\n Please use -help to see the manual\n");
            return -1;
        }
    if (std::fabs(A.threshold - 520) < 0.0001) {                       // ICONGPU.cu:317-323
        if (A.data_type == 1) A.threshold = 0.03f;
        if (A.data_type == 2) A.threshold = -0.03f;
    }
    int slicetotal = A.yend - A.ystart + 1;
    printf("parameter:\ninput : %s\ntiltfile : %s\noutputPath : %s\nslice : %d,%d\n", A.input.c_str(), A.tilt.c_str(),
           A.out.c_str(), A.ystart, A.yend);
    printf("ICONIteration : %d,%d,%d\ndataType : %d\nthreshold : %f\n", A.iters[0], A.iters[1], A.iters[2], A.data_type,
           A.threshold);
    if (A.thickness != 0) printf("thickness : %d\n", A.thickness);
    int used = std::min((int)A.gpus.size(), std::max(slicetotal, 0));
    printf("use GPU : ");
    for (int d = 0; d < used; ++d) printf("%d ", A.gpus[d]);
    printf("\n");
    if (used == 0) {
        printf("Notice : No GPU is specified to use!\n");
        return 0;
    }
    if (A.skip_cv == 1) printf("skip cross validation!\n");
    std::string cvdir = join(A.out, "crossValidation"), recdir = join(A.out, "reconstruction");
    mkdir(cvdir.c_str(), 0755);
    mkdir(recdir.c_str(), 0755);

    MrcHeader inh;
    std::string err;
    if (!mrc_read_header(A.input, inh, err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    std::vector<float> tilts;
    {
        FILE *tf = fopen(A.tilt.c_str(), "r");
        if (!tf) {
            printf("\nCan not open anglefile!\n");
            return 1;
        }
        float t;
        while (fscanf(tf, "%f", &t) == 1) tilts.push_back(t);
        fclose(tf);
    }
    if ((int)tilts.size() != inh.nz) {
        printf("tilt file has %zu angles but the stack has %d sections\n", tilts.size(), inh.nz);
        return 1;
    }
    if (A.ystart < 0 || A.yend >= inh.ny || slicetotal <= 0) {
        printf("slice range %d,%d outside 0..%d\n", A.ystart, A.yend, inh.ny - 1);
        return 1;
    }
    const int thickness = A.thickness == 0 ? inh.nx : A.thickness;   // MainCode.cu:14-16
    // The whole stack in one read, into pinned memory when it can be had.
    const size_t stack_n = (size_t)inh.nx * inh.ny * inh.nz;
    std::vector<float> stack_pageable;
    float *stack = nullptr;
    if (icon_host_alloc(sizeof(float) * stack_n, (void **)&stack) != ICON_OK) {
        stack_pageable.resize(stack_n);
        stack = stack_pageable.data();
    }
    struct FreeHost {
        float *p;
        bool pinned;
        ~FreeHost()
        {
            if (pinned) icon_host_free(p);
        }
    } free_host{stack, stack_pageable.empty()};
    if (!mrc_read_sections_into(A.input, inh, 0, inh.nz, stack, err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    // Tilt of the smallest |angle| among the negated angles (MainCode.cu:46-49).
    int omit = 0;
    {
        float om = -tilts[0];
        for (int k = 0; k < (int)tilts.size(); ++k)
            if (std::fabs(om) > std::fabs(-tilts[k])) {
                om = -tilts[k];
                omit = k;
            }
    }
    // Slice partition in proportion to SM count (ICONGPU.cu:398-449).
    std::vector<Job> jobs(used);
    {
        double smsum = 0;
        for (int d = 0; d < used; ++d) smsum += std::max(1, A.gpus[d] < (int)sm.size() ? sm[A.gpus[d]] : 1);
        int start = 0;
        for (int d = 0; d < used; ++d) {
            int share = (d == used - 1) ? slicetotal - start
                                        : (int)std::floor(std::max(1, sm[A.gpus[d]]) / smsum * slicetotal);
            jobs[d].device = A.gpus[d];
            jobs[d].y0 = A.ystart + start;
            jobs[d].y1 = A.ystart + start + share;
            printf("thread %d using GPU %d , deals with slices : start %d end %d\n", d, A.gpus[d], jobs[d].y0, jobs[d].y1 - 1);
            start += share;
        }
    }
    std::vector<float> rp_full((size_t)slicetotal * inh.nx, 0.f), rp_cv((size_t)slicetotal * inh.nx, 0.f);
    std::vector<float> volume;
    if (!A.volume.empty()) volume.assign((size_t)slicetotal * inh.nx * thickness, 0.f);
    std::vector<std::thread> threads;
    for (auto &job : jobs)
        threads.emplace_back([&, jp = &job] {
            run_job(*jp, A, inh, tilts, thickness, stack, omit, rp_full, rp_cv, volume.empty() ? nullptr : &volume, recdir);
        });
    for (auto &t : threads) t.join();
    for (auto &job : jobs)
        if (job.rc) {
            printf("running state: fail!\nError message: %s\n", job.err.c_str());
            return 1;
        }
    if (!A.warm.empty()) {
        long long acc = 0, redo = 0;
        for (auto &job : jobs) {
            acc += job.warm_accepted;
            redo += job.warm_redone;
        }
        printf("warm start: %lld of %lld slices accepted, %lld solved again from zero\n", acc, acc + redo, redo);
    }
    if (!A.volume.empty()) {
        MrcHeader vh = inh;
        vh.nx = inh.nx;
        vh.ny = thickness;
        vh.nz = slicetotal;
        vh.mx = inh.nx;
        vh.my = thickness;
        vh.mz = slicetotal;
        vh.next = 0;
        if (!mrc_write_float(A.volume, vh, volume.data(), err)) {
            printf("%s\n", err.c_str());
            return 1;
        }
    }
    if (A.skip_cv == 0) {                                               // ICONGPU.cu:468-592
        std::vector<float> gt((size_t)slicetotal * inh.nx);
        for (int y = A.ystart, k = 0; y <= A.yend; ++y, ++k)
            std::memcpy(&gt[(size_t)k * inh.nx], &stack[((size_t)omit * inh.ny + y) * inh.nx], sizeof(float) * inh.nx);
        auto save2d = [&](const std::string &name, const std::vector<float> &d) {
            MrcHeader oh = inh;                                          // saveMRC_real.cu:9-31
            oh.mz = inh.mx;
            oh.zlen = inh.xlen;
            oh.nx = inh.nx;
            oh.ny = slicetotal;
            oh.nz = 1;
            std::string e;
            if (!mrc_write_float(join(cvdir, name), oh, d.data(), e)) printf("%s\n", e.c_str());
        };
        save2d("GroundTruth.mrc", gt);
        save2d("fullRec_reProjection.mrc", rp_full);
        save2d("crossV_reprojection.mrc", rp_cv);
        int half = inh.nx / 2;
        double resstep = 1.0 / inh.nx;
        auto write_frc = [&](const std::string &name, const std::vector<float> &rp) {
            std::vector<float> frc(half > 0 ? half : 1);
            if (icon_frc(gt.data(), rp.data(), inh.nx, slicetotal, 10, frc.data()) != ICON_OK) return;
            FILE *f = fopen(join(cvdir, name).c_str(), "w");
            if (!f) return;
            for (int k = 0; k < half; ++k) fprintf(f, "%f %f\n", resstep * k, frc[k]);
            fclose(f);
        };
        write_frc("fullRec.frc", rp_full);
        write_frc("crossV.frc", rp_cv);
    }
    if (A.loo) {
        // Every tilt left out in turn, all the left-out solves in one batched
        // schedule on the first listed GPU (icon_loo_sweep); per tilt the
        // smoothed FRC of its reprojections against its projection, written
        // as crossV.frc is.
        const int nz = inh.nz, nx = inh.nx;
        std::vector<float> rows((size_t)slicetotal * nz * nx);
        for (int s = 0; s < slicetotal; ++s)
            for (int i = 0; i < nz; ++i)
                std::memcpy(&rows[((size_t)s * nz + i) * nx], &stack[((size_t)i * inh.ny + A.ystart + s) * nx],
                            sizeof(float) * nx);
        icon_solve_cfg cfg{A.iters[0], A.iters[1], A.iters[2], A.data_type, A.threshold};
        const int half = nx / 2;
        std::vector<float> frc((size_t)nz * (half > 0 ? half : 1));
        std::vector<int> iters(nz);
        if (icon_loo_sweep(rows.data(), nx, thickness, nz, tilts.data(), &cfg, slicetotal, A.batch, 0.0, A.gpus[0],
                           frc.data(), nullptr, iters.data(), A.op) != ICON_OK) {
            printf("running state: fail!\nError message: leave-one-out sweep: %s\n", icon_last_error());
            return 1;
        }
        const std::string loodir = join(cvdir, "loo");
        mkdir(loodir.c_str(), 0755);
        FILE *sum = fopen(join(cvdir, "loo_summary.txt").c_str(), "w");
        if (sum) fprintf(sum, "# tilt index, angle, mean FRC over the rings, iterations\n");
        for (int k = 0; k < nz; ++k) {
            char name[32];
            snprintf(name, sizeof name, "tilt%03d.frc", k);
            FILE *f = fopen(join(loodir, name).c_str(), "w");
            double mean = 0.0;
            for (int q = 0; q < half; ++q) {
                if (f) fprintf(f, "%f %f\n", (1.0 / nx) * q, frc[(size_t)k * half + q]);   // as crossV.frc
                mean += frc[(size_t)k * half + q];
            }
            if (f) fclose(f);
            if (sum) fprintf(sum, "%d %f %f %d\n", k, tilts[k], half > 0 ? mean / half : 0.0, iters[k]);
        }
        if (sum) fclose(sum);
        printf("leave-one-out: %d tilts, FRC files in %s\n", nz, loodir.c_str());
    }
    printf("running state:\n   ICON-GPU finish!\n");
    return 0;
}
