/*
 * ref_harness.cu -- drives the reference's own ICON-GPU routines on a test
 * case and dumps every stage, so that the oracle and the CUDA path can be
 * checked against the reference itself.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.sh against the
 * reference sources (tomography/ICON_GPU_v1.2.9/sourceCode/ICON-GPU, compiled
 * unmodified for sm_100a) into oracle/_ref/ref_harness; run on a B200 by
 * tests/golden/make_golden.py.  Nothing here is part of the product.
 *
 * The set-up repeats what Lib_2D2 does before its slice loop
 * (MainCode.cu:38-109) and, per slice, what its loop body does up to the
 * reprojection (MainCode.cu:115-142), calling the reference's routines:
 * readSlicePart, complexMulDoubleCU, cunfft_adjoint_2d2, complexCopyCU,
 * Iteration3, reProject_NFFT2; plus single calls of cunfft_trafo_2d_R2C2,
 * cunfft_trafo_2d2 and cunfft_adjoint_2d2 on given inputs.
 *
 * case file (little endian):
 *   int32[10]  magic 0x49434F4E, nx, thickness, nz, S, a, b, c, dataType, 0
 *   float32    threshold
 *   float32    tilts[nz]            (values as in a .tlt file)
 *   float32    rows[S][nz][nx]      (row y of every tilt, per slice y)
 *   float32    img_r[N0*N1]         (Y fastest)
 *   float32    img_c[N0*N1][2]
 *   float32    f[M][2]
 * output file: float32 arrays, in order
 *   fwd_r[M][2], fwd_c[M][2], adj[N0*N1][2],
 *   then per slice: b[M][2], Ahwb[N0*N1][2], m[N0*N1], reproj[nx]
 */
#include "MainCode.cuh"

static void die(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    exit(2);
}

static void rd(void *p, size_t sz, size_t n, FILE *f)
{
    if (fread(p, sz, n, f) != n) die("short read of case file");
}

static void wr(const void *p, size_t sz, size_t n, FILE *f)
{
    if (fwrite(p, sz, n, f) != n) die("short write of output file");
}

static void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
        exit(3);
    }
}

int main(int argc, char **argv)
{
    if (argc != 4) die("usage: ref_harness case.bin out.bin scratch_dir");
    FILE *cf = fopen(argv[1], "rb");
    if (!cf) die("cannot open case file");
    int hd[10];
    rd(hd, sizeof(int), 10, cf);
    if (hd[0] != 0x49434F4E) die("bad magic");
    int nx = hd[1], thickness = hd[2], nz = hd[3], S = hd[4];
    int ia = hd[5], ib = hd[6], ic = hd[7], dataType = hd[8];
    float threshold;
    rd(&threshold, sizeof(float), 1, cf);
    if (nz > 180) die("more than 180 tilts (the reference's thital buffer)");
    if (nz > thickness) die("nz > thickness overflows the reference's alpha scratch");
    float *tlt = (float *)malloc(sizeof(float) * nz);
    rd(tlt, sizeof(float), nz, cf);
    size_t R = (size_t)nz * nx;
    float *rows = (float *)malloc(sizeof(float) * R * S);
    rd(rows, sizeof(float), R * S, cf);
    int N0 = nx, N1 = thickness, M = nx * nz;
    size_t NN = (size_t)N0 * N1;
    float *img_r = (float *)malloc(sizeof(float) * NN);
    float *img_c = (float *)malloc(sizeof(float) * 2 * NN);
    float *fv = (float *)malloc(sizeof(float) * 2 * (size_t)M);
    rd(img_r, sizeof(float), NN, cf);
    rd(img_c, sizeof(float), 2 * NN, cf);
    rd(fv, sizeof(float), 2 * (size_t)M, cf);
    fclose(cf);

    /* A tilt-series MRC file of S y-rows, so readSlicePart reads it through
     * the reference's own mrc_read_slice(..., 'y', ...). */
    char stack_path[1200];
    snprintf(stack_path, sizeof stack_path, "%s/harness_stack.mrc", argv[3]);
    MrcHeader head;
    memset(&head, 0, sizeof head);
    head.nx = nx;
    head.ny = S;
    head.nz = nz;
    head.mode = MRC_MODE_FLOAT;
    head.mx = nx;
    head.my = S;
    head.mz = nz;
    head.xlen = (float)nx;
    head.ylen = (float)S;
    head.zlen = (float)nz;
    {
        FILE *sf = fopen(stack_path, "wb");
        if (!sf) die("cannot create scratch stack");
        wr(&head, 1024, 1, sf);
        for (int i = 0; i < nz; i++)
            for (int y = 0; y < S; y++)
                wr(rows + (size_t)y * R + (size_t)i * nx, sizeof(float), nx, sf);
        fclose(sf);
    }
    FILE *infile = fopen(stack_path, "rb");
    if (!infile) die("cannot reopen scratch stack");

    /* MainCode.cu:38-49 */
    float *thital = (float *)malloc(180 * sizeof(float));
    for (int i = 0; i < nz; i++) thital[i] = -tlt[i];
    float omitang = thital[0];
    for (int i = 0; i < nz; i++)
        if (fabs(omitang) > fabs(thital[i])) omitang = thital[i];
    /* MainCode.cu:52-58 */
    DATATYPE *weight = (DATATYPE *)malloc(sizeof(DATATYPE) * M);
    Weight(weight, &head, thital);
    GICONPara GP;
    initGICONPara2(&GP, nx, thickness, nz, weight);
    DATATYPE *bpx2D = (DATATYPE *)malloc(2 * sizeof(DATATYPE) * M);
    px2D(bpx2D, &head, thital);
    /* MainCode.cu:60-80 */
    int N[2] = {N0, N1}, n[2];
    DATATYPE thita[2];
    float uptop;
    uptop = pow(2, ceil(log10(N[0]) / log10(2.0)));
    thita[0] = 2.0 * uptop / (double)N[0];
    uptop = pow(2, ceil(log10(N[1]) / log10(2.0)));
    thita[1] = 2.0 * uptop / (double)N[1];
    n[0] = ceil(thita[0] * N[0]);
    n[1] = ceil(thita[1] * N[1]);
    DATATYPE *px1d = (DATATYPE *)malloc(sizeof(DATATYPE) * nx);
    for (int k = 0; k < nx; k++) px1d[k] = ((DATATYPE)k - (DATATYPE)nx / 2.0) / (DATATYPE)nx;
    cunfftplan1d plan1d;
    cunfft_initPlan_1d(&plan1d, nx, thita[0], nx, NFFTM, px1d);
    /* MainCode.cu:88-109 */
    cunfftplan2d2 plan2d, plan2d_reProj;
    DATATYPE *ck2dCU;
    CUFFTDATATYPE *g2dCU;
    cufftHandle planTmp2d;
    ck(cudaMalloc((void **)&ck2dCU, sizeof(DATATYPE) * NN), "malloc ck");
    ck(cudaMalloc((void **)&g2dCU, sizeof(CUFFTDATATYPE) * (size_t)n[0] * n[1]), "malloc g");
    if (cufftPlan2d(&planTmp2d, n[0], n[1], CUFFTTYPE) != CUFFT_SUCCESS) die("cufftPlan2d");
    int flags = CUNFFTPLAN_NO_MALLOC_CK | CUNFFTPLAN_NO_MALLOC_G | CUNFFTPLAN_NO_MALLOC_PLAN | CUNFFTPLAN_NO_PRECOMPUTE;
    cunfft_mallocPlan_2d2(&plan2d, N[0], N[1], thita, M, NFFTM, flags);
    plan2d.ckCU = ck2dCU;
    plan2d.gCU = g2dCU;
    plan2d.planTmp = planTmp2d;
    cunfft_initPlan_2d2(&plan2d, N[0], N[1], thita, M, NFFTM, bpx2D);
    MrcHeader head_line = head;
    head_line.nz = 1;
    float thital2[1] = {omitang};
    px2D(bpx2D, &head_line, thital2);
    cunfft_mallocPlan_2d2(&plan2d_reProj, N[0], N[1], thita, N[0], NFFTM, flags);
    plan2d_reProj.ckCU = ck2dCU;
    plan2d_reProj.gCU = g2dCU;
    plan2d_reProj.planTmp = planTmp2d;
    cunfft_initPlan_2d2(&plan2d_reProj, N[0], N[1], thita, N[0], NFFTM, bpx2D);
    ck(cudaDeviceSynchronize(), "plan set-up");

    FILE *of = fopen(argv[2], "wb");
    if (!of) die("cannot open output");
    float *buf = (float *)malloc(sizeof(float) * 2 * (NN > (size_t)M ? NN : (size_t)M));

    /* Single transforms on given inputs. */
    ck(cudaMemcpy(GP.mCU, img_r, sizeof(float) * NN, cudaMemcpyHostToDevice), "img_r");
    cunfft_trafo_2d_R2C2(plan2d, GP.fCU, GP.mCU);
    ck(cudaMemcpy(buf, GP.fCU, sizeof(float) * 2 * M, cudaMemcpyDeviceToHost), "fwd_r");
    wr(buf, sizeof(float), 2 * (size_t)M, of);
    ck(cudaMemcpy(GP.fhatCU, img_c, sizeof(float) * 2 * NN, cudaMemcpyHostToDevice), "img_c");
    cunfft_trafo_2d2(plan2d, GP.fCU, GP.fhatCU);
    ck(cudaMemcpy(buf, GP.fCU, sizeof(float) * 2 * M, cudaMemcpyDeviceToHost), "fwd_c");
    wr(buf, sizeof(float), 2 * (size_t)M, of);
    ck(cudaMemcpy(GP.fCU, fv, sizeof(float) * 2 * M, cudaMemcpyHostToDevice), "f");
    cunfft_adjoint_2d2(plan2d, GP.fCU, GP.fhatCU);
    ck(cudaMemcpy(buf, GP.fhatCU, sizeof(float) * 2 * NN, cudaMemcpyDeviceToHost), "adj");
    wr(buf, sizeof(float), 2 * NN, of);

    /* The slice loop body of Lib_2D2 (MainCode.cu:115-142). */
    int iternum = ia + ib + ic;
    int before[10] = {ia, ic, 1, dataType, 1, 0, 0, 0, 0, 0};
    float betain[10] = {threshold, (float)thickness, 0, 0, 0, 0, 0, 0, 0, 0};
    DATATYPE *reproj = (DATATYPE *)malloc(sizeof(DATATYPE) * nx);
    for (int y = 0; y < S; y++) {
        readSlicePart(plan1d, GP.fhat1dCU, GP.fCU, infile, &head, y);
        ck(cudaMemcpy(buf, GP.fCU, sizeof(float) * 2 * M, cudaMemcpyDeviceToHost), "b");
        wr(buf, sizeof(float), 2 * (size_t)M, of);
        complexMulDoubleCU<<<dim3(GRIDDIMX, ((M - 1) / BLOCKDIM) / GRIDDIMX + 1), dim3(BLOCKDIMX, BLOCKDIMY)>>>(GP.fCU, GP.weightCU, M);
        cunfft_adjoint_2d2(plan2d, GP.fCU, GP.fhatCU);
        complexCopyCU<<<dim3(GRIDDIMX, ((N0 * N1 - 1) / BLOCKDIM) / GRIDDIMX + 1), dim3(BLOCKDIMX, BLOCKDIMY)>>>(GP.AhwbCU, GP.fhatCU, N0 * N1);
        ck(cudaMemcpy(buf, GP.AhwbCU, sizeof(float) * 2 * NN, cudaMemcpyDeviceToHost), "Ahwb");
        wr(buf, sizeof(float), 2 * NN, of);
        Iteration3(plan2d, GP, &head, iternum, y, argv[3], before, betain);
        ck(cudaMemcpy(buf, GP.mCU, sizeof(float) * NN, cudaMemcpyDeviceToHost), "m");
        wr(buf, sizeof(float), NN, of);
        reProject_NFFT2(plan1d, plan2d_reProj, GP, reproj);
        wr(reproj, sizeof(float), nx, of);
    }
    ck(cudaDeviceSynchronize(), "slice loop");
    fclose(of);
    fclose(infile);
    remove(stack_path);
    printf("ref_harness: %d slices done\n", S);
    return 0;
}
