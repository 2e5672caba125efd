/*
 * icon_oracle_geom.c -- precision-independent geometry of the ICON path:
 * grid sizes, window parameters, node positions and density weights.
 *
 * TEST INFRASTRUCTURE ONLY (see icon_oracle.h).  These values define the
 * operator A itself, so both the FP64 and FP32 oracles use the float values the
 * reference computes.  Built with -ffp-contract=off so that no multiply-add is
 * fused where the reference rounds twice.
 */
#include <math.h>
#include <stdlib.h>
#include "icon_oracle.h"

/* The reference's PI macro (nufft_gpu_v8.cuh:8) and the px2D pi (px2D.cuh:8). */
#define REF_PI 3.1415926535898
#define REF_PI_PX2D 3.14159265

/* MainCode.cu:66-71: uptop = pow(2,ceil(log10(N)/log10(2.0))) stored as float,
 * thita = 2.0*uptop/(double)N stored as float, n = ceil(thita*N) in float.
 * NU:471-476: b = 2*thita*m/((2*thita-1)*PI), bf = 1/sqrt(PI*b), both float. */
void ora_grid_params(int N, float *theta, int *n, float *b, float *bf)
{
    float uptop = (float)pow(2, ceil(log10((double)N) / log10(2.0)));
    float th = (float)(2.0 * uptop / (double)N);
    float prod = th * (float)N;               /* float*int -> float */
    int nn = (int)ceilf(prod);
    float bb = (float)((double)(2 * th * ORA_M) / ((double)(2 * th - 1) * REF_PI));
    float bff = (float)(1.0 / sqrt(REF_PI * (double)bb));
    if (theta) *theta = th;
    if (n) *n = nn;
    if (b) *b = bb;
    if (bf) *bf = bff;
}

/* px2D.cu:8-26 (TFunction2) and :29-47 (px2D): s_0 = -1/2, s_k = s_{k-1} + 1/nx
 * accumulated in float; x0 = s*cos(angle*pi/180), x1 = s*sin(angle*pi/180)
 * evaluated in double and stored as float. */
void ora_px2d(int nx, int nz, const float *theta_neg, float *xy)
{
    float *s = (float *)malloc(sizeof(float) * (size_t)nx);
    float step = (float)(1.0 / nx);
    s[0] = (float)(-1.0 / 2);
    for (int k = 1; k < nx; k++) s[k] = s[k - 1] + step;
    for (int i = 0; i < nz; i++) {
        double a = (double)theta_neg[i] * REF_PI_PX2D / 180;
        double c = cos(a), sn = sin(a);
        for (int k = 0; k < nx; k++) {
            xy[2 * ((size_t)i * nx + k)] = (float)((double)s[k] * c);
            xy[2 * ((size_t)i * nx + k) + 1] = (float)((double)s[k] * sn);
        }
    }
    free(s);
}

/* weight.cu:8-41: w = c*|dtheta*(j-center)| with center = nx/2 (integer), one
 * sided difference doubled at the two end tilts, and 180/(4*nz) at j == center.
 * The difference and its product with (j-center) are float operations. */
void ora_weight(int nx, int nz, const float *t, float *w)
{
    int center = nx / 2;
    for (int i = 0; i < nz; i++) {
        for (int j = 0; j < nx; j++) {
            float v;
            if (j == center) {
                v = (float)(180.0 / (4 * nz));
            } else if (i == 0) {
                float d = (t[i + 1] - t[i]) * (float)(j - center);
                v = (float)(2.0 * fabsf(d));
            } else if (i == nz - 1) {
                float d = (t[i - 1] - t[i]) * (float)(j - center);
                v = (float)(2.0 * fabsf(d));
            } else {
                float d = (t[i - 1] - t[i + 1]) * (float)(j - center);
                v = (float)(1.0 * fabsf(d));
            }
            w[(size_t)i * nx + j] = v;
        }
    }
}
