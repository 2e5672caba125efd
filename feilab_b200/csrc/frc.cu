// frc.cu -- Fourier ring correlation on the host, as the reference's
// cross-validation computes it (calFRC_nonsqure, calFRC.cu:93-174, and
// frcSmooth, ICONGPU.cu:59-91).  C ABI in include/icon_tools.h.
#include <cmath>
#include <complex>
#include <vector>

#include "icon_b200.h"
#include "icon_tools.h"

extern "C" void icon_internal_set_error(const char *msg);

namespace {

// 1-D DFT of any length (radix-2 for powers of two, Bluestein otherwise), in
// double; used for the FRC of the cross-validation outputs.
void fft_pow2(std::vector<std::complex<double>> &a, bool inverse)
{
    size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        double ang = 2 * M_PI / (double)len * (inverse ? 1 : -1);
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                std::complex<double> w = std::polar(1.0, ang * (double)k);
                std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

void fft_any(std::vector<std::complex<double>> &a)
{
    size_t n = a.size();
    if ((n & (n - 1)) == 0) {
        fft_pow2(a, false);
        return;
    }
    size_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    std::vector<std::complex<double>> w(n), x(m), y(m);
    for (size_t k = 0; k < n; ++k) w[k] = std::polar(1.0, -M_PI * (double)((k * k) % (2 * n)) / (double)n);
    for (size_t k = 0; k < n; ++k) x[k] = a[k] * w[k];
    y[0] = std::conj(w[0]);
    for (size_t k = 1; k < n; ++k) y[k] = y[m - k] = std::conj(w[k]);
    fft_pow2(x, false);
    fft_pow2(y, false);
    for (size_t i = 0; i < m; ++i) x[i] *= y[i];
    fft_pow2(x, true);
    for (size_t k = 0; k < n; ++k) a[k] = x[k] * w[k] / (double)m;
}

// calFRC_nonsqure (calFRC.cu:93-174): 2-D FFT of two nx-by-ny images (nx
// fastest), ring sums with the y frequency scaled by (nx/ny)^2, FRC per ring
// r < nx/2, frc[0] = 1.
std::vector<float> frc_nonsquare(const std::vector<float> &a, const std::vector<float> &b, int nx, int ny)
{
    auto fft2 = [&](const std::vector<float> &img) {
        std::vector<std::complex<double>> f((size_t)nx * ny);
        for (size_t i = 0; i < f.size(); ++i) f[i] = img[i];
        std::vector<std::complex<double>> line(nx);
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) line[i] = f[(size_t)j * nx + i];
            fft_any(line);
            for (int i = 0; i < nx; ++i) f[(size_t)j * nx + i] = line[i];
        }
        std::vector<std::complex<double>> col(ny);
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < ny; ++j) col[j] = f[(size_t)j * nx + i];
            fft_any(col);
            for (int j = 0; j < ny; ++j) f[(size_t)j * nx + i] = col[j];
        }
        return f;
    };
    std::vector<std::complex<double>> A = fft2(a), Bf = fft2(b);
    int nx2 = nx / 2, ny2 = ny / 2;
    std::vector<double> up(nx2 + 1, 0.0), l1(nx2 + 1, 0.0), l2(nx2 + 1, 0.0);
    float damp = ((float)nx / (float)ny) * ((float)nx / (float)ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int i1 = (i + nx2) % nx, j1 = (j + ny2) % ny;
            int r = (int)std::floor(std::sqrt((float)((i1 - nx2) * (i1 - nx2)) + (float)((j1 - ny2) * (j1 - ny2)) * damp));
            if (r < nx2) {
                std::complex<double> p = A[(size_t)j * nx + i], q = Bf[(size_t)j * nx + i];
                up[r] += p.real() * q.real() + p.imag() * q.imag();
                l1[r] += std::norm(p);
                l2[r] += std::norm(q);
            }
        }
    std::vector<float> frc(nx2 > 0 ? nx2 : 1, 0.f);
    frc[0] = 1.f;
    for (int i = 1; i < nx2; ++i) {
        double d = std::sqrt(l1[i]) * std::sqrt(l2[i]);
        frc[i] = d != 0 ? (float)(up[i] / d) : 0.f;
    }
    return frc;
}

// frcSmooth (ICONGPU.cu:59-91): moving average over `overlap` bins.
void frc_smooth(std::vector<float> &frc, int size, int overlap)
{
    std::vector<float> t(size);
    for (int i = 0; i < size; ++i) {
        int jbe = i - overlap / 2;
        if (jbe < 0) jbe = 0;
        int jen = jbe + overlap;
        if (jen > size - 1) {
            jbe -= jen - size + 1;
            jen = size - 1;
        }
        if (jbe < 0) jbe = 0;
        float sum = 0;
        int num = 0;
        for (int j = jbe; j < jen; ++j) {
            sum += frc[j];
            ++num;
        }
        t[i] = num ? sum / num : 0.f;
    }
    for (int i = 0; i < size; ++i) frc[i] = t[i];
}

}  // namespace

extern "C" icon_status icon_frc(const float *a, const float *b, int nx, int ny, int smooth_overlap, float *frc_out)
{
    if (!a || !b || !frc_out || nx < 2 || ny < 1) {
        icon_internal_set_error("icon_frc: bad argument");
        return ICON_ERR_INVALID;
    }
    std::vector<float> va(a, a + (size_t)nx * ny), vb(b, b + (size_t)nx * ny);
    std::vector<float> f = frc_nonsquare(va, vb, nx, ny);
    if (smooth_overlap > 0) frc_smooth(f, nx / 2, smooth_overlap);
    for (int i = 0; i < nx / 2; ++i) frc_out[i] = f[i];
    return ICON_OK;
}
