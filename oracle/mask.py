"""CPU restatement of ICONMask3 (volume assembly with the cross-validation mask).

TEST INFRASTRUCTURE ONLY: the tests compare the library's GPU version with
these functions and with fixtures the reference binary wrote; nothing in the
library imports this module.

Reference: tomography/ICON_GPU_v1.2.9/sourceCode/ICONMask3/
ICONCrossVMaskIn2D_weightOnlyOnSampled.cu (MK below)
  angular steps          MK:996-1016   largest span -> fallback radius;
                                       mean step -> weighting radius r_full
  radius from FRC files  MK:1033-1100  crossV / fullRec, last index >= 0.5
                                       and >= 0.3 (searched from the end)
  sampling mask          MK:1107-1139  one line through the centre per tilt,
                                       rotated by -tilt-90 deg and splatted
                                       bilinearly, summed, clipped at 1
  filter                 MK:369-456    genMask: 1 inside the radius, a
                                       Gaussian roll-off (max with the
                                       sampling mask) out to radius + width,
                                       the sampling mask beyond; times
                                       rr / r_full on sampled frequencies
  per slice              MK:479-600    R2C, times filter, C2R, / (n*n)
  volume                 MK:1162-1220  rows ystart .. ystart+thickness of
                                       each slice, ystart = n/2 - t/2 + zshift
Float and double steps follow the reference; the FFTs here are numpy's in
double precision (the reference uses cuFFT in float).
"""
import math

import numpy as np

PI_180 = 0.01745329252


def angular_steps(tilts):
    t = np.asarray(tilts, np.float32)
    span = float(np.float32(t.max()) - np.float32(t.min()))
    biggest_radius = int(math.ceil(2 * 180.0 / 3.1415926 / span))
    mean = np.float32(0.0)
    for i in range(len(t) - 1):
        mean = np.float32(mean + np.float32(abs(np.float32(t[i + 1] - t[i]))))
    mean = np.float32(mean / np.float32(len(t) - 1))
    return biggest_radius, float(mean)


def radius_rates(n, tilts, radius=None, crossv=None, fullrec=None):
    """(radius05 rate, radius03 rate, explicit radius?) as MK:1025-1106."""
    biggest_radius, _ = angular_steps(tilts)
    if radius is None:
        cv = np.asarray(crossv, np.float32).copy()
        fr = np.asarray(fullrec, np.float32)
        size = len(cv)
        if size < n / 2 - 1 or len(fr) < n / 2 - 1:
            radius = biggest_radius
        else:
            for i in range(size):
                if fr[i] != 0:
                    cv[i] = np.float32(cv[i] / fr[i])
            r05 = next((i for i in range(size - 1, -1, -1) if cv[i] >= 0.5), -1)
            r03 = next((i for i in range(size - 1, -1, -1) if cv[i] >= 0.3), -1)
            if r05 > r03 or r03 == 0:
                radius = biggest_radius
            else:
                return float(np.float32(r05) / np.float32(size)), float(np.float32(r03) / np.float32(size)), False
    return float(np.float32(radius) / np.float32(n / 2.0)), 0.0, True


def sampling_mask(n, tilts):
    """origmask[n][n] (MK:1107-1139)."""
    nx = ny = n
    orig = np.zeros((ny, nx), np.float32)
    for th in np.asarray(tilts, np.float32):
        ang = float(-th - 90) * PI_180
        c, s = np.float32(math.cos(ang)), np.float32(math.sin(ang))
        rot = np.zeros((ny, nx), np.float32)
        i = nx // 2
        for j in range(ny):
            a, b = np.float32(i - nx // 2), np.float32(j - ny // 2)
            xf = np.float32(np.float32(np.float32(a * c) - np.float32(b * s)) + np.float32(nx // 2))
            yf = np.float32(np.float32(np.float32(a * s) + np.float32(b * c)) + np.float32(ny // 2))
            xi, yi = int(xf), int(yf)
            dx, dy = np.float32(xf - np.float32(xi)), np.float32(yf - np.float32(yi))
            one = np.float32(1.0)
            for (yy, xx, w) in ((yi, xi, (one - dx) * (one - dy)), (yi + 1, xi, (one - dx) * dy),
                                (yi, xi + 1, dx * (one - dy)), (yi + 1, xi + 1, dx * dy)):
                if 0 <= xx < nx and 0 <= yy < ny:
                    rot[yy, xx] = np.float32(rot[yy, xx] + np.float32(w))
        orig += rot
    orig[orig > 1] = 1.0
    return orig


def half_filter(n, tilts, rate05, rate03, explicit, gauss_width=None):
    """realMask * weighting on the half spectrum [n][n/2+1] (MK:369-456, 458-468)."""
    orig = sampling_mask(n, tilts)
    _, mean_step = angular_steps(tilts)
    r_full = int(math.ceil(2.0 / (mean_step / 360.0 * 2 * 3.1415926)))
    radius05 = int(float(np.float32(n)) / 2.0 * rate05)
    radius03 = int(float(np.float32(n)) / 2.0 * rate03)
    if not explicit:
        glmax = (radius03 - radius05) if gauss_width is None else gauss_width
    else:
        glmax = int(10.0 * (n / 150.0)) if gauss_width is None else gauss_width
    if glmax < 10.0 * (n / 150.0):
        glmax = int(10.0 * (n / 150.0))
    radius = radius05
    gradius = radius + glmax
    glen = gradius - radius
    c = glen / 3.0
    e0 = math.exp(-(glen * glen) / (2 * c * c))
    nh = n // 2 + 1
    mask = np.ones((n, nh), np.float32)
    weight = np.ones((n, nh), np.float32)
    for j in range(n):
        j1 = (j + n // 2) % n
        for i in range(nh):
            i1 = (i + n // 2) % n
            rr = int(math.sqrt((i1 - n // 2) ** 2 + (j1 - n // 2) ** 2))
            o = float(orig[j1, i1])
            if rr >= radius:
                if rr <= gradius:
                    x = rr - radius
                    w2 = (math.exp(-(x * x) / (2 * c * c)) - e0) / (1 - e0)
                    mask[j, i] = np.float32(max(o, w2))
                else:
                    mask[j, i] = np.float32(o)
            if rr > r_full and abs(o) > 0.00001:
                weight[j, i] = np.float32(np.float32(rr) / np.float32(r_full))
    return (mask * weight).astype(np.float32)


def apply(slices, filt, ystart, thickness):
    """slices (S, n, n) -> cropped filtered slices (S, thickness, n)."""
    n = slices.shape[-1]
    out = []
    for sl in np.asarray(slices, np.float64):
        spec = np.fft.rfft2(sl) * filt.astype(np.float64)
        res = np.fft.irfft2(spec, s=(n, n))          # irfft2 divides by n*n
        out.append(res[ystart:ystart + thickness].astype(np.float32))
    return np.stack(out)


def assemble(slices, ystart, thickness):
    return np.ascontiguousarray(np.asarray(slices, np.float32)[:, ystart:ystart + thickness])
