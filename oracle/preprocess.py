"""CPU restatement of ICONPreProcess (stack pre-processing before ICON-GPU).

TEST INFRASTRUCTURE ONLY: the tests compare the library's GPU pre-pass with
these functions and with fixtures the reference binary wrote; nothing in the
library imports this module.

Reference: tomography/ICON_GPU_v1.2.9/sourceCode/ICONPreProcess/ICONPreProcess.c
  minusmode  :29-70   mode of a 256-bin histogram over the central 80 % of
                      the image (10 % margins), subtracted from every pixel
  normalize  :73-85   variance set to 0.33 * thickness / cos(angle)
  main       :216-300 every projection minus its mode; with a tilt file and
                      a thickness, then normalised with angle = -tilt
Arithmetic follows the reference: float pixels, double min/max/step/mode and
double sums; the histogram index floor((v - min) / step) equals 256 for the
largest pixel, which the reference writes one past its array and never
counts, so it is not counted here either.
"""
import math

import numpy as np


def minus_mode(img):
    """img (ny, nx) float32 -> (img - mode as float32, mode)."""
    img = np.asarray(img, np.float32)
    ny, nx = img.shape
    xe, ye = int(nx * 0.1), int(ny * 0.1)
    core = img[ye:ny - ye, xe:nx - xe].astype(np.float64)
    lo, hi = float(core.min()), float(core.max())
    step = (hi - lo) / 256.0
    if step == 0.0:
        mode = lo                      # constant core (the reference divides by zero)
    else:
        idx = np.floor((core - lo) / step).astype(np.int64).ravel()
        hist = np.bincount(idx[idx < 256], minlength=256)
        mode = int(np.argmax(hist)) * step + lo     # first bin with the largest count
    out = (img.astype(np.float64) - mode).astype(np.float32)
    return out, mode


def normalize(img, tilt_deg, thickness):
    """Variance normalisation of one mode-subtracted projection (float32)."""
    img = np.asarray(img, np.float32)
    size = img.size
    angle = np.float32(-np.float32(tilt_deg))                      # thita[k] *= -1
    factor = 0.33 * thickness / math.cos(float(angle) / 180.0 * 3.1415926)
    terms = (img / np.float32(size)).astype(np.float64)            # in[i]/size in float
    mean = float(terms.sum())
    var = float((((img.astype(np.float64) - mean) ** 2) / size).sum())
    return (img.astype(np.float64) / math.sqrt(var) * math.sqrt(factor)).astype(np.float32)


def preprocess(stack, tilts=None, thickness=None):
    """stack (nz, ny, nx) float32 -> pre-processed stack."""
    out = np.empty_like(np.asarray(stack, np.float32))
    for k in range(out.shape[0]):
        out[k], _ = minus_mode(stack[k])
        if tilts is not None and thickness:
            out[k] = normalize(out[k], tilts[k], thickness)
    return out
