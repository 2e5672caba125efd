"""MRC image files: the 1024-byte header of the reference's MrcHeader
(mrcfile3.h:52-126, packed, little endian) and float / short / byte data.

Used by tests and benchmarks to write tilt series and read reconstructions;
the command-line tool has its own C++ reader and writer
(feilab_b200/csrc/mrc_io.cpp) with the same layout.
"""
from __future__ import annotations

import numpy as np

HEADER_DTYPE = np.dtype([
    ("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("mode", "<i4"),
    ("nxstart", "<i4"), ("nystart", "<i4"), ("nzstart", "<i4"),
    ("mx", "<i4"), ("my", "<i4"), ("mz", "<i4"),
    ("xlen", "<f4"), ("ylen", "<f4"), ("zlen", "<f4"),
    ("alpha", "<f4"), ("beta", "<f4"), ("gamma", "<f4"),
    ("mapc", "<i4"), ("mapr", "<i4"), ("maps", "<i4"),
    ("amin", "<f4"), ("amax", "<f4"), ("amean", "<f4"),
    ("ispg", "<i2"), ("nsymbt", "<i2"),
    ("next", "<i4"), ("creatid", "<i2"), ("blank", "V30"),
    ("nint", "<i2"), ("nreal", "<i2"), ("blank2", "V20"),
    ("imodStamp", "<i4"), ("imodFlags", "<i4"),
    ("idtype", "<i2"), ("lens", "<i2"), ("nd1", "<i2"), ("nd2", "<i2"), ("vd1", "<i2"), ("vd2", "<i2"),
    ("tiltangles", "<f4", (6,)),
    ("xorg", "<f4"), ("yorg", "<f4"), ("zorg", "<f4"),
    ("cmap", "S4"), ("stamp", "S4"), ("rms", "<f4"),
    ("nlabl", "<i4"), ("labels", "S80", (10,)),
])
assert HEADER_DTYPE.itemsize == 1024

MODE_DTYPE = {0: np.uint8, 1: np.int16, 2: np.float32, 6: np.uint16}


def new_header(nx, ny, nz, mode=2) -> np.ndarray:
    """A header initialised like mrc_init_head (mrcfile3.c:40-90)."""
    h = np.zeros(1, HEADER_DTYPE)[0]
    h["nx"], h["ny"], h["nz"], h["mode"] = nx, ny, nz, mode
    h["mx"], h["my"], h["mz"] = nx, ny, nz
    h["xlen"], h["ylen"], h["zlen"] = nx, ny, nz
    h["alpha"] = h["beta"] = h["gamma"] = 90
    h["mapc"], h["mapr"], h["maps"] = 1, 2, 3
    h["ispg"] = 1
    h["cmap"] = b"MAP "
    h["stamp"] = b"D\x00\x00\x00"
    h["imodStamp"] = 1146047817
    return h


def read(path):
    """Returns (header, data) with data shaped (nz, ny, nx).  The data start
    is file size minus data size, as mrc_read_slice computes it
    (mrcfile3.c:757-775), so extended headers are skipped."""
    with open(path, "rb") as f:
        raw = f.read()
    h = np.frombuffer(raw[:1024], HEADER_DTYPE)[0].copy()
    dt = np.dtype(MODE_DTYPE[int(h["mode"])])
    n = int(h["nx"]) * int(h["ny"]) * int(h["nz"])
    start = len(raw) - n * dt.itemsize
    data = np.frombuffer(raw[start:], dt).reshape(int(h["nz"]), int(h["ny"]), int(h["nx"]))
    return h, data


def stats(data: np.ndarray):
    """amin, amax, amean, rms as mrc_update_head computes them for float data
    (mrcfile3.c:113-517): double sums, rms = sqrt(mean((v - mean)^2))."""
    d = data.astype(np.float64)
    mean = d.sum() / d.size
    return float(d.min()), float(d.max()), float(mean), float(np.sqrt(((d - mean) ** 2).sum() / d.size))


def write(path, data: np.ndarray, header=None):
    """Writes (nz, ny, nx) data (float32 unless the header says otherwise)
    with statistics updated as mrc_update_head does."""
    data = np.asarray(data)
    if data.ndim == 2:
        data = data[None]
    nz, ny, nx = data.shape
    h = new_header(nx, ny, nz) if header is None else header.copy()
    h["nx"], h["ny"], h["nz"] = nx, ny, nz
    dt = np.dtype(MODE_DTYPE[int(h["mode"])])
    arr = np.ascontiguousarray(data.astype(dt, copy=False))
    amin, amax, amean, rms = stats(arr)
    h["amin"], h["amax"], h["amean"], h["rms"] = amin, amax, amean, rms
    nxt = int(h["next"])
    with open(path, "wb") as f:
        f.write(h.tobytes())
        if nxt > 0:
            f.write(b"\x00" * nxt)
        f.write(arr.tobytes())


def write_tilt_series(path, rows: np.ndarray):
    """rows (S, ntilt, nx) -> stack nx x S x ntilt (y = slice index, z = tilt)."""
    r = np.asarray(rows, np.float32)
    write(path, np.ascontiguousarray(r.transpose(1, 0, 2)))


def write_tlt(path, tilts):
    with open(path, "w") as f:
        for t in tilts:
            f.write(f"{float(t):.2f}\n")
