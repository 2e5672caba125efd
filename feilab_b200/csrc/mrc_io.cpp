// mrc_io.cpp -- MRC reading and writing for the icon-gpu tool (see mrc_io.h).
#include "mrc_io.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace {

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

size_t mode_bytes(int mode)
{
    switch (mode) {
    case MRC_BYTE: return 1;
    case MRC_SHORT:
    case MRC_USHORT: return 2;
    case MRC_FLOAT: return 4;
    default: return 0;
    }
}

}  // namespace

bool mrc_read_header(const std::string &path, MrcHeader &h, std::string &err)
{
    File fl;
    fl.f = fopen(path.c_str(), "rb");
    if (!fl.f) {
        err = "cannot open " + path;
        return false;
    }
    if (fread(&h, sizeof h, 1, fl.f) != 1) {
        err = "short MRC header in " + path;
        return false;
    }
    if (h.nx <= 0 || h.ny <= 0 || h.nz <= 0 || mode_bytes(h.mode) == 0) {
        err = "unsupported MRC file " + path + " (mode " + std::to_string(h.mode) + ")";
        return false;
    }
    return true;
}

bool mrc_read_sections_into(const std::string &path, const MrcHeader &h, int z0, int z1, float *out,
                            std::string &err)
{
    File fl;
    fl.f = fopen(path.c_str(), "rb");
    if (!fl.f) {
        err = "cannot open " + path;
        return false;
    }
    size_t ps = mode_bytes(h.mode), sec = (size_t)h.nx * h.ny;
    fseeko(fl.f, 0, SEEK_END);
    long long fsize = ftello(fl.f);
    long long dsize = (long long)sec * h.nz * ps;
    long long start = fsize - dsize;
    if (start < 1024) {
        err = "MRC file " + path + " is shorter than its header says";
        return false;
    }
    if (z0 < 0 || z1 > h.nz || z0 > z1) {
        err = "section range out of bounds";
        return false;
    }
    size_t n = sec * (size_t)(z1 - z0);
    fseeko(fl.f, start + (long long)z0 * sec * ps, SEEK_SET);
    if (h.mode == MRC_FLOAT) {                // straight into the caller's buffer
        if (n && fread(out, 4, n, fl.f) != n) {
            err = "short read of " + path;
            return false;
        }
        return true;
    }
    // Integer modes: read in blocks of one section and convert.
    std::vector<unsigned char> raw(sec * ps);
    for (size_t done = 0; done < n; done += sec) {
        if (fread(raw.data(), ps, sec, fl.f) != sec) {
            err = "short read of " + path;
            return false;
        }
        float *o = out + done;
        switch (h.mode) {
        case MRC_BYTE:
            for (size_t i = 0; i < sec; ++i) o[i] = (float)raw[i];
            break;
        case MRC_SHORT:
            for (size_t i = 0; i < sec; ++i) {
                int16_t v;
                std::memcpy(&v, &raw[2 * i], 2);
                o[i] = (float)v;
            }
            break;
        default:   // MRC_USHORT
            for (size_t i = 0; i < sec; ++i) {
                uint16_t v;
                std::memcpy(&v, &raw[2 * i], 2);
                o[i] = (float)v;
            }
            break;
        }
    }
    return true;
}

bool mrc_read_sections(const std::string &path, const MrcHeader &h, int z0, int z1, std::vector<float> &out,
                       std::string &err)
{
    if (z0 < 0 || z1 > h.nz || z0 > z1) {
        err = "section range out of bounds";
        return false;
    }
    out.resize((size_t)h.nx * h.ny * (z1 - z0));
    return mrc_read_sections_into(path, h, z0, z1, out.data(), err);
}

bool mrc_write_float(const std::string &path, MrcHeader h, const float *data, std::string &err)
{
    size_t n = (size_t)h.nx * h.ny * h.nz;
    h.mode = MRC_FLOAT;
    double sum = 0.0, amin = n ? data[0] : 0.0, amax = amin;
    size_t sec = (size_t)h.nx * h.ny;
    for (int z = 0; z < h.nz; ++z) {          // per-section partial sums, as mrc_update_head
        double s = 0.0;
        for (size_t i = 0; i < sec; ++i) {
            double v = data[z * sec + i];
            if (v > amax) amax = v;
            if (v < amin) amin = v;
            s += v;
        }
        sum += s;
    }
    double mean = n ? sum / (double)n : 0.0;
    double sd = 0.0;
    for (int z = 0; z < h.nz; ++z) {
        double s = 0.0;
        for (size_t i = 0; i < sec; ++i) {
            double d = data[z * sec + i] - mean;
            s += d * d;
        }
        sd += s;
    }
    h.amin = (float)amin;
    h.amax = (float)amax;
    h.amean = (float)mean;
    h.rms = (float)(n ? std::sqrt(sd / (double)n) : 0.0);
    File fl;
    fl.f = fopen(path.c_str(), "wb");
    if (!fl.f) {
        err = "cannot create " + path;
        return false;
    }
    bool ok = fwrite(&h, sizeof h, 1, fl.f) == 1;
    if (ok && h.next > 0) {
        std::vector<char> zeros((size_t)h.next, 0);
        ok = fwrite(zeros.data(), 1, zeros.size(), fl.f) == zeros.size();
    }
    if (ok && n) ok = fwrite(data, 4, n, fl.f) == n;
    if (!ok) err = "write failed for " + path;
    return ok;
}
