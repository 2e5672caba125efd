// mrc_io.h -- MRC image files for the icon-gpu command-line tool.
//
// The header is the 1024-byte packed MrcHeader of the reference
// (mrcfile3.h:52-126): it is a file format, so the field order and sizes are
// the same.  Data start at file size minus data size, as mrc_read_slice
// computes it (mrcfile3.c:757-775), so extended headers are skipped.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#pragma pack(push, 1)
struct MrcHeader {
    int32_t nx, ny, nz, mode;
    int32_t nxstart, nystart, nzstart;
    int32_t mx, my, mz;
    float xlen, ylen, zlen;
    float alpha, beta, gamma;
    int32_t mapc, mapr, maps;
    float amin, amax, amean;
    int16_t ispg, nsymbt;
    int32_t next;
    int16_t creatid;
    char blank[30];
    int16_t nint, nreal;
    char blank2[20];
    int32_t imodStamp, imodFlags;
    int16_t idtype, lens, nd1, nd2, vd1, vd2;
    float tiltangles[6];
    float xorg, yorg, zorg;
    char cmap[4];
    char stamp[4];
    float rms;
    int32_t nlabl;
    char labels[10][80];
};
#pragma pack(pop)
static_assert(sizeof(MrcHeader) == 1024, "MRC header must be 1024 bytes");

enum { MRC_BYTE = 0, MRC_SHORT = 1, MRC_FLOAT = 2, MRC_USHORT = 6 };

// Reads the header; false (with a message in err) on failure.
bool mrc_read_header(const std::string &path, MrcHeader &h, std::string &err);

// Reads sections [z0, z1) of the file as float (modes 0, 1, 2, 6), data
// [z - z0][y][x].
bool mrc_read_sections(const std::string &path, const MrcHeader &h, int z0, int z1, std::vector<float> &out,
                       std::string &err);

// The same into out[(z1 - z0) * ny * nx] (e.g. pinned memory): one read for
// float files, one section at a time for the integer modes.
bool mrc_read_sections_into(const std::string &path, const MrcHeader &h, int z0, int z1, float *out,
                            std::string &err);

// Writes a float file with header `h` (nx, ny, nz, mode set by the caller;
// `next` bytes of zeros follow the header) and the statistics amin, amax,
// amean and rms recomputed from the data as mrc_update_head does
// (mrcfile3.c:113-517: double sums, rms = population standard deviation).
bool mrc_write_float(const std::string &path, MrcHeader h, const float *data, std::string &err);
