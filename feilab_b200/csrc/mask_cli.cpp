// mask_cli.cpp -- icon-mask: drop-in for the reference's ICONMask3
// (sourceCode/ICONMask3/ICONCrossVMaskIn2D_weightOnlyOnSampled.cu:602-1236,
// MK below): reads the slices reconstruction/midNNNNN.mrc that ICON-GPU (or
// icon-gpu) wrote, filters every slice with the cross-validation mask on the
// GPU (icon_mask_*), keeps `thickness` rows about the centre and writes one
// MRC volume (nx x thickness x slices).  Same flags and defaults:
//
//   icon-mask -i DIR -s first,last -th thickness -t angles.tlt -o vol.mrc
//             (-r radius | -cf crossV.frc -ff fullRec.frc) [-z zshift]
//             [-gw gaussWidth] [-nm 1]
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "icon_tools.h"
#include "mrc_io.h"

namespace {

void help()
{
    printf("ICONMask parameters\n");
    printf("-inputPath (-i) : directory of the reconstructed slices (midNNNNN.mrc)\n");
    printf("-slice (-s) : first,last slice\n");
    printf("-thickness (-th) : thickness of the output volume\n");
    printf("-radius (-r) : mask radius in pixels (instead of -cf and -ff)\n");
    printf("-tiltfile (-t) : tilt angles\n");
    printf("-output (-o) : output volume\n");
    printf("-crossVfrc (-cf) / -fullRecfrc (-ff) : FRC files of the cross validation\n");
    printf("-zshift (-z) : shift of the kept rows (default 0)\n");
    printf("-gaussWidth (-gw) : width of the Gaussian roll-off\n");
    printf("-noMask (-nm) : 1 assembles the volume without the mask\n");
    printf("-help (-h) : this help\n");
}

bool read_frc(const std::string &path, std::vector<float> &v)
{
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return false;
    float a, b;
    while (fscanf(f, "%f %f", &a, &b) == 2) v.push_back(b);
    fclose(f);
    return true;
}

std::string mid_name(const std::string &dir, int i)
{
    char buf[32];
    snprintf(buf, sizeof buf, "/mid%05d.mrc", i);
    return dir + buf;
}

}  // namespace

int main(int argc, char **argv)
{
    std::string in, tlt, out, cf, ff;
    int s0 = 0, s1 = -1, thickness = 0, radius = -1, zshift = 0, gw = 0, nomask = 0;
    bool have[6] = {false, false, false, false, false, false};   // i, s, th, t, o, r
    bool have_cf = false, have_ff = false;
    for (int i = 1; i < argc;) {
        std::string a = argv[i];
        if (a.size() < 2 || a[0] != '-') {
            ++i;
            continue;
        }
        std::string k = a.substr(1);
        if (k == "help" || k == "h") {
            help();
            return 1;   // MK:726-731
        }
        if (i + 1 >= argc) break;
        std::string v = argv[i + 1];
        if (k == "inputPath" || k == "i") { in = v; have[0] = true; }
        else if (k == "slice" || k == "s") { have[1] = sscanf(v.c_str(), "%d,%d", &s0, &s1) == 2; }
        else if (k == "thickness" || k == "th") { thickness = atoi(v.c_str()); have[2] = true; }
        else if (k == "tiltfile" || k == "t") { tlt = v; have[3] = true; }
        else if (k == "output" || k == "o") { out = v; have[4] = true; }
        else if (k == "radius" || k == "r") { radius = atoi(v.c_str()); have[5] = true; }
        else if (k == "crossVfrc" || k == "cf") { cf = v; have_cf = true; }
        else if (k == "fullRecfrc" || k == "ff") { ff = v; have_ff = true; }
        else if (k == "zshift" || k == "z") zshift = atoi(v.c_str());
        else if (k == "gaussWidth" || k == "gw") gw = atoi(v.c_str());
        else if (k == "noMask" || k == "nm") nomask = atoi(v.c_str());
        i += 2;
    }
    if (!(have[0] && have[1] && have[2] && have[3] && have[4])) {
        printf("parameter error!\n'-inputPath' or '-slice' or '-thickness' or '-tiltfile' or '-output' are missed!\n"
               "Please use -help to see the manual\n");
        return -1;
    }
    if (nomask != 1 && !have[5] && !(have_cf && have_ff)) {
        printf("parameter error!\n'-radius' or ('-crossVfrc' & 'fullRecfrc') are missed!\nPlease use -help to see the manual\n");
        return -1;
    }
    std::vector<float> tilts;
    {
        FILE *f = fopen(tlt.c_str(), "r");
        if (!f) {
            printf("\nCannot open file %s strike any key exit!\n", tlt.c_str());
            return -1;
        }
        float v;
        while (fscanf(f, "%f", &v) == 1) tilts.push_back(v);
        fclose(f);
    }
    const int S = s1 - s0 + 1;
    std::string err;
    MrcHeader h0;
    if (S < 1 || !mrc_read_header(mid_name(in, s0), h0, err)) {
        printf("\nCan not open infile %s!\n", mid_name(in, s0).c_str());
        return 1;
    }
    const int n = h0.nx;
    if (h0.ny != n) {
        printf("the slices are %d x %d; the mask needs square slices (ICON-GPU without -thi)\n", h0.nx, h0.ny);
        return 1;
    }
    const int ystart = n / 2 - thickness / 2 + zshift;   // MK:1162
    if (thickness < 1 || ystart < 0 || ystart + thickness > n) {
        printf("zshift & thickness make the size of volume out of limitation!\n");
        return 1;
    }
    icon_mask *mask = nullptr;
    if (nomask != 1) {
        std::vector<float> cv, fr;
        if (!have[5]) {
            if (!read_frc(cf, cv)) {
                printf("\nCannot open file '%s' strike any key exit!", cf.c_str());
                return 1;
            }
            if (!read_frc(ff, fr)) {
                printf("\nCannot open file '%s' strike any key exit!", ff.c_str());
                return 1;
            }
        }
        float r05 = 0, r03 = 0;
        int expl = 0;
        if (icon_mask_radius(n, tilts.data(), (int)tilts.size(), have[5] ? radius : -1, cv.empty() ? nullptr : cv.data(),
                             fr.empty() ? nullptr : fr.data(), (int)std::min(cv.size(), fr.size()), &r05, &r03,
                             &expl) != ICON_OK ||
            icon_mask_create(n, tilts.data(), (int)tilts.size(), r05, r03, expl, gw, 16, &mask) != ICON_OK) {
            printf("running state: fail!\nError message: %s\n", icon_last_error());
            return 1;
        }
        printf("mask radius rate (frc 0.5) %f, (frc 0.3) %f\n", r05, r03);
    }
    std::vector<float> vol((size_t)S * thickness * n), slices((size_t)S * n * n), sl;
    for (int k = 0; k < S; ++k) {
        MrcHeader h;
        const std::string fn = mid_name(in, s0 + k);
        if (!mrc_read_header(fn, h, err) || !mrc_read_sections(fn, h, 0, 1, sl, err) || h.nx != n || h.ny != n) {
            printf("\nCan not open infile %s!\n", fn.c_str());
            return 1;
        }
        std::memcpy(&slices[(size_t)k * n * n], sl.data(), sizeof(float) * n * n);
    }
    if (mask) {
        if (icon_mask_apply_host(mask, slices.data(), S, ystart, thickness, vol.data()) != ICON_OK) {
            printf("running state: fail!\nError message: %s\n", icon_last_error());
            return 1;
        }
        icon_mask_destroy(mask);
    } else {   // MK:43-368: the rows alone
        for (int k = 0; k < S; ++k)
            std::memcpy(&vol[(size_t)k * thickness * n], &slices[((size_t)k * n + ystart) * n],
                        sizeof(float) * (size_t)thickness * n);
    }
    MrcHeader oh = h0;   // MK:1152-1157: the first slice's header, new sizes, float
    oh.nx = n;
    oh.ny = thickness;
    oh.nz = S;
    oh.mode = MRC_FLOAT;
    if (!mrc_write_float(out, oh, vol.data(), err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    printf("running state:\n   ICONMask finish!\n");
    return nomask == 1 ? 1 : 0;   // the reference returns 1 after the no-mask assembly (MK:777-782)
}
