// preprocess_cli.cpp -- icon-preprocess: drop-in for the reference's
// ICONPreProcess tool (sourceCode/ICONPreProcess/ICONPreProcess.c:89-300),
// same flags and output, with the work done on the GPU by icon_preprocess.
//
//   icon-preprocess -i stack.mrc -o out.mrc [-t angles.tlt -th thickness]
//
// Without both -t and -th only the mode is subtracted (as the reference
// prints, normalisation is then not executed).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "icon_tools.h"
#include "mrc_io.h"

namespace {

void help()
{
    printf("preProcess parameter\n######\n");
    printf("-input (-i) : the tilt series.\n######\n");
    printf("-tiltfile (-t) : the file containing aligned tilt angle of each projection image. If this option is not "
           "used, then only subtract the mode value of projection images.\n######\n");
    printf("-thickness (-th) : the thickness of specimen in pixel. If this option is not used, then only subtract the "
           "mode value of projection images\n######\n");
    printf("-output (-o) : preProcessed projection file.\n######\n");
    printf("-help (-h) : for help.\n");
}

}  // namespace

int main(int argc, char **argv)
{
    std::string in, tlt, out;
    int thickness = 0;
    bool have_in = false, have_t = false, have_th = false, have_out = false;
    for (int i = 1; i < argc;) {
        std::string a = argv[i];
        if (a.size() < 2 || a[0] != '-') {
            ++i;
            continue;
        }
        std::string k = a.substr(1);
        if (k == "help" || k == "h") {
            help();
            return 0;
        }
        if (i + 1 >= argc) break;
        std::string v = argv[i + 1];
        if (k == "input" || k == "i") { in = v; have_in = true; }
        else if (k == "tiltfile" || k == "t") { tlt = v; have_t = true; }
        else if (k == "thickness" || k == "th") { thickness = atoi(v.c_str()); have_th = true; }
        else if (k == "output" || k == "o") { out = v; have_out = true; }
        i += 2;
    }
    if (!have_in || !have_out) {
        printf("parameter error!\n'-input' or '-output' is missed!\nPlease use -help to see the manual\n");
        return -1;
    }
    if (!(have_t && have_th)) printf("tiltfile or thickness is not specified. Normalization will not be executed\n");
    printf("parameter:\ninput : %s\n", in.c_str());
    if (have_t) printf("tiltfile : %s\n", tlt.c_str());
    if (have_th) printf("thickness : %d\n", thickness);
    printf("output : %s\n", out.c_str());

    MrcHeader h;
    std::string err;
    if (!mrc_read_header(in, h, err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    std::vector<float> stack;
    if (!mrc_read_sections(in, h, 0, h.nz, stack, err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    std::vector<float> tilts;
    if (have_t && have_th) {
        FILE *f = fopen(tlt.c_str(), "r");
        if (!f) {
            printf("\nCannot open file '%s' strike any key exit!", tlt.c_str());
            return 1;
        }
        float v;
        while (fscanf(f, "%f", &v) == 1) tilts.push_back(v);
        fclose(f);
        if ((int)tilts.size() < h.nz) {
            printf("tilt file has %zu angles but the stack has %d sections\n", tilts.size(), h.nz);
            return 1;
        }
    }
    icon_status rc = icon_preprocess_host(stack.data(), stack.data(), h.nx, h.ny, h.nz,
                                          tilts.empty() ? nullptr : tilts.data(), tilts.empty() ? 0 : thickness);
    if (rc != ICON_OK) {
        printf("running state: fail!\nError message: %s\n", icon_last_error());
        return 1;
    }
    MrcHeader oh = h;   // header copied from the input, float mode, statistics recomputed
    oh.mode = MRC_FLOAT;
    if (!mrc_write_float(out, oh, stack.data(), err)) {
        printf("%s\n", err.c_str());
        return 1;
    }
    return 0;
}
