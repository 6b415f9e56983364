// dft.out: the reference's direct-DFT imager command line (src/dft/dft.cpp) on
// the B200 library.  Same flags: -theta -lambda -image -vis -blocks
// -threadblock -device -bl_min -bl_max -flat (-blocks/-threadblock are
// accepted and ignored: the launch shape is the library's).  Additional:
// -precision=fp32|reduced|fp64 (default reduced), -hermitian (factor 2, the
// gridder pipeline's image scale).  grid_size = floor(lambda*theta + 0.5)
// (src/dft/dft.cpp:171); writes the real image as float64 rows.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/radio_gridders.h"
#include "flags.h"

static int die(const char *what)
{
    std::fprintf(stderr, "%s: %s\n", what, rg_last_error());
    return 1;
}

int main(int argc, char **argv)
{
    using namespace cli;
    if (has(argc, argv, "help")) {
        std::printf("dft.out (B200): -theta -lambda -image -vis [-device -bl_min -bl_max -precision -hermitian]\n");
        return 0;
    }
    std::string visfile, image, prec;
    if (!value(argc, argv, "vis", &visfile)) {
        std::printf("No Visibility File Specified!! \n");
        return 0;
    }
    if (!has(argc, argv, "theta") || !has(argc, argv, "lambda")) {
        std::printf("No theta/lambda given!! \n");
        return 0;
    }
    const double theta = number(argc, argv, "theta", 0), lambda = number(argc, argv, "lambda", 0);
    const int N = (int)std::floor(lambda * theta + 0.5);
    const int device = (int)number(argc, argv, "device", 0);
    const double bl_min = number(argc, argv, "bl_min", 0), bl_max = number(argc, argv, "bl_max", DBL_MAX);
    int mode = RG_DFT_FP64_REDUCED;
    if (value(argc, argv, "precision", &prec)) mode = prec == "fp32" ? RG_DFT_FP32_NAIVE : (prec == "fp64" ? RG_DFT_FP64 : mode);
    const double factor = has(argc, argv, "hermitian") ? 2.0 : 1.0;
    value(argc, argv, "image", &image);
    rg_context *ctx;
    if (rg_context_create(device, &ctx) != RG_OK) return die("context");
    rg_vis_data vd;
    if (rg_read_vis_hdf5(visfile.c_str(), bl_min, bl_max, &vd) != RG_OK) return die("visibilities");
    rg_vis vis = {vd.u, vd.v, vd.w, vd.vis, vd.n};
    std::vector<double> img((size_t)N * N);
    if (rg_dft_image(ctx, img.data(), N, theta, &vis, mode, factor) != RG_OK) return die("dft");
    if (!image.empty()) {
        std::printf("Writing Image to File... \n");
        std::ofstream f(image, std::ios::binary);
        f.write((const char *)img.data(), (std::streamsize)(img.size() * sizeof(double)));
    }
    rg_free_vis_data(&vd);
    rg_context_destroy(ctx);
    return 0;
}
