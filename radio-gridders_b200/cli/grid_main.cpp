// grid.out: the reference's GPU imager command line (src/grid/grid.cpp) on the
// B200 library.  Same flags: -theta -lambda -image -wkernel -vis -subgrid
// -margin -winc -bl_min -bl_max -wproj -flat -device (-flat is accepted; the
// flat layout is always used).  Additional: -grid=FILE writes the hermitian uv
// grid (complex128 rows, as src/reference/main.c:261-268), -weight applies
// uniform weighting first (src/reference/main.c:153), -learned=FILE grids
// W-projection with a learned w-kernel network (float32 parameter file in
// rg_mlp_get_params order; -learned_ksize/-learned_wmax/-learned_scale give
// the rg_mlp_create arguments it was trained with).
// The image is the reference CPU pipeline's dirty image (hermitian, shift,
// FFT sign -1, shift; real part as float64 rows, src/reference/main.c:269-294).
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/radio_gridders.h"
#include "flags.h"

static void help()
{
    std::printf(
        "\ngrid.out (B200)\n\n"
        "\t-theta               Field of View (Radians)\n"
        "\t-lambda              Number of Wavelengths\n"
        "\t-image               Image File\n"
        "\t-wkernel             Input W-Kernels\n"
        "\t-vis                 Input Visibilities\n"
        "\t-subgrid             W-Towers Subgrid Size\n"
        "\t-margin              W-Towers Margin Size\n"
        "\t-winc                W-Plane Increment Size\n"
        "\t-bl_min              Minimum Baseline Length (metres, first uvw sample)\n"
        "\t-bl_max              Maximum Baseline Length (metres, first uvw sample)\n"
        "\t-wproj               W-Projection Mode\n"
        "\t-device              GPU Device to use (Default: 0)\n"
        "\t-grid                uv grid output file (complex128, after make_hermitian)\n"
        "\t-weight              uniform weighting before gridding\n"
        "\t-akern               A-kernel file: AW-projection with -wkernel (src/reference/main.c:32)\n"
        "\t-simple              nearest-cell gridding, no w-kernel (grid_CPU.out without --wkern)\n"
        "\t-learned             learned w-kernel parameter file (float32, W-projection)\n"
        "\t-learned_ksize       learned kernel support (Default: 16)\n"
        "\t-learned_wmax        learned kernel w range it was trained on (Default: 2000)\n"
        "\t-learned_scale       learned kernel output scale (Default: 0.05)\n\n");
}

static int die(const char *what)
{
    std::fprintf(stderr, "%s: %s\n", what, rg_last_error());
    return 1;
}

// Timing line, then the hermitian uv grid (-grid) and the dirty image (-image)
// as raw float64 (src/reference/main.c:258-294).
static int write_outputs(rg_context *ctx, std::vector<double> &grid, int N, const std::string &gridfile,
                         const std::string &image)
{
    const char *names[64];
    float ms[64];
    const int nt = rg_last_timings(ctx, names, ms, 64);
    float total = 0;
    for (int i = 0; i < nt; i++) total += ms[i];
    std::printf("Gridder Elapsed Time: %.6f seconds\n", total / 1000.0);
    if (!gridfile.empty()) {
        std::vector<double> h = grid;
        if (rg_make_hermitian(ctx, h.data(), N) != RG_OK) return die("make_hermitian");
        std::ofstream f(gridfile, std::ios::binary);
        f.write((const char *)h.data(), (std::streamsize)(h.size() * sizeof(double)));
    }
    if (!image.empty()) {
        std::vector<double> img((size_t)N * N);
        if (rg_image_from_grid(ctx, grid.data(), N, img.data(), nullptr) != RG_OK) return die("image");
        std::printf("Writing Image to File... \n");
        std::ofstream f(image, std::ios::binary);
        f.write((const char *)img.data(), (std::streamsize)(img.size() * sizeof(double)));
    }
    return 0;
}

int main(int argc, char **argv)
{
    using namespace cli;
    if (has(argc, argv, "help")) {
        help();
        return 0;
    }
    std::string visfile, wkfile, image, gridfile, learned;
    if (!value(argc, argv, "vis", &visfile)) {
        std::printf("No Visibility File Specified!! \n");
        help();
        return 0;
    }
    const bool wproj = has(argc, argv, "wproj");
    value(argc, argv, "learned", &learned);
    const bool simple = has(argc, argv, "simple");
    if (!value(argc, argv, "wkernel", &wkfile) && learned.empty() && !simple) {
        std::printf("No W-Kernel File Specified!! \n");
        help();
        return 0;
    }
    if (!has(argc, argv, "theta")) {
        std::printf("No theta given!! \n");
        help();
        return 0;
    }
    if (!has(argc, argv, "lambda")) {
        std::printf("No lambda given!! \n");
        help();
        return 0;
    }
    const double theta = number(argc, argv, "theta", 0), lambda = number(argc, argv, "lambda", 0);
    const int device = (int)number(argc, argv, "device", 0);
    const double bl_min = number(argc, argv, "bl_min", 0), bl_max = number(argc, argv, "bl_max", DBL_MAX);
    const bool awproj = has(argc, argv, "akern");
    if (!wproj && !awproj && !simple &&
        (!has(argc, argv, "subgrid") || !has(argc, argv, "margin") || !has(argc, argv, "winc"))) {
        std::printf("Missing W-Towers Parameters. Check subgrid/margin/winc\n");
        help();
        return 0;
    }
    const int subgrid = (int)number(argc, argv, "subgrid", 0), margin = (int)number(argc, argv, "margin", 0);
    const double winc = number(argc, argv, "winc", 0);
    value(argc, argv, "image", &image);
    value(argc, argv, "grid", &gridfile);
    const int N = (int)std::floor(lambda * theta);  // src/grid/grid.cpp:195
    if (N <= 0) {
        std::fprintf(stderr, "Invalid grid configuration!\n");
        return 1;
    }

    rg_context *ctx;
    if (rg_context_create(device, &ctx) != RG_OK) return die("context");
    std::string akfile;
    if (value(argc, argv, "akern", &akfile) && !wkfile.empty()) {
        // AW-projection (src/reference/main.c:207-233): hierarchical
        // visibilities, A-kernel channel frequencies pick the w-planes
        rg_vis_bl_data hd;
        if (rg_read_vis_bl_hdf5(visfile.c_str(), bl_min, bl_max, &hd) != RG_OK) return die("visibilities");
        std::printf("Have %d baselines and %lld visibilities\n", hd.bl_count,
                    (long long)hd.bl_count * hd.time_count * hd.freq_count);
        rg_wkern_data wd;
        if (rg_read_wkern_hdf5(wkfile.c_str(), theta, &wd) != RG_OK) return die("w-kernels");
        rg_akern_data ad;
        if (rg_read_akern_hdf5(akfile.c_str(), theta, &ad) != RG_OK) return die("A-kernels");
        const int64_t nv = (int64_t)hd.bl_count * hd.time_count * hd.freq_count;
        if (has(argc, argv, "weight") && nv > 0) {  // main.c:153, on the same visibility order
            std::vector<double> u(nv), v(nv), w(nv);
            int64_t k = 0;
            for (int b = 0; b < hd.bl_count; b++)
                for (int t = 0; t < hd.time_count; t++)
                    for (int f = 0; f < hd.freq_count; f++, k++) {
                        const double *uvw = hd.uvw + ((size_t)b * hd.time_count + t) * 3;
                        const double fr = hd.freq[(size_t)b * hd.freq_count + f];
                        u[k] = uvw[0] * fr / 299792458.0;
                        v[k] = uvw[1] * fr / 299792458.0;
                        w[k] = uvw[2] * fr / 299792458.0;
                    }
            rg_vis fv = {u.data(), v.data(), w.data(), hd.vis, nv};
            if (rg_weight(ctx, N, theta, &fv, hd.vis) != RG_OK) return die("weighting");
        }
        rg_wkern wk = {wd.data, wd.plane_count, wd.size, wd.oversampling, wd.w_min, wd.w_step};
        rg_akern ak = {ad.antenna_count, ad.time_count, ad.freq_count, ad.size_x, ad.size_y, ad.t_min, ad.t_step,
                       ad.f_min, ad.f_step, ad.freq, ad.time, ad.data};
        rg_vis_bl vb = {hd.bl_count, hd.time_count, hd.freq_count, hd.antenna1, hd.antenna2,
                        hd.time, hd.freq, hd.uvw, hd.vis};
        std::vector<double> grid((size_t)N * N * 2, 0.0);
        std::printf("Gridder: AW-projection (ignoring convolution)\n");
        rg_context_set_profiling(ctx, 1);
        if (rg_grid_awprojection(ctx, grid.data(), N, theta, &vb, &wk, &ak, 0, hd.bl_count, RG_GRID_OVERWRITE) !=
            RG_OK)
            return die("gridding");
        const int rc = write_outputs(ctx, grid, N, gridfile, image);
        rg_free_akern_data(&ad);
        rg_free_wkern_data(&wd);
        rg_free_vis_bl_data(&hd);
        rg_context_destroy(ctx);
        return rc;
    }
    rg_vis_data vd;
    if (rg_read_vis_hdf5(visfile.c_str(), bl_min, bl_max, &vd) != RG_OK) return die("visibilities");
    std::printf("Have %lld baselines and %lld visibilities\n", (long long)vd.bl_count, (long long)vd.n);
    if (has(argc, argv, "weight") && vd.n > 0) {
        rg_vis v = {vd.u, vd.v, vd.w, vd.vis, vd.n};
        if (rg_weight(ctx, N, theta, &v, vd.vis) != RG_OK) return die("weighting");
    }
    rg_vis vis = {vd.u, vd.v, vd.w, vd.vis, vd.n};
    std::vector<double> grid((size_t)N * N * 2, 0.0);
    rg_context_set_profiling(ctx, 1);
    if (simple) {  // grid_CPU.out without a w-kernel file (src/reference/main.c:200-206)
        std::printf("Gridder: Simple imaging\n");
        if (rg_grid_simple(ctx, grid.data(), N, theta, &vis, RG_GRID_OVERWRITE) != RG_OK) return die("gridding");
    } else if (!learned.empty()) {
        rg_mlp *mlp;
        const int lk = (int)number(argc, argv, "learned_ksize", 16);
        const double lw = number(argc, argv, "learned_wmax", 2000.0);
        const double ls = number(argc, argv, "learned_scale", 0.05);
        if (rg_mlp_create(ctx, lk, lw, ls, 0, &mlp) != RG_OK) return die("learned kernel");
        std::vector<float> p(rg_mlp_param_count());
        std::ifstream f(learned, std::ios::binary);
        if (!f.read((char *)p.data(), (std::streamsize)(p.size() * sizeof(float)))) {
            std::fprintf(stderr, "cannot read %s\n", learned.c_str());
            return 1;
        }
        if (rg_mlp_set_params(ctx, mlp, p.data()) != RG_OK) return die("learned kernel");
        std::printf("W-Projection Gridder (learned kernel)...\n");
        if (rg_grid_wprojection_learned(ctx, mlp, grid.data(), N, theta, &vis, RG_GRID_OVERWRITE) != RG_OK)
            return die("gridding");
        rg_mlp_destroy(mlp);
    } else {
        rg_wkern_data wd;
        if (rg_read_wkern_hdf5(wkfile.c_str(), theta, &wd) != RG_OK) return die("w-kernels");
        rg_wkern wk = {wd.data, wd.plane_count, wd.size, wd.oversampling, wd.w_min, wd.w_step};
        std::printf("w kernels:   %.2f - %.2f lambda (step %.2f lambda)\n", wd.w_min,
                    wd.w_min + (wd.plane_count - 1) * wd.w_step, wd.w_step);
        rg_status st;
        if (wproj) {
            std::printf("W-Projection Gridder...\n");
            st = rg_grid_wprojection(ctx, grid.data(), N, theta, &vis, &wk, RG_GRID_OVERWRITE);
        } else {
            std::printf("W-Towers Gridder...\n");
            st = rg_grid_wtowers(ctx, grid.data(), N, theta, &vis, &wk, subgrid, margin, winc, RG_GRID_OVERWRITE);
        }
        if (st != RG_OK) return die("gridding");
        rg_free_wkern_data(&wd);
    }
    const int rc = write_outputs(ctx, grid, N, gridfile, image);
    rg_free_vis_data(&vd);
    rg_context_destroy(ctx);
    return rc;
}
