// File-level entry points with the argument lists of the reference's host
// wrappers (src/grid/grid_common.cuh:49-62, src/dft/dft_common.cuh:16-18), so
// a caller written against those (grid.cpp, dft.cpp) changes only the function
// name: read the crocodile HDF5 files, grid (or transform), make the dirty
// image and leave it in the caller's complex N x N buffers (real part = image,
// imaginary part 0).  The image is the reference CPU pipeline's
// (src/reference/main.c:258-294: hermitian, shift, FFT, shift); the
// reference's GPU wrappers give half of it mirrored (no hermitian step, an
// inverse FFT).  Errors come back as rg_status, never exit().
#include <algorithm>
#include <vector>

#include "rg_internal.h"

using namespace rg;

namespace {

struct FileRun {
    rg_context *ctx = nullptr;
    rg_vis_data vd{};
    bool have_vis = false;
    ~FileRun()
    {
        if (have_vis) rg_free_vis_data(&vd);
        if (ctx) rg_context_destroy(ctx);
    }
};

rg_status open_run(FileRun &run, const char *visfile, double bl_min, double bl_max)
{
    if (!visfile) return fail(RG_ERR_INVALID_ARGUMENT, "visfile is NULL");
    int device = 0;
    RG_CUDA(cudaGetDevice(&device));
    RG_CHECK(rg_context_create(device, &run.ctx));
    RG_CHECK(rg_read_vis_hdf5(visfile, bl_min, bl_max, &run.vd));
    run.have_vis = true;
    return RG_OK;
}

// image (N*N float64, host) -> complex (re = image, im = 0) into the device
// buffer and, when given, the host buffer
rg_status deliver(const std::vector<double> &img, double *dev, double *host, int N)
{
    std::vector<double> z((size_t)2 * N * N, 0.0);
    for (size_t i = 0; i < img.size(); i++) z[2 * i] = img[i];
    if (dev) RG_CUDA(cudaMemcpy(dev, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice));
    if (host) std::copy(z.begin(), z.end(), host);
    return RG_OK;
}

rg_status grid_files(const char *visfile, const char *wkernfile, double *grid, double *gridh, int N,
                     double theta, double bl_min, double bl_max, bool towers, int S, int M, double winc)
{
    if (!wkernfile || !grid) return fail(RG_ERR_INVALID_ARGUMENT, "wkernfile and grid must be non-NULL");
    if (N < 2) return fail(RG_ERR_INVALID_ARGUMENT, "grid_size must be >= 2");
    FileRun run;
    RG_CHECK(open_run(run, visfile, bl_min, bl_max));
    rg_wkern_data wd;
    RG_CHECK(rg_read_wkern_hdf5(wkernfile, theta, &wd));
    rg_wkern wk = {wd.data, wd.plane_count, wd.size, wd.oversampling, wd.w_min, wd.w_step};
    rg_vis vis = {run.vd.u, run.vd.v, run.vd.w, run.vd.vis, run.vd.n};
    // the caller's N x N complex device buffer holds the uv grid, then the image
    rg_status st = towers ? rg_grid_wtowers(run.ctx, grid, N, theta, &vis, &wk, S, M, winc, RG_GRID_OVERWRITE)
                          : rg_grid_wprojection(run.ctx, grid, N, theta, &vis, &wk, RG_GRID_OVERWRITE);
    rg_free_wkern_data(&wd);
    if (st != RG_OK) return st;
    std::vector<double> img((size_t)N * N);
    RG_CHECK(rg_image_from_grid(run.ctx, grid, N, img.data(), nullptr));
    return deliver(img, grid, gridh, N);
}

}  // namespace

extern "C" {

rg_status rg_wtowers_cuda_flat(const char *visfile, const char *wkernfile, double *grid, double *gridh,
                               int grid_size, double theta, double lambda, double bl_min, double bl_max,
                               int subgrid_size, int subgrid_margin, double winc)
{
    (void)lambda;  // the caller derives grid_size from it (grid.cpp:195)
    return grid_files(visfile, wkernfile, grid, gridh, grid_size, theta, bl_min, bl_max, true, subgrid_size,
                      subgrid_margin, winc);
}

rg_status rg_wproj_cuda_flat(const char *visfile, const char *wkernfile, double *grid, double *gridh,
                             int grid_size, double theta, double lambda, double bl_min, double bl_max,
                             int threads_per_block)
{
    (void)lambda;
    (void)threads_per_block;  // launch shapes are the library's own
    return grid_files(visfile, wkernfile, grid, gridh, grid_size, theta, bl_min, bl_max, false, 0, 0, 0.0);
}

rg_status rg_image_dft_host_flat(const char *visfile, double *grid_host, double *grid_dev, int grid_size,
                                 double theta, double lambda, double bl_min, double bl_max, int blocks,
                                 int threads_block)
{
    (void)lambda;
    (void)blocks;
    (void)threads_block;
    if (!grid_host && !grid_dev) return fail(RG_ERR_INVALID_ARGUMENT, "no output buffer");
    if (grid_size < 2) return fail(RG_ERR_INVALID_ARGUMENT, "grid_size must be >= 2");
    FileRun run;
    RG_CHECK(open_run(run, visfile, bl_min, bl_max));
    rg_vis vis = {run.vd.u, run.vd.v, run.vd.w, run.vd.vis, run.vd.n};
    std::vector<double> img((size_t)grid_size * grid_size);
    RG_CHECK(rg_dft_image(run.ctx, img.data(), grid_size, theta, &vis, RG_DFT_FP64_REDUCED, 1.0));
    return deliver(img, grid_dev, grid_host, grid_size);
}

}  // extern "C"
