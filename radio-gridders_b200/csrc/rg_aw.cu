// AW-projection and the hierarchical visibility and A-kernel files it needs.
//
// The reference's grid_awprojection (src/reference/grid.c:595-637) grids each
// visibility with the kernel convolve_aw_kernels (:557-593) prepared for its
// baseline, time and nearest A-kernel frequency channel: the w-kernel plane
// nearest to w = uvw_w * f_A / c, f_A being the frequency of antenna 1's
// A-kernel for that time slot and channel (load_akern's kern_by_atf,
// src/common/hdf5.c:652-820).  The A x W convolution itself is a placeholder
// in the reference ("it doesn't matter for this test, so we just copy the
// w-kernel", grid.c:583-590), so the grid is a W-projection grid whose plane
// choice follows the A-kernel channels; that is what is computed here: the
// per-visibility plane w is formed on the host in the reference's arithmetic,
// then the visibilities go through the device W-projection path
// (prepare_wproj_kernel + romein_kernel, FP32 sub-cell taps, FP64 grid).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "hdf5_lite.h"
#include "rg_internal.h"

using namespace rg;

namespace {

constexpr double kC = 299792458.0;  // src/reference/grid.c:19

double *dup_doubles(const std::vector<double> &v)
{
    double *p = (double *)std::malloc(sizeof(double) * (v.size() ? v.size() : 1));
    if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(double) * v.size());
    return p;
}

std::string fmt_g(double x)
{
    char b[64];
    std::snprintf(b, sizeof(b), "%g", x);
    return b;
}

// index of the nearest sample of an evenly spaced axis (count 1: always 0)
int nearest_index(double x, double x0, double step, int count)
{
    if (count == 1) return 0;
    return (int)std::floor((x - x0) / step + .5);
}

}  // namespace

extern "C" {

rg_status rg_read_vis_bl_hdf5(const char *path, double bl_min, double bl_max, rg_vis_bl_data *out)
{
    if (!path || !out) return fail(RG_ERR_INVALID_ARGUMENT, "path and out must be non-NULL");
    std::memset(out, 0, sizeof(*out));
    std::vector<int32_t> a1, a2;
    std::vector<double> time, freq, uvw, vis;
    int nt = -1, nf = -1;
    bool uniform = true;
    RG_CHECK(visit_vis_hdf5(path, bl_min, bl_max, [&](const BaselineRecord &r) {
        if (nt < 0) {
            nt = (int)r.time.size();
            nf = (int)r.freq.size();
        }
        if ((int)r.time.size() != nt || (int)r.freq.size() != nf) {
            uniform = false;
            return;
        }
        a1.push_back(r.a1);
        a2.push_back(r.a2);
        time.insert(time.end(), r.time.begin(), r.time.end());
        freq.insert(freq.end(), r.freq.begin(), r.freq.end());
        uvw.insert(uvw.end(), r.uvw.begin(), r.uvw.end());
        vis.insert(vis.end(), r.vis.begin(), r.vis.end());
    }));
    if (!uniform) return fail(RG_ERR_UNSUPPORTED, "baselines with different time or frequency counts");
    out->bl_count = (int)a1.size();
    out->time_count = nt < 0 ? 0 : nt;
    out->freq_count = nf < 0 ? 0 : nf;
    out->antenna1 = (int32_t *)std::malloc(sizeof(int32_t) * (a1.size() + 1));
    out->antenna2 = (int32_t *)std::malloc(sizeof(int32_t) * (a2.size() + 1));
    out->time = dup_doubles(time);
    out->freq = dup_doubles(freq);
    out->uvw = dup_doubles(uvw);
    out->vis = dup_doubles(vis);
    if (!out->antenna1 || !out->antenna2 || !out->time || !out->freq || !out->uvw || !out->vis) {
        rg_free_vis_bl_data(out);
        return fail(RG_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    if (!a1.empty()) {
        std::memcpy(out->antenna1, a1.data(), sizeof(int32_t) * a1.size());
        std::memcpy(out->antenna2, a2.data(), sizeof(int32_t) * a2.size());
    }
    return RG_OK;
}

void rg_free_vis_bl_data(rg_vis_bl_data *d)
{
    if (!d) return;
    std::free(d->antenna1);
    std::free(d->antenna2);
    std::free(d->time);
    std::free(d->freq);
    std::free(d->uvw);
    std::free(d->vis);
    std::memset(d, 0, sizeof(*d));
}

rg_status rg_read_akern_hdf5(const char *path, double theta, rg_akern_data *out)
{
    if (!path || !out) return fail(RG_ERR_INVALID_ARGUMENT, "path and out must be non-NULL");
    std::memset(out, 0, sizeof(*out));
    h5::File f;
    std::string err;
    if (!f.open(path, &err)) return fail(RG_ERR_IO, err);
    const std::string gname = "akern/" + fmt_g(theta);  // src/common/hdf5.c:667-668
    h5::Object g;
    if (!f.find(gname, &g, &err) || !g.is_group) return fail(RG_ERR_IO, "could not open '" + gname + "' in " + path);
    struct Kern {
        double t, fr;
        std::vector<double> data;
    };
    std::map<int, std::vector<Kern>> by_ant;
    std::vector<std::pair<std::string, uint64_t>> ants;
    if (!f.entries(g, &ants, &err)) return fail(RG_ERR_IO, err);
    int tcount = -1, fcount = -1, sx = 0, sy = 0;
    double tmin = 1e300, tmax = -1e300, fmin = 1e300, fmax = -1e300;
    for (auto &a : ants) {
        h5::Object ag;
        std::vector<std::pair<std::string, uint64_t>> times;
        if (!f.object_at(a.second, &ag, &err) || !f.entries(ag, &times, &err)) return fail(RG_ERR_IO, err);
        if (tcount < 0) tcount = (int)times.size();
        if ((int)times.size() != tcount) continue;  // inconsistent time slots are ignored (hdf5.c:711-714)
        const int ant = std::atoi(a.first.c_str());
        for (auto &t : times) {
            h5::Object tg;
            std::vector<std::pair<std::string, uint64_t>> freqs;
            if (!f.object_at(t.second, &tg, &err) || !f.entries(tg, &freqs, &err)) return fail(RG_ERR_IO, err);
            if (fcount < 0) fcount = (int)freqs.size();
            if ((int)freqs.size() != fcount) continue;
            const double tv = std::atof(t.first.c_str());
            tmin = std::min(tmin, tv);
            tmax = std::max(tmax, tv);
            for (auto &fq : freqs) {
                h5::Object fg, kd;
                std::vector<std::pair<std::string, uint64_t>> fe;
                if (!f.object_at(fq.second, &fg, &err) || !f.entries(fg, &fe, &err)) return fail(RG_ERR_IO, err);
                const double fv = std::atof(fq.first.c_str());
                fmin = std::min(fmin, fv);
                fmax = std::max(fmax, fv);
                uint64_t ka = 0;
                for (auto &q : fe)
                    if (q.first == "kern") ka = q.second;
                if (!ka || !f.object_at(ka, &kd, &err) || kd.ds.dims.size() != 2) continue;
                const int d0 = (int)kd.ds.dims[0], d1 = (int)kd.ds.dims[1];
                if (sx == 0) {
                    sy = d0;
                    sx = d1;
                }
                if (d0 != sy || d1 != sx) continue;  // inconsistent dimensions are ignored
                Kern k;
                k.t = tv;
                k.fr = fv;
                if (!f.read_doubles(kd.ds, &k.data, &err)) return fail(RG_ERR_IO, err);
                by_ant[ant].push_back(std::move(k));
            }
        }
    }
    const int nant = (int)ants.size();
    if (nant == 0 || tcount <= 0 || fcount <= 0 || sx == 0)
        return fail(RG_ERR_IO, std::string("no A-kernels in ") + path);
    // evenly spaced axes from the extremes (hdf5.c:772-773), then each
    // (antenna, time, frequency) slot takes the antenna's nearest kernel in
    // |dt| + |df| (hdf5.c:782-810)
    const double tstep = tcount > 1 ? (tmax - tmin) / (tcount - 1) : 1.0;
    const double fstep = fcount > 1 ? (fmax - fmin) / (fcount - 1) : 1.0;
    const size_t per = (size_t)sx * sy * 2, slots = (size_t)nant * tcount * fcount;
    out->data = (double *)std::calloc(per * slots, sizeof(double));
    out->freq = (double *)std::calloc(slots, sizeof(double));
    out->time = (double *)std::calloc(slots, sizeof(double));
    if (!out->data || !out->freq || !out->time) {
        rg_free_akern_data(out);
        return fail(RG_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    for (int ant = 0; ant < nant; ant++) {
        auto it = by_ant.find(ant);
        if (it == by_ant.end() || it->second.empty()) {
            rg_free_akern_data(out);
            return fail(RG_ERR_IO, "A-kernel antennas must be numbered 0.." + std::to_string(nant - 1));
        }
        const std::vector<Kern> &ks = it->second;
        for (int t = 0; t < tcount; t++)
            for (int fi = 0; fi < fcount; fi++) {
                const double tw = tmin + t * tstep, fw = fmin + fi * fstep;
                size_t best = 0;
                for (size_t j = 1; j < ks.size(); j++)
                    if (std::fabs(ks[j].t - tw) + std::fabs(ks[j].fr - fw) <
                        std::fabs(ks[best].t - tw) + std::fabs(ks[best].fr - fw))
                        best = j;
                const size_t slot = ((size_t)ant * tcount + t) * fcount + fi;
                out->time[slot] = ks[best].t;
                out->freq[slot] = ks[best].fr;
                std::memcpy(out->data + per * slot, ks[best].data.data(), sizeof(double) * per);
            }
    }
    out->antenna_count = nant;
    out->time_count = tcount;
    out->freq_count = fcount;
    out->size_x = sx;
    out->size_y = sy;
    out->t_min = tmin;
    out->t_step = tstep;
    out->f_min = fmin;
    out->f_step = fstep;
    return RG_OK;
}

void rg_free_akern_data(rg_akern_data *d)
{
    if (!d) return;
    std::free(d->data);
    std::free(d->freq);
    std::free(d->time);
    std::memset(d, 0, sizeof(*d));
}

rg_status rg_write_akern_hdf5(const char *path, double theta, const rg_akern *ak)
{
    if (!path || !ak || !ak->freq || !ak->time || !ak->data || ak->antenna_count < 1 || ak->time_count < 1 ||
        ak->freq_count < 1 || ak->size_x < 1 || ak->size_y < 1)
        return fail(RG_ERR_INVALID_ARGUMENT, "bad A-kernel table");
    h5::Writer wr;
    const int g0 = wr.add_group(0, "akern");
    const int g1 = wr.add_group(g0, fmt_g(theta));
    const size_t per = (size_t)ak->size_x * ak->size_y * 2;
    for (int a = 0; a < ak->antenna_count; a++) {
        const int ga = wr.add_group(g1, std::to_string(a));
        for (int t = 0; t < ak->time_count; t++) {
            const size_t s0 = ((size_t)a * ak->time_count + t) * ak->freq_count;
            char name[64];
            std::snprintf(name, sizeof(name), "%.17g", ak->time[s0]);
            const int gt = wr.add_group(ga, name);
            for (int fi = 0; fi < ak->freq_count; fi++) {
                std::snprintf(name, sizeof(name), "%.17g", ak->freq[s0 + fi]);
                const int gf = wr.add_group(gt, name);
                wr.add_dataset_c128(gf, "kern", {(uint64_t)ak->size_y, (uint64_t)ak->size_x},
                                    ak->data + per * (s0 + fi));
            }
        }
    }
    std::string err;
    if (!wr.write(path, &err)) return fail(RG_ERR_IO, err);
    return RG_OK;
}

rg_status rg_grid_awprojection(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis_bl *vis,
                               const rg_wkern *wkern, const rg_akern *akern, int bl_min, int bl_max, int flags)
{
    if (!ctx || !uvgrid || !vis || !wkern || !akern || !akern->freq)
        return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    RG_CHECK(check_wkern(wkern));
    // src/reference/grid.c:562-563
    if (akern->size_x != wkern->size || akern->size_y != wkern->size)
        return fail(RG_ERR_INVALID_ARGUMENT, "A-kernel and w-kernel sizes differ");
    if (akern->antenna_count < 1 || akern->time_count < 1 || akern->freq_count < 1)
        return fail(RG_ERR_INVALID_ARGUMENT, "empty A-kernel table");
    if (vis->bl_count < 0 || vis->time_count < 0 || vis->freq_count < 0)
        return fail(RG_ERR_INVALID_ARGUMENT, "negative counts");
    if (bl_min < 0 || bl_max > vis->bl_count || bl_min > bl_max)
        return fail(RG_ERR_INVALID_ARGUMENT, "baseline range outside [0, bl_count]");
    const int nt = vis->time_count, nf = vis->freq_count, FA = akern->freq_count, TA = akern->time_count;
    const int64_t n = (int64_t)(bl_max - bl_min) * nt * nf;
    if (n > 0 && (!vis->antenna1 || !vis->time || !vis->freq || !vis->uvw || !vis->vis))
        return fail(RG_ERR_INVALID_ARGUMENT, "visibility arrays must be non-NULL");
    // per visibility: u, v at its own frequency (uvw_lambda, grid.c:21-24) and
    // the w that picks its plane (convolve_aw_kernels, grid.c:571-582)
    std::vector<double> u((size_t)n), v((size_t)n), w((size_t)n), wa((size_t)nt * FA);
    size_t k = 0;
    for (int bl = bl_min; bl < bl_max; bl++) {
        const double *bt = vis->time + (size_t)bl * nt, *bf = vis->freq + (size_t)bl * nf;
        const double *bu = vis->uvw + (size_t)bl * nt * 3;
        const int a1 = vis->antenna1[bl];
        if (a1 < 0 || a1 >= akern->antenna_count) return fail(RG_ERR_INVALID_ARGUMENT, "antenna without A-kernels");
        for (int t = 0; t < nt; t++) {
            const int atime = nearest_index(bt[t], akern->t_min, akern->t_step, TA);
            if (atime < 0 || atime >= TA) return fail(RG_ERR_INVALID_ARGUMENT, "time outside the A-kernel table");
            for (int af = 0; af < FA; af++)
                wa[(size_t)t * FA + af] = bu[t * 3 + 2] * akern->freq[((size_t)a1 * TA + atime) * FA + af] / kC;
        }
        for (int t = 0; t < nt; t++)
            for (int fi = 0; fi < nf; fi++, k++) {
                const int afreq = nearest_index(bf[fi], akern->f_min, akern->f_step, FA);
                if (afreq < 0 || afreq >= FA)
                    return fail(RG_ERR_INVALID_ARGUMENT, "frequency outside the A-kernel table");
                u[k] = bu[t * 3 + 0] * bf[fi] / kC;
                v[k] = bu[t * 3 + 1] * bf[fi] / kC;
                w[k] = wa[(size_t)t * FA + afreq];
            }
    }
    rg_vis flat;
    flat.u = u.data();
    flat.v = v.data();
    flat.w = w.data();
    flat.vis = vis->vis + (size_t)bl_min * nt * nf * 2;
    flat.n = n;
    return rg_grid_wprojection(ctx, uvgrid, grid_size, theta, &flat, wkern, flags);
}

}  // extern "C"
