// Crocodile HDF5 visibility and w-kernel files through the C ABI.  Layouts
// (the reference's loaders, src/reference/hdf5.c and src/common/hdf5.c):
//   visibilities: /vis/<a1>/<a2>/{frequency[nf], time[nt], uvw[nt][3] (metres),
//                 vis[nt][nf][1] {r, i}}  (hierarchical), or the legacy flat
//                 /vis/{uvw, time, frequency, vis, antenna1, antenna2} where every
//                 row is one baseline-time;
//   w-kernels:    /wkern/<theta as %g>/<w>/kern[ov][ov][S][S] {r, i}.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "hdf5_lite.h"
#include "rg_internal.h"

using namespace rg;

namespace {

constexpr double kC = 299792458.0;  // src/reference/hdf5.c:12

// One baseline group (src/reference/hdf5.c:64-96, :305-349): its time, frequency,
// uvw (metres) and visibility arrays, if the first uvw sample's (u, v) length
// lies in [bl_min, bl_max) (src/reference/hdf5.c:104-106).
bool read_baseline(h5::File &f, const h5::Object &g, double bl_min, double bl_max, BaselineRecord *rec, bool *kept,
                   std::string *err)
{
    std::vector<std::pair<std::string, uint64_t>> ent;
    if (!f.entries(g, &ent, err)) return false;
    std::map<std::string, uint64_t> by;
    for (auto &e : ent) by[e.first] = e.second;
    const char *need[4] = {"frequency", "time", "uvw", "vis"};
    h5::Object o[4];
    for (int i = 0; i < 4; i++) {
        auto it = by.find(need[i]);
        if (it == by.end() || !f.object_at(it->second, &o[i], err)) {
            *err = std::string("baseline group lacks '") + need[i] + "'";
            return false;
        }
    }
    if (!f.read_doubles(o[0].ds, &rec->freq, err) || !f.read_doubles(o[1].ds, &rec->time, err) ||
        !f.read_doubles(o[2].ds, &rec->uvw, err) || !f.read_doubles(o[3].ds, &rec->vis, err))
        return false;
    const size_t nt = rec->time.size(), nf = rec->freq.size();
    if (rec->uvw.size() != nt * 3 || rec->vis.size() != nt * nf * 2) {
        *err = "inconsistent baseline dataset shapes";
        return false;
    }
    *kept = false;
    if (nt == 0) return true;
    const double len = std::sqrt(rec->uvw[0] * rec->uvw[0] + rec->uvw[1] * rec->uvw[1]);
    *kept = !(len < bl_min || len >= bl_max);
    return true;
}

double *copy_out(const std::vector<double> &v)
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

}  // namespace

namespace rg {

rg_status visit_vis_hdf5(const char *path, double bl_min, double bl_max,
                         const std::function<void(const BaselineRecord &)> &fn)
{
    h5::File f;
    std::string err;
    if (!f.open(path, &err)) return fail(RG_ERR_IO, err);
    h5::Object vg;
    if (!f.find("vis", &vg, &err) || !vg.is_group)
        return fail(RG_ERR_IO, std::string("no 'vis' group in ") + path + (err.empty() ? "" : ": " + err));
    std::vector<std::pair<std::string, uint64_t>> ent;
    if (!f.entries(vg, &ent, &err)) return fail(RG_ERR_IO, err);
    bool legacy = false;
    for (auto &e : ent) legacy |= e.first == "uvw";
    if (legacy) {  // src/reference/hdf5.c:173-247: one baseline per row
        std::map<std::string, uint64_t> by;
        for (auto &e : ent) by[e.first] = e.second;
        h5::Object ou, of, ov, ot, oa1, oa2;
        if (!by.count("frequency") || !by.count("vis") || !f.object_at(by["uvw"], &ou, &err) ||
            !f.object_at(by["frequency"], &of, &err) || !f.object_at(by["vis"], &ov, &err))
            return fail(RG_ERR_IO, "incomplete flat 'vis' group");
        std::vector<double> uvw, freq, vis, time;
        std::vector<int64_t> a1, a2;
        if (!f.read_doubles(ou.ds, &uvw, &err) || !f.read_doubles(of.ds, &freq, &err) ||
            !f.read_doubles(ov.ds, &vis, &err))
            return fail(RG_ERR_IO, err);
        const size_t nt = uvw.size() / 3, nf = freq.size();
        if (vis.size() != nt * nf * 2) return fail(RG_ERR_IO, "inconsistent flat visibility shapes");
        // antenna and time columns, when present (AW-projection needs them)
        if (by.count("time") && f.object_at(by["time"], &ot, &err)) f.read_doubles(ot.ds, &time, &err);
        if (by.count("antenna1") && f.object_at(by["antenna1"], &oa1, &err)) f.read_int64(oa1.ds, &a1, &err);
        if (by.count("antenna2") && f.object_at(by["antenna2"], &oa2, &err)) f.read_int64(oa2.ds, &a2, &err);
        for (size_t t = 0; t < nt; t++) {
            const double len = std::sqrt(uvw[3 * t] * uvw[3 * t] + uvw[3 * t + 1] * uvw[3 * t + 1]);
            if (len < bl_min || len >= bl_max) continue;
            BaselineRecord r;
            r.a1 = t < a1.size() ? (int)a1[t] : -1;
            r.a2 = t < a2.size() ? (int)a2[t] : -1;
            r.time.assign(1, t < time.size() ? time[t] : 0.0);
            r.freq = freq;
            r.uvw.assign(uvw.begin() + 3 * t, uvw.begin() + 3 * t + 3);
            r.vis.assign(vis.begin() + 2 * t * nf, vis.begin() + 2 * (t + 1) * nf);
            fn(r);
        }
    } else {  // src/reference/hdf5.c:249-303: antenna_count = children + 1
        std::map<std::string, uint64_t> a1s;
        for (auto &e : ent) a1s[e.first] = e.second;
        const int antennas = (int)ent.size() + 1;
        for (int a1 = 0; a1 < antennas - 1; a1++) {
            auto it1 = a1s.find(std::to_string(a1));
            if (it1 == a1s.end()) continue;
            h5::Object g1;
            if (!f.object_at(it1->second, &g1, &err)) return fail(RG_ERR_IO, err);
            std::vector<std::pair<std::string, uint64_t>> e2;
            if (!f.entries(g1, &e2, &err)) return fail(RG_ERR_IO, err);
            std::map<std::string, uint64_t> a2s;
            for (auto &e : e2) a2s[e.first] = e.second;
            for (int a2 = a1 + 1; a2 < antennas; a2++) {
                auto it2 = a2s.find(std::to_string(a2));
                if (it2 == a2s.end()) continue;
                h5::Object g2;
                BaselineRecord r;
                bool kept = false;
                if (!f.object_at(it2->second, &g2, &err) || !read_baseline(f, g2, bl_min, bl_max, &r, &kept, &err))
                    return fail(RG_ERR_IO, "baseline " + std::to_string(a1) + "/" + std::to_string(a2) + ": " + err);
                if (!kept) continue;
                r.a1 = a1;
                r.a2 = a2;
                fn(r);
            }
        }
    }
    return RG_OK;
}

}  // namespace rg

extern "C" {

rg_status rg_read_vis_hdf5(const char *path, double bl_min, double bl_max, rg_vis_data *out)
{
    if (!path || !out) return fail(RG_ERR_INVALID_ARGUMENT, "path and out must be non-NULL");
    std::memset(out, 0, sizeof(*out));
    // flattened in baseline, time-major, frequency-minor order as
    // flatten_visibilities_CUDA does (src/common/hdf5.c:827-872)
    std::vector<double> u, v, w, vis;
    int64_t baselines = 0;
    RG_CHECK(rg::visit_vis_hdf5(path, bl_min, bl_max, [&](const BaselineRecord &r) {
        const size_t nt = r.time.size(), nf = r.freq.size();
        baselines++;
        for (size_t t = 0; t < nt; t++)
            for (size_t k = 0; k < nf; k++) {
                u.push_back(r.uvw[3 * t + 0] * r.freq[k] / kC);
                v.push_back(r.uvw[3 * t + 1] * r.freq[k] / kC);
                w.push_back(r.uvw[3 * t + 2] * r.freq[k] / kC);
                vis.push_back(r.vis[2 * (t * nf + k)]);
                vis.push_back(r.vis[2 * (t * nf + k) + 1]);
            }
    }));
    out->n = (int64_t)u.size();
    out->bl_count = baselines;
    out->u = copy_out(u);
    out->v = copy_out(v);
    out->w = copy_out(w);
    out->vis = copy_out(vis);
    if (!out->u || !out->v || !out->w || !out->vis) {
        rg_free_vis_data(out);
        return fail(RG_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    return RG_OK;
}

void rg_free_vis_data(rg_vis_data *d)
{
    if (!d) return;
    std::free(d->u);
    std::free(d->v);
    std::free(d->w);
    std::free(d->vis);
    std::memset(d, 0, sizeof(*d));
}

rg_status rg_read_wkern_hdf5(const char *path, double theta, rg_wkern_data *out)
{
    if (!path || !out) return fail(RG_ERR_INVALID_ARGUMENT, "path and out must be non-NULL");
    std::memset(out, 0, sizeof(*out));
    h5::File f;
    std::string err;
    if (!f.open(path, &err)) return fail(RG_ERR_IO, err);
    const std::string gname = "wkern/" + fmt_g(theta);  // src/reference/hdf5.c:339-341
    h5::Object g;
    if (!f.find(gname, &g, &err) || !g.is_group)
        return fail(RG_ERR_IO, "could not open '" + gname + "' in " + path);
    std::vector<std::pair<std::string, uint64_t>> ent;
    if (!f.entries(g, &ent, &err)) return fail(RG_ERR_IO, err);
    if (ent.empty()) return fail(RG_ERR_IO, std::string("no w-kernels in ") + path);
    struct Plane {
        double w;
        std::vector<double> data;
    };
    std::vector<Plane> planes;
    int ov = 0, sy = 0, sx = 0;
    for (auto &e : ent) {
        h5::Object pg, kd;
        std::vector<std::pair<std::string, uint64_t>> pe;
        if (!f.object_at(e.second, &pg, &err) || !f.entries(pg, &pe, &err)) return fail(RG_ERR_IO, err);
        uint64_t ka = 0;
        bool found = false;
        for (auto &q : pe)
            if (q.first == "kern") {
                ka = q.second;
                found = true;
            }
        if (!found || !f.object_at(ka, &kd, &err)) return fail(RG_ERR_IO, "plane " + e.first + " lacks 'kern'");
        if (kd.ds.dims.size() != 4) return fail(RG_ERR_IO, "w-kernel dataset must be 4-dimensional");
        const int d0 = (int)kd.ds.dims[0], d1 = (int)kd.ds.dims[1], d2 = (int)kd.ds.dims[2], d3 = (int)kd.ds.dims[3];
        if (ov == 0) {
            ov = d0;
            sy = d2;
            sx = d3;
        }
        if (d0 != ov || d1 != ov || d2 != sy || d3 != sx) continue;  // inconsistent planes are ignored
        Plane p;
        p.w = std::atof(e.first.c_str());
        if (!f.read_doubles(kd.ds, &p.data, &err)) return fail(RG_ERR_IO, err);
        planes.push_back(std::move(p));
    }
    if (planes.empty() || ov <= 0 || sx != sy) return fail(RG_ERR_IO, "invalid w-kernel dimensions");
    double wmin = planes[0].w, wmax = planes[0].w;
    for (auto &p : planes) {
        wmin = std::min(wmin, p.w);
        wmax = std::max(wmax, p.w);
    }
    const int n = (int)planes.size();
    const double step = n > 1 ? (wmax - wmin) / (n - 1) : 1.0;
    const size_t per = (size_t)ov * ov * sy * sx * 2;
    out->data = (double *)std::malloc(sizeof(double) * per * n);
    if (!out->data) return fail(RG_ERR_OUT_OF_MEMORY, "host allocation failed");
    for (int i = 0; i < n; i++) {  // kern_by_w: nearest kernel to w_min + i*step (hdf5.c:478-492)
        const double w = wmin + i * step;
        int best = 0;
        for (int j = 1; j < n; j++)
            if (std::fabs(planes[j].w - w) < std::fabs(planes[best].w - w)) best = j;
        std::memcpy(out->data + per * i, planes[best].data.data(), sizeof(double) * per);
    }
    out->plane_count = n;
    out->size = sx;
    out->oversampling = ov;
    out->w_min = wmin;
    out->w_step = step;
    return RG_OK;
}

void rg_free_wkern_data(rg_wkern_data *d)
{
    if (!d) return;
    std::free(d->data);
    std::memset(d, 0, sizeof(*d));
}

rg_status rg_write_vis_hdf5(const char *path, int n_bl, int n_time, int n_freq, const int *ant1, const int *ant2,
                            const double *time, const double *freq, const double *uvw, const double *vis)
{
    if (!path || n_bl < 0 || n_time < 1 || n_freq < 1 || (n_bl > 0 && (!ant1 || !ant2 || !time || !freq || !uvw || !vis)))
        return fail(RG_ERR_INVALID_ARGUMENT, "bad visibility arrays");
    h5::Writer wr;
    const int vg = wr.add_group(0, "vis");
    std::map<int, int> a1g;
    for (int b = 0; b < n_bl; b++) {
        if (!a1g.count(ant1[b])) a1g[ant1[b]] = wr.add_group(vg, std::to_string(ant1[b]));
        const int g = wr.add_group(a1g[ant1[b]], std::to_string(ant2[b]));
        wr.add_dataset_f64(g, "frequency", {(uint64_t)n_freq}, freq + (size_t)b * n_freq);
        wr.add_dataset_f64(g, "time", {(uint64_t)n_time}, time + (size_t)b * n_time);
        wr.add_dataset_f64(g, "uvw", {(uint64_t)n_time, 3}, uvw + (size_t)b * n_time * 3);
        wr.add_dataset_c128(g, "vis", {(uint64_t)n_time, (uint64_t)n_freq, 1}, vis + (size_t)b * n_time * n_freq * 2);
    }
    std::string err;
    if (!wr.write(path, &err)) return fail(RG_ERR_IO, err);
    return RG_OK;
}

rg_status rg_write_vis_flat_hdf5(const char *path, int n_rows, int n_freq, const int *ant1, const int *ant2,
                                 const double *time, const double *freq, const double *uvw, const double *vis)
{
    if (!path || n_rows < 0 || n_freq < 1 || (n_rows > 0 && (!ant1 || !ant2 || !time || !freq || !uvw || !vis)))
        return fail(RG_ERR_INVALID_ARGUMENT, "bad visibility arrays");
    h5::Writer wr;
    const int vg = wr.add_group(0, "vis");
    wr.add_attr_str(vg, "type", "Visibility");
    std::vector<int64_t> a1(ant1, ant1 + n_rows), a2(ant2, ant2 + n_rows);
    wr.add_dataset_i64(vg, "antenna1", {(uint64_t)n_rows}, a1.data());
    wr.add_dataset_i64(vg, "antenna2", {(uint64_t)n_rows}, a2.data());
    wr.add_dataset_f64(vg, "frequency", {(uint64_t)n_freq}, freq);
    wr.add_dataset_f64(vg, "time", {(uint64_t)n_rows}, time);
    wr.add_dataset_f64(vg, "uvw", {(uint64_t)n_rows, 3}, uvw);
    wr.add_dataset_c128(vg, "vis", {(uint64_t)n_rows, (uint64_t)n_freq, 1}, vis);
    std::string err;
    if (!wr.write(path, &err)) return fail(RG_ERR_IO, err);
    return RG_OK;
}

rg_status rg_write_wkern_hdf5(const char *path, double theta, const rg_wkern *wk)
{
    if (!path || !wk || !wk->data || wk->plane_count < 1 || wk->size < 1 || wk->oversampling < 1)
        return fail(RG_ERR_INVALID_ARGUMENT, "bad w-kernel table");
    h5::Writer wr;
    const int g0 = wr.add_group(0, "wkern");
    const int g1 = wr.add_group(g0, fmt_g(theta));
    const size_t per = (size_t)wk->oversampling * wk->oversampling * wk->size * wk->size * 2;
    for (int p = 0; p < wk->plane_count; p++) {
        char name[64];
        std::snprintf(name, sizeof(name), "%.17g", wk->w_min + p * wk->w_step);
        const int g = wr.add_group(g1, name);
        const uint64_t ov = (uint64_t)wk->oversampling, s = (uint64_t)wk->size;
        wr.add_dataset_c128(g, "kern", {ov, ov, s, s}, wk->data + per * p);
    }
    std::string err;
    if (!wr.write(path, &err)) return fail(RG_ERR_IO, err);
    return RG_OK;
}

}  // extern "C"

extern "C" {

rg_status rg_hdf5_read_f64(const char *path, const char *dataset, double *out, int64_t capacity, int64_t *dims,
                           int *ndims)
{
    if (!path || !dataset || !ndims) return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    h5::File f;
    std::string err;
    if (!f.open(path, &err)) return fail(RG_ERR_IO, err);
    h5::Object o;
    if (!f.find(dataset, &o, &err) || o.is_group) return fail(RG_ERR_IO, std::string("no dataset ") + dataset);
    // a compound {r, i} element reads as a trailing axis of its member count
    std::vector<uint64_t> shape = o.ds.dims;
    if (o.ds.type.cls == 6) shape.push_back(o.ds.type.members.size());
    if (shape.size() > 8) return fail(RG_ERR_UNSUPPORTED, "more than 8 dimensions");
    *ndims = (int)shape.size();
    for (size_t i = 0; i < shape.size() && dims; i++) dims[i] = (int64_t)shape[i];
    if (!out) return RG_OK;
    std::vector<double> v;
    if (!f.read_doubles(o.ds, &v, &err)) return fail(RG_ERR_IO, err);
    if ((int64_t)v.size() > capacity) return fail(RG_ERR_INVALID_ARGUMENT, "output capacity too small");
    std::memcpy(out, v.data(), sizeof(double) * v.size());
    return RG_OK;
}

rg_status rg_hdf5_attr_f64(const char *path, const char *object, const char *name, double *out)
{
    if (!path || !object || !name || !out) return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    h5::File f;
    std::string err;
    if (!f.open(path, &err)) return fail(RG_ERR_IO, err);
    h5::Object o;
    if (!f.find(object, &o, &err)) return fail(RG_ERR_IO, std::string("no object ") + object);
    if (!f.attr_double(o, name, out)) return fail(RG_ERR_IO, std::string("no numeric attribute ") + name);
    return RG_OK;
}

}  // extern "C"
