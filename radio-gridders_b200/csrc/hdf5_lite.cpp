// HDF5 subset reader/writer (see hdf5_lite.h).  Field layouts follow the HDF5
// File Format Specification: superblock versions 0/1 (II.A), symbol table
// entries (III.C), version-1 B-trees of group nodes (III.A.1), symbol table
// nodes (III.B), local heaps (III.D), version-1 object headers (IV.A.1) and the
// dataspace, datatype, fill value, layout, attribute, continuation and symbol
// table messages (IV.A.2).
#include "hdf5_lite.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>

namespace h5 {

static const uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
static const uint64_t kUndef = ~0ull;

static uint64_t pad8(uint64_t n) { return (n + 7) & ~7ull; }

uint64_t File::get(uint64_t off, int n) const
{
    uint64_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint64_t)buf_[off + i] << (8 * i);
    return v;
}

bool File::open(const std::string &path, std::string *err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        *err = "cannot open " + path;
        return false;
    }
    buf_.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    uint64_t sb = kUndef;
    for (uint64_t off = 0; off + 8 <= buf_.size(); off = off ? off * 2 : 512) {
        if (std::memcmp(buf_.data() + off, kSig, 8) == 0) {
            sb = off;
            break;
        }
        if (off > (1ull << 40)) break;
    }
    if (sb == kUndef || !inb(sb, 24)) {
        *err = path + " is not an HDF5 file";
        return false;
    }
    const int version = buf_[sb + 8];
    if (version > 1) {
        *err = "HDF5 superblock version " + std::to_string(version) + " is not supported (0 or 1)";
        return false;
    }
    so_ = buf_[sb + 13];
    sl_ = buf_[sb + 14];
    if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) {
        *err = "unsupported HDF5 offset/length sizes";
        return false;
    }
    uint64_t p = sb + (version == 0 ? 24 : 28);
    if (!inb(p, 4 * so_ + 2 * so_ + 24)) {
        *err = "truncated HDF5 superblock";
        return false;
    }
    base_ = get(p, so_);
    p += 4 * so_;                     // base, free-space, end-of-file, driver info
    root_ohdr_ = get(p + so_, so_);  // root symbol table entry: name offset, object header
    return true;
}

static bool parse_type(const uint8_t *d, size_t avail, Type *t, size_t *used, std::string *err)
{
    if (avail < 8) {
        *err = "truncated datatype";
        return false;
    }
    t->cls = d[0] & 0x0f;
    const int version = d[0] >> 4;
    t->size = (uint32_t)(d[4] | (d[5] << 8) | (d[6] << 16) | ((uint32_t)d[7] << 24));
    size_t n = 8;
    switch (t->cls) {
        case 0:  // fixed point
            if (d[1] & 1) {
                *err = "big-endian integers are not supported";
                return false;
            }
            t->is_signed = (d[1] & 0x08) != 0;
            n += 4;
            break;
        case 1:  // floating point
            if (d[1] & 1) {
                *err = "big-endian floats are not supported";
                return false;
            }
            n += 12;
            break;
        case 3:  // fixed-length string
            break;
        case 6: {  // compound
            const int nmem = d[1] | (d[2] << 8);
            for (int m = 0; m < nmem; m++) {
                std::string name((const char *)d + n, strnlen((const char *)d + n, avail - n));
                size_t off_member;
                if (version < 3) {
                    n += pad8(name.size() + 1);
                    if (n + 4 > avail) { *err = "truncated compound"; return false; }
                    off_member = d[n] | (d[n + 1] << 8) | (d[n + 2] << 16) | ((size_t)d[n + 3] << 24);
                    n += 4;
                    if (version == 1) n += 28;  // dimensionality, permutation, dimension sizes
                } else {
                    n += name.size() + 1;
                    int ob = 1;
                    while ((1ull << (8 * ob)) <= t->size && ob < 8) ob++;
                    off_member = 0;
                    for (int i = 0; i < ob; i++) off_member |= (size_t)d[n + i] << (8 * i);
                    n += ob;
                }
                Type mt;
                size_t mu = 0;
                if (!parse_type(d + n, avail - n, &mt, &mu, err)) return false;
                n += mu;
                t->members.emplace_back(name, (uint32_t)off_member);
                t->member_types.push_back(mt);
            }
            break;
        }
        default:
            *err = "HDF5 datatype class " + std::to_string(t->cls) + " is not supported";
            return false;
    }
    *used = n;
    return true;
}

bool File::parse_object(uint64_t addr, Object *o, std::string *err)
{
    const uint64_t a = base_ + addr;
    if (!inb(a, 16) || buf_[a] != 1) {
        *err = "unsupported or corrupt object header (only version 1 headers are read)";
        return false;
    }
    const int nmsg = (int)get(a + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks = {{a + 16, get(a + 8, 4)}};
    int seen = 0;
    for (size_t bi = 0; bi < blocks.size() && seen < nmsg; bi++) {
        uint64_t p = blocks[bi].first, end = p + blocks[bi].second;
        if (!inb(blocks[bi].first, blocks[bi].second)) {
            *err = "object header block outside the file";
            return false;
        }
        while (p + 8 <= end && seen < nmsg) {
            const int type = (int)get(p, 2);
            const uint64_t size = get(p + 2, 2);
            const uint8_t *d = buf_.data() + p + 8;
            if (p + 8 + size > end) {
                *err = "object header message overruns its block";
                return false;
            }
            seen++;
            switch (type) {
                case 0x0001: {  // dataspace
                    const int ver = d[0], nd = d[1];
                    const uint8_t *dims = d + (ver == 1 ? 8 : 4);
                    o->ds.dims.clear();
                    for (int i = 0; i < nd; i++) {
                        uint64_t v = 0;
                        for (int b = 0; b < sl_; b++) v |= (uint64_t)dims[i * sl_ + b] << (8 * b);
                        o->ds.dims.push_back(v);
                    }
                    break;
                }
                case 0x0003: {
                    size_t used;
                    if (!parse_type(d, size, &o->ds.type, &used, err)) return false;
                    break;
                }
                case 0x0008: {  // layout
                    const int ver = d[0];
                    if (ver >= 3) {
                        const int cls = d[1];
                        if (cls == 1) {
                            uint64_t v = 0, s = 0;
                            for (int b = 0; b < so_; b++) v |= (uint64_t)d[2 + b] << (8 * b);
                            for (int b = 0; b < sl_; b++) s |= (uint64_t)d[2 + so_ + b] << (8 * b);
                            o->ds.address = v;
                            o->ds.bytes = s;
                        } else if (cls == 0) {
                            const int n = d[2] | (d[3] << 8);
                            o->ds.compact.assign(d + 4, d + 4 + n);
                            o->ds.is_compact = true;
                            o->ds.bytes = n;
                        } else {
                            *err = "chunked HDF5 datasets are not supported";
                            return false;
                        }
                    } else {
                        const int cls = d[2];
                        if (cls != 1) {
                            *err = "only contiguous version-1/2 layouts are supported";
                            return false;
                        }
                        uint64_t v = 0;
                        for (int b = 0; b < so_; b++) v |= (uint64_t)d[8 + b] << (8 * b);
                        o->ds.address = v;
                        o->ds.bytes = 0;  // computed from dims and type
                    }
                    break;
                }
                case 0x0011: {  // symbol table
                    o->is_group = true;
                    o->btree = 0;
                    o->heap = 0;
                    for (int b = 0; b < so_; b++) o->btree |= (uint64_t)d[b] << (8 * b);
                    for (int b = 0; b < so_; b++) o->heap |= (uint64_t)d[so_ + b] << (8 * b);
                    break;
                }
                case 0x0010: {  // continuation
                    uint64_t off = 0, len = 0;
                    for (int b = 0; b < so_; b++) off |= (uint64_t)d[b] << (8 * b);
                    for (int b = 0; b < sl_; b++) len |= (uint64_t)d[so_ + b] << (8 * b);
                    blocks.emplace_back(base_ + off, len);
                    break;
                }
                case 0x000C: {  // attribute
                    const int ver = d[0];
                    const int name_size = d[2] | (d[3] << 8);
                    const int dt_size = d[4] | (d[5] << 8);
                    const int ds_size = d[6] | (d[7] << 8);
                    size_t q = ver == 3 ? 9 : 8;
                    std::string name((const char *)d + q, strnlen((const char *)d + q, name_size));
                    q += ver == 1 ? pad8(name_size) : name_size;
                    Type t;
                    size_t used;
                    if (!parse_type(d + q, dt_size, &t, &used, err)) {
                        err->clear();  // an unreadable attribute is ignored
                        break;
                    }
                    q += ver == 1 ? pad8(dt_size) : dt_size;
                    const uint8_t *sp = d + q;
                    uint64_t count = 1;
                    const int nd = sp[1];
                    const uint8_t *dims = sp + (sp[0] == 1 ? 8 : 4);
                    for (int i = 0; i < nd; i++) {
                        uint64_t v = 0;
                        for (int b = 0; b < sl_; b++) v |= (uint64_t)dims[i * sl_ + b] << (8 * b);
                        count *= v;
                    }
                    q += ver == 1 ? pad8(ds_size) : ds_size;
                    const uint64_t nbytes = count * t.size;
                    if (q + nbytes <= size) {
                        o->attr_raw[name].assign(d + q, d + q + nbytes);
                        o->attr_type[name] = t;
                    }
                    break;
                }
                default:
                    break;
            }
            p += 8 + size;
        }
    }
    return true;
}

bool File::walk_btree(uint64_t addr, uint64_t heap_data, std::vector<std::pair<std::string, uint64_t>> *out,
                      std::string *err, int depth)
{
    const uint64_t a = base_ + addr;
    if (depth > 32 || !inb(a, 8 + 2 * so_) || std::memcmp(buf_.data() + a, "TREE", 4) != 0 || buf_[a + 4] != 0) {
        *err = "corrupt group B-tree";
        return false;
    }
    const int level = buf_[a + 5];
    const int entries = (int)get(a + 6, 2);
    uint64_t p = a + 8 + 2 * so_;
    for (int i = 0; i < entries; i++) {
        p += sl_;  // key
        if (!inb(p, so_)) {
            *err = "truncated group B-tree";
            return false;
        }
        const uint64_t child = get(p, so_);
        p += so_;
        if (level > 0) {
            if (!walk_btree(child, heap_data, out, err, depth + 1)) return false;
            continue;
        }
        const uint64_t s = base_ + child;
        if (!inb(s, 8) || std::memcmp(buf_.data() + s, "SNOD", 4) != 0) {
            *err = "corrupt symbol table node";
            return false;
        }
        const int nsym = (int)get(s + 6, 2);
        const uint64_t esz = 2 * so_ + 24;
        for (int k = 0; k < nsym; k++) {
            const uint64_t e = s + 8 + k * esz;
            if (!inb(e, esz)) {
                *err = "truncated symbol table node";
                return false;
            }
            const uint64_t name_off = get(e, so_), ohdr = get(e + so_, so_);
            const uint64_t np = heap_data + name_off;
            if (!inb(np, 1)) {
                *err = "symbol name outside the file";
                return false;
            }
            out->emplace_back(std::string((const char *)buf_.data() + np,
                                          strnlen((const char *)buf_.data() + np, buf_.size() - np)),
                              ohdr);
        }
    }
    return true;
}

bool File::children(const Object &g, std::vector<std::string> *names, std::string *err)
{
    if (!g.is_group) {
        *err = "not a group";
        return false;
    }
    const uint64_t h = base_ + g.heap;
    if (!inb(h, 8 + 2 * sl_ + so_) || std::memcmp(buf_.data() + h, "HEAP", 4) != 0) {
        *err = "corrupt local heap";
        return false;
    }
    const uint64_t data = base_ + get(h + 8 + 2 * sl_, so_);
    std::vector<std::pair<std::string, uint64_t>> ent;
    if (!walk_btree(g.btree, data, &ent, err, 0)) return false;
    names->clear();
    for (auto &e : ent) names->push_back(e.first);
    return true;
}

bool File::entries(const Object &g, std::vector<std::pair<std::string, uint64_t>> *out, std::string *err)
{
    if (!g.is_group) {
        *err = "not a group";
        return false;
    }
    const uint64_t h = base_ + g.heap;
    if (!inb(h, 8 + 2 * sl_ + so_) || std::memcmp(buf_.data() + h, "HEAP", 4) != 0) {
        *err = "corrupt local heap";
        return false;
    }
    const uint64_t data = base_ + get(h + 8 + 2 * sl_, so_);
    out->clear();
    return walk_btree(g.btree, data, out, err, 0);
}

bool File::object_at(uint64_t addr, Object *o, std::string *err) { return parse_object(addr, o, err); }

bool File::child_addr(const Object &g, const std::string &name, uint64_t *addr, std::string *err)
{
    const uint64_t h = base_ + g.heap;
    if (!inb(h, 8 + 2 * sl_ + so_) || std::memcmp(buf_.data() + h, "HEAP", 4) != 0) {
        *err = "corrupt local heap";
        return false;
    }
    const uint64_t data = base_ + get(h + 8 + 2 * sl_, so_);
    std::vector<std::pair<std::string, uint64_t>> ent;
    if (!walk_btree(g.btree, data, &ent, err, 0)) return false;
    for (auto &e : ent)
        if (e.first == name) {
            *addr = e.second;
            return true;
        }
    return false;
}

bool File::find(const std::string &path, Object *out, std::string *err)
{
    Object cur;
    if (!parse_object(root_ohdr_, &cur, err)) return false;
    size_t i = 0;
    while (i < path.size()) {
        while (i < path.size() && path[i] == '/') i++;
        if (i >= path.size()) break;
        size_t j = path.find('/', i);
        const std::string comp = path.substr(i, j == std::string::npos ? std::string::npos : j - i);
        i = j == std::string::npos ? path.size() : j;
        if (!cur.is_group) return false;
        uint64_t addr;
        if (!child_addr(cur, comp, &addr, err)) return false;
        Object next;
        if (!parse_object(addr, &next, err)) return false;
        cur = next;
    }
    *out = cur;
    return true;
}

static uint64_t count_of(const Dataset &ds)
{
    uint64_t n = 1;
    for (auto d : ds.dims) n *= d;
    return n;
}

bool File::read_doubles(const Dataset &ds, std::vector<double> *out, std::string *err)
{
    const uint64_t n = count_of(ds);
    const Type &t = ds.type;
    int per = 0;
    if (t.cls == 1 && t.size == 8) per = 1;
    else if (t.cls == 6 && t.size == 16 && t.members.size() == 2 && t.member_types[0].cls == 1 &&
             t.member_types[0].size == 8 && t.member_types[1].cls == 1 && t.member_types[1].size == 8 &&
             t.members[0].second == 0 && t.members[1].second == 8)
        per = 2;
    else if (t.cls == 0 && t.size == 8) {
        std::vector<int64_t> v;
        if (!read_int64(ds, &v, err)) return false;
        out->assign(v.begin(), v.end());
        return true;
    } else {
        *err = "dataset is not float64, int64 or a {float64, float64} compound";
        return false;
    }
    const uint64_t bytes = n * 8 * per;
    out->resize(n * per);
    if (ds.is_compact) {
        if (ds.compact.size() < bytes) { *err = "short compact dataset"; return false; }
        std::memcpy(out->data(), ds.compact.data(), bytes);
        return true;
    }
    if (ds.address == kUndef || !inb(base_ + ds.address, bytes)) {
        *err = "dataset data outside the file";
        return false;
    }
    std::memcpy(out->data(), buf_.data() + base_ + ds.address, bytes);
    return true;
}

bool File::read_int64(const Dataset &ds, std::vector<int64_t> *out, std::string *err)
{
    const uint64_t n = count_of(ds);
    if (ds.type.cls != 0 || (ds.type.size != 8 && ds.type.size != 4)) {
        *err = "dataset is not an integer";
        return false;
    }
    const uint64_t bytes = n * ds.type.size;
    const uint8_t *src = nullptr;
    if (ds.is_compact) src = ds.compact.size() >= bytes ? ds.compact.data() : nullptr;
    else if (ds.address != kUndef && inb(base_ + ds.address, bytes)) src = buf_.data() + base_ + ds.address;
    if (!src) {
        *err = "dataset data outside the file";
        return false;
    }
    out->resize(n);
    for (uint64_t i = 0; i < n; i++) {
        if (ds.type.size == 8) {
            int64_t v;
            std::memcpy(&v, src + 8 * i, 8);
            (*out)[i] = v;
        } else {
            int32_t v;
            std::memcpy(&v, src + 4 * i, 4);
            (*out)[i] = ds.type.is_signed ? v : (int64_t)(uint32_t)v;
        }
    }
    return true;
}

bool File::attr_double(const Object &o, const std::string &name, double *v)
{
    auto it = o.attr_raw.find(name);
    if (it == o.attr_raw.end()) return false;
    const Type &t = o.attr_type.at(name);
    if (t.cls == 1 && t.size == 8 && it->second.size() >= 8) {
        std::memcpy(v, it->second.data(), 8);
        return true;
    }
    if (t.cls == 1 && t.size == 4 && it->second.size() >= 4) {
        float f;
        std::memcpy(&f, it->second.data(), 4);
        *v = f;
        return true;
    }
    if (t.cls == 0 && t.size == 8 && it->second.size() >= 8) {
        int64_t i;
        std::memcpy(&i, it->second.data(), 8);
        *v = (double)i;
        return true;
    }
    return false;
}

bool File::attr_string(const Object &o, const std::string &name, std::string *v)
{
    auto it = o.attr_raw.find(name);
    if (it == o.attr_raw.end() || o.attr_type.at(name).cls != 3) return false;
    v->assign((const char *)it->second.data(), strnlen((const char *)it->second.data(), it->second.size()));
    return true;
}

// ---------------------------------------------------------------------------
// writer
// ---------------------------------------------------------------------------
namespace {
constexpr int kLeafK = 4;  // symbol table node capacity 2K (the library default)

struct Out {
    std::vector<uint8_t> b;
    uint64_t alloc(uint64_t n)
    {
        const uint64_t a = pad8(b.size());
        b.resize(a + pad8(n), 0);
        return a;
    }
    void put(uint64_t at, uint64_t v, int n)
    {
        for (int i = 0; i < n; i++) b[at + i] = (uint8_t)(v >> (8 * i));
    }
};

void type_f64(std::vector<uint8_t> &m)
{
    const uint8_t t[20] = {0x11, 0x20, 63, 0, 8, 0, 0, 0, 0, 0, 64, 0, 52, 11, 0, 52, 0xff, 0x03, 0, 0};
    m.insert(m.end(), t, t + 20);
}

void type_i64(std::vector<uint8_t> &m)
{
    const uint8_t t[12] = {0x10, 0x08, 0, 0, 8, 0, 0, 0, 0, 0, 64, 0};
    m.insert(m.end(), t, t + 12);
}

void type_c128(std::vector<uint8_t> &m)
{
    const uint8_t head[8] = {0x16, 2, 0, 0, 16, 0, 0, 0};
    m.insert(m.end(), head, head + 8);
    for (int k = 0; k < 2; k++) {
        uint8_t name[8] = {0};
        name[0] = k == 0 ? 'r' : 'i';
        m.insert(m.end(), name, name + 8);
        uint8_t off[4] = {(uint8_t)(8 * k), 0, 0, 0};
        m.insert(m.end(), off, off + 4);
        uint8_t dims[28] = {0};  // dimensionality 0, reserved, permutation, reserved, sizes
        m.insert(m.end(), dims, dims + 28);
        type_f64(m);
    }
}

void message(std::vector<uint8_t> &area, int type, const std::vector<uint8_t> &data)
{
    const uint64_t n = pad8(data.size());
    const uint8_t h[8] = {(uint8_t)type, (uint8_t)(type >> 8), (uint8_t)n, (uint8_t)(n >> 8), 0, 0, 0, 0};
    area.insert(area.end(), h, h + 8);
    area.insert(area.end(), data.begin(), data.end());
    area.resize(area.size() + (n - data.size()), 0);
}
}  // namespace

struct Writer::Node {
    bool group = true;
    std::string name;
    int parent = -1;
    std::vector<int> kids;
    std::vector<uint64_t> dims;
    int kind = 0;  // 1 f64, 2 i64, 3 c128
    std::vector<uint8_t> data;
    std::vector<std::pair<std::string, double>> attrs;
    std::vector<std::pair<std::string, std::string>> sattrs;
    uint64_t ohdr = 0;
};

Writer::Writer() { nodes_.push_back(new Node()); }

int Writer::add_group(int parent, const std::string &name)
{
    Node *n = new Node();
    n->name = name;
    n->parent = parent;
    nodes_.push_back(n);
    const int id = (int)nodes_.size() - 1;
    nodes_[parent]->kids.push_back(id);
    return id;
}

void Writer::add_dataset(int parent, const std::string &name, const std::vector<uint64_t> &dims, int kind,
                         const void *data, size_t elem)
{
    Node *n = new Node();
    n->group = false;
    n->name = name;
    n->parent = parent;
    n->dims = dims;
    n->kind = kind;
    uint64_t count = 1;
    for (auto d : dims) count *= d;
    n->data.assign((const uint8_t *)data, (const uint8_t *)data + count * elem);
    nodes_.push_back(n);
    nodes_[parent]->kids.push_back((int)nodes_.size() - 1);
}

void Writer::add_dataset_f64(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                             const double *data)
{
    add_dataset(parent, name, dims, 1, data, 8);
}

void Writer::add_dataset_i64(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                             const int64_t *data)
{
    add_dataset(parent, name, dims, 2, data, 8);
}

void Writer::add_dataset_c128(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                              const double *interleaved)
{
    add_dataset(parent, name, dims, 3, interleaved, 16);
}

void Writer::add_attr_f64(int group, const std::string &name, double v) { nodes_[group]->attrs.emplace_back(name, v); }

void Writer::add_attr_str(int group, const std::string &name, const std::string &v)
{
    nodes_[group]->sattrs.emplace_back(name, v);
}

bool Writer::write(const std::string &path, std::string *err)
{
    // B-tree node capacity 2K children, K >= 16 (the library default), large
    // enough that every group fits one leaf-level B-tree node
    size_t most = 0;
    for (Node *n : nodes_) most = std::max(most, n->kids.size());
    const size_t snods = (most + 2 * kLeafK - 1) / (2 * kLeafK);
    const int kInternalK = (int)std::max<size_t>(16, (snods + 1) / 2);
    Out o;
    const uint64_t sb = o.alloc(96);  // superblock v0 + root symbol table entry
    // objects, children before parents so addresses are known
    struct GroupAddr {
        uint64_t btree, heap;
    };
    std::vector<GroupAddr> gaddr(nodes_.size());
    std::function<void(int)> build = [&](int id) {
        Node *n = nodes_[id];
        if (!n->group) {
            std::vector<uint8_t> area;
            std::vector<uint8_t> sp = {1, (uint8_t)n->dims.size(), 0, 0, 0, 0, 0, 0};
            for (auto d : n->dims)
                for (int b = 0; b < 8; b++) sp.push_back((uint8_t)(d >> (8 * b)));
            message(area, 0x0001, sp);
            std::vector<uint8_t> dt;
            if (n->kind == 1) type_f64(dt);
            else if (n->kind == 2) type_i64(dt);
            else type_c128(dt);
            message(area, 0x0003, dt);
            message(area, 0x0005, {2, 1, 2, 0});  // fill value: early allocation, never written
            const uint64_t hdr = o.alloc(16 + area.size() + 8 * 4);
            const uint64_t dat = o.alloc(n->data.size());
            std::memcpy(o.b.data() + dat, n->data.data(), n->data.size());
            std::vector<uint8_t> lay = {3, 1};
            for (int b = 0; b < 8; b++) lay.push_back((uint8_t)(dat >> (8 * b)));
            for (int b = 0; b < 8; b++) lay.push_back((uint8_t)((uint64_t)n->data.size() >> (8 * b)));
            message(area, 0x0008, lay);
            o.b[hdr] = 1;
            o.put(hdr + 2, 4, 2);  // messages
            o.put(hdr + 4, 1, 4);  // reference count
            o.put(hdr + 8, area.size(), 4);
            o.b.resize(std::max<size_t>(o.b.size(), hdr + 16 + area.size()));
            std::memcpy(o.b.data() + hdr + 16, area.data(), area.size());
            n->ohdr = hdr;
            return;
        }
        for (int k : n->kids) build(k);
        // children sorted by name (B-tree order)
        std::vector<int> kids = n->kids;
        std::sort(kids.begin(), kids.end(), [&](int a, int b) { return nodes_[a]->name < nodes_[b]->name; });
        // local heap: "" at 0, then names
        std::vector<uint8_t> heap(8, 0);
        std::vector<uint64_t> name_off;
        for (int k : kids) {
            name_off.push_back(heap.size());
            const std::string &s = nodes_[k]->name;
            heap.insert(heap.end(), s.begin(), s.end());
            heap.resize(pad8(heap.size() + 1), 0);
        }
        const uint64_t heap_data = o.alloc(heap.size());
        std::memcpy(o.b.data() + heap_data, heap.data(), heap.size());
        const uint64_t hh = o.alloc(32);
        std::memcpy(o.b.data() + hh, "HEAP", 4);
        o.put(hh + 8, heap.size(), 8);
        o.put(hh + 16, kUndef, 8);
        o.put(hh + 24, heap_data, 8);
        // symbol table nodes of up to 2*kLeafK entries
        const int per = 2 * kLeafK;
        const int nsnod = (int)((kids.size() + per - 1) / per);
        if (nsnod > 2 * kInternalK) {
            *err = "group too large for the writer";
            return;
        }
        std::vector<uint64_t> snods;
        for (int s = 0; s < std::max(nsnod, 1); s++) {
            const uint64_t a = o.alloc(8 + per * 40);
            std::memcpy(o.b.data() + a, "SNOD", 4);
            o.b[a + 4] = 1;
            const int cnt = (int)std::min<size_t>(per, kids.size() - std::min<size_t>(kids.size(), (size_t)s * per));
            o.put(a + 6, cnt, 2);
            for (int e = 0; e < cnt; e++) {
                const int k = kids[s * per + e];
                o.put(a + 8 + e * 40, name_off[s * per + e], 8);
                o.put(a + 8 + e * 40 + 8, nodes_[k]->ohdr, 8);
            }
            snods.push_back(a);
        }
        const uint64_t bt = o.alloc(24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8);
        std::memcpy(o.b.data() + bt, "TREE", 4);
        o.b[bt + 4] = 0;  // group node
        o.b[bt + 5] = 0;  // leaf level
        const int used = kids.empty() ? 0 : nsnod;
        o.put(bt + 6, used, 2);
        o.put(bt + 8, kUndef, 8);
        o.put(bt + 16, kUndef, 8);
        uint64_t p = bt + 24;
        o.put(p, 0, 8);  // key 0: the empty name
        p += 8;
        for (int s = 0; s < used; s++) {
            o.put(p, snods[s], 8);
            p += 8;
            const size_t last = std::min(kids.size(), (size_t)(s + 1) * per) - 1;
            o.put(p, name_off[last], 8);
            p += 8;
        }
        gaddr[id] = {bt, hh};
        std::vector<uint8_t> area;
        std::vector<uint8_t> stab;
        for (int b = 0; b < 8; b++) stab.push_back((uint8_t)(bt >> (8 * b)));
        for (int b = 0; b < 8; b++) stab.push_back((uint8_t)(hh >> (8 * b)));
        message(area, 0x0011, stab);
        for (auto &at : n->attrs) {
            std::vector<uint8_t> m = {1, 0, (uint8_t)(at.first.size() + 1), 0, 20, 0, 8, 0};
            std::vector<uint8_t> nm(at.first.begin(), at.first.end());
            nm.resize(pad8(at.first.size() + 1), 0);
            m.insert(m.end(), nm.begin(), nm.end());
            std::vector<uint8_t> dt;
            type_f64(dt);
            dt.resize(24, 0);
            m.insert(m.end(), dt.begin(), dt.end());
            const uint8_t space[8] = {1, 0, 0, 0, 0, 0, 0, 0};
            m.insert(m.end(), space, space + 8);
            uint8_t val[8];
            std::memcpy(val, &at.second, 8);
            m.insert(m.end(), val, val + 8);
            message(area, 0x000C, m);
        }
        for (auto &at : n->sattrs) {
            // attribute message v1: string datatype (class 3, version 1, null
            // terminated ASCII, no properties: 8 bytes), scalar dataspace
            const uint32_t len = (uint32_t)at.second.size() + 1;
            std::vector<uint8_t> m = {1, 0, (uint8_t)(at.first.size() + 1), 0, 8, 0, 8, 0};
            std::vector<uint8_t> nm(at.first.begin(), at.first.end());
            nm.resize(pad8(at.first.size() + 1), 0);
            m.insert(m.end(), nm.begin(), nm.end());
            const uint8_t dt[8] = {0x13, 0, 0, 0, (uint8_t)len, (uint8_t)(len >> 8), (uint8_t)(len >> 16),
                                   (uint8_t)(len >> 24)};
            m.insert(m.end(), dt, dt + 8);
            const uint8_t space[8] = {1, 0, 0, 0, 0, 0, 0, 0};
            m.insert(m.end(), space, space + 8);
            std::vector<uint8_t> val(at.second.begin(), at.second.end());
            val.push_back(0);
            m.insert(m.end(), val.begin(), val.end());
            message(area, 0x000C, m);
        }
        const uint64_t hdr = o.alloc(16 + area.size());
        o.b[hdr] = 1;
        o.put(hdr + 2, 1 + n->attrs.size() + n->sattrs.size(), 2);
        o.put(hdr + 4, 1, 4);
        o.put(hdr + 8, area.size(), 4);
        std::memcpy(o.b.data() + hdr + 16, area.data(), area.size());
        n->ohdr = hdr;
    };
    err->clear();
    build(0);
    if (!err->empty()) return false;
    // superblock version 0
    std::memcpy(o.b.data() + sb, kSig, 8);
    o.b[sb + 13] = 8;
    o.b[sb + 14] = 8;
    o.put(sb + 16, kLeafK, 2);
    o.put(sb + 18, kInternalK, 2);
    o.put(sb + 24, 0, 8);            // base address
    o.put(sb + 32, kUndef, 8);       // free-space info
    o.put(sb + 40, o.b.size(), 8);   // end of file
    o.put(sb + 48, kUndef, 8);       // driver info
    o.put(sb + 56, 0, 8);            // root: link name offset
    o.put(sb + 64, nodes_[0]->ohdr, 8);
    o.put(sb + 72, 1, 4);            // cache type 1: scratch holds B-tree and heap addresses
    o.put(sb + 80, gaddr[0].btree, 8);
    o.put(sb + 88, gaddr[0].heap, 8);
    std::ofstream f(path, std::ios::binary);
    if (!f) {
        *err = "cannot create " + path;
        return false;
    }
    f.write((const char *)o.b.data(), (std::streamsize)o.b.size());
    return (bool)f;
}

}  // namespace h5
