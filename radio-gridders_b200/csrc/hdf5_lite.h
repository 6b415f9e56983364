// A small reader/writer for the subset of HDF5 the crocodile visibility and
// w-kernel files use (the files the reference reads with libhdf5 in
// src/reference/hdf5.c and src/common/hdf5.c): superblock version 0/1,
// version-1 object headers with continuation blocks, symbol-table groups
// (version-1 B-trees, symbol nodes, local heaps), contiguous or compact
// datasets, little-endian IEEE float/integer and compound types, fixed-length
// string and scalar numeric attributes.  Written from the published HDF5 file
// format specification (version 2.0 document, sections II-IV).
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace h5 {

struct Type {
    int cls = -1;          // 0 fixed-point, 1 float, 3 string, 6 compound
    uint32_t size = 0;
    bool is_signed = false;
    std::vector<std::pair<std::string, uint32_t>> members;  // compound: name, offset
    std::vector<Type> member_types;
};

struct Dataset {
    std::vector<uint64_t> dims;
    Type type;
    uint64_t address = UINT64_MAX;  // contiguous
    uint64_t bytes = 0;
    std::vector<uint8_t> compact;   // compact layout
    bool is_compact = false;
};

struct Object {
    bool is_group = false;
    uint64_t btree = 0, heap = 0;   // group
    Dataset ds;                     // dataset
    std::map<std::string, std::vector<uint8_t>> attr_raw;
    std::map<std::string, Type> attr_type;
};

class File {
public:
    bool open(const std::string &path, std::string *err);
    // object at a '/'-separated path from the root; false if missing
    bool find(const std::string &path, Object *out, std::string *err);
    // children names of a group, sorted as the B-tree stores them
    bool children(const Object &group, std::vector<std::string> *names, std::string *err);
    // (name, object header address) of a group's children
    bool entries(const Object &group, std::vector<std::pair<std::string, uint64_t>> *out, std::string *err);
    bool object_at(uint64_t addr, Object *o, std::string *err);
    // read a whole dataset as doubles (float64 / int64 / compound of float64s)
    bool read_doubles(const Dataset &ds, std::vector<double> *out, std::string *err);
    bool read_int64(const Dataset &ds, std::vector<int64_t> *out, std::string *err);
    bool attr_double(const Object &o, const std::string &name, double *v);
    bool attr_string(const Object &o, const std::string &name, std::string *v);

private:
    std::vector<uint8_t> buf_;
    uint64_t base_ = 0;
    int so_ = 8, sl_ = 8;
    uint64_t root_ohdr_ = 0;
    bool parse_object(uint64_t addr, Object *o, std::string *err);
    bool child_addr(const Object &group, const std::string &name, uint64_t *addr, std::string *err);
    bool walk_btree(uint64_t addr, uint64_t heap_data, std::vector<std::pair<std::string, uint64_t>> *out,
                    std::string *err, int depth);
    uint64_t get(uint64_t off, int n) const;
    bool inb(uint64_t off, uint64_t n) const { return off <= buf_.size() && n <= buf_.size() - off; }
};

// Writer: builds a whole file in memory.
class Writer {
public:
    Writer();
    int add_group(int parent, const std::string &name);        // returns group id (root = 0)
    void add_dataset_f64(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                         const double *data);
    void add_dataset_i64(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                         const int64_t *data);
    // complex as compound {r: f64, i: f64}
    void add_dataset_c128(int parent, const std::string &name, const std::vector<uint64_t> &dims,
                          const double *interleaved);
    void add_attr_f64(int group, const std::string &name, double v);
    // fixed-length, null-terminated ASCII string attribute
    void add_attr_str(int group, const std::string &name, const std::string &v);
    bool write(const std::string &path, std::string *err);

private:
    struct Node;
    std::vector<Node *> nodes_;
    void add_dataset(int parent, const std::string &name, const std::vector<uint64_t> &dims, int kind,
                     const void *data, size_t elem);
};

}  // namespace h5
