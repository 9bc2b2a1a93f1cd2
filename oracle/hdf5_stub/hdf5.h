/*
 * Minimal stand-in for the HDF5 C API, used ONLY to compile the unmodified
 * reference solver (pearl_serial.cpp) as a test oracle in an environment
 * without libhdf5.  It is test infrastructure, never linked into the product.
 *
 * It implements exactly the calls the reference makes (attribute, dataset,
 * dataspace, datatype, property and file handles) on top of an in-memory
 * object table.  A "file" is written on H5Fflush/H5Fclose in a small
 * self-describing container format so that the reference can also read its
 * own checkpoints back (restart) and tests can compare stored fields:
 *
 *   PEARL-H5-STUB 1\n
 *   D <name> <ny> <nx>\n<ny*nx little-endian float64>\n      (datasets)
 *   A <name> d <hex-float>\n                                  (double attrs)
 *   A <name> s <nbytes>\n<bytes>\n                            (string attrs)
 *   END\n
 */
#ifndef PEARL_HDF5_STUB_H
#define PEARL_HDF5_STUB_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include <sys/stat.h>

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

namespace pearl_h5stub {

enum Kind { K_FILE = 1, K_SPACE, K_TYPE, K_PLIST, K_ATTR, K_DSET };

struct Entry {
    char kind = 'D';               // 'D' dataset, 'd' double attr, 's' string attr
    std::string name;
    hsize_t dims[2] = {0, 0};
    std::vector<double> data;
    std::string text;
};

struct FileRec {
    std::string path;
    bool writable = false;
    std::vector<Entry> entries;
    Entry* find(const std::string& n, bool dataset) {
        for (auto& e : entries)
            if (e.name == n && ((e.kind == 'D') == dataset)) return &e;
        return nullptr;
    }
};

struct Obj {
    explicit Obj(Kind k = K_FILE) : kind(k) {}
    Kind kind;
    // dataspace
    int rank = 0;
    hsize_t dims[2] = {0, 0};
    // datatype: 0 double, >0 string of that size
    size_t str_size = 0;
    bool is_string = false;
    // attribute / dataset
    hid_t file = -1;
    std::string name;
    std::shared_ptr<FileRec> rec;
};

inline std::map<hid_t, Obj>& table() {
    static std::map<hid_t, Obj> t;
    return t;
}
inline hid_t next_id() {
    static hid_t n = 1000;
    return ++n;
}
inline hid_t add(const Obj& o) {
    hid_t id = next_id();
    table().emplace(id, o);
    return id;
}
inline Obj* get(hid_t id) {
    auto it = table().find(id);
    return it == table().end() ? nullptr : &it->second;
}
inline herr_t drop(hid_t id) {
    return table().erase(id) ? 0 : -1;
}

inline bool write_container(const FileRec& r) {
    FILE* f = std::fopen(r.path.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "PEARL-H5-STUB 1\n");
    for (const auto& e : r.entries) {
        if (e.kind == 'D') {
            std::fprintf(f, "D %s %llu %llu\n", e.name.c_str(), e.dims[0], e.dims[1]);
            std::fwrite(e.data.data(), sizeof(double), e.data.size(), f);
            std::fprintf(f, "\n");
        } else if (e.kind == 'd') {
            std::fprintf(f, "A %s d %a\n", e.name.c_str(), e.data.empty() ? 0.0 : e.data[0]);
        } else {
            std::fprintf(f, "A %s s %zu\n", e.name.c_str(), e.text.size());
            std::fwrite(e.text.data(), 1, e.text.size(), f);
            std::fprintf(f, "\n");
        }
    }
    std::fprintf(f, "END\n");
    return std::fclose(f) == 0;
}

inline bool read_container(FileRec& r) {
    FILE* f = std::fopen(r.path.c_str(), "rb");
    if (!f) return false;
    char line[4096];
    if (!std::fgets(line, sizeof line, f) || std::strncmp(line, "PEARL-H5-STUB 1", 15) != 0) {
        std::fclose(f);
        return false;
    }
    bool ok = false;
    while (std::fgets(line, sizeof line, f)) {
        if (std::strncmp(line, "END", 3) == 0) { ok = true; break; }
        char name[2048];
        Entry e;
        if (line[0] == 'D') {
            unsigned long long ny = 0, nx = 0;
            if (std::sscanf(line, "D %2047s %llu %llu", name, &ny, &nx) != 3) break;
            e.kind = 'D';
            e.name = name;
            e.dims[0] = ny;
            e.dims[1] = nx;
            e.data.resize(static_cast<size_t>(ny * nx));
            if (std::fread(e.data.data(), sizeof(double), e.data.size(), f) != e.data.size()) break;
            std::fgetc(f);
        } else if (line[0] == 'A') {
            char t = 0;
            char rest[2048];
            if (std::sscanf(line, "A %2047s %c %2047s", name, &t, rest) != 3) break;
            e.name = name;
            if (t == 'd') {
                e.kind = 'd';
                e.data.push_back(std::strtod(rest, nullptr));
            } else {
                e.kind = 's';
                size_t n = static_cast<size_t>(std::strtoull(rest, nullptr, 10));
                e.text.resize(n);
                if (n && std::fread(&e.text[0], 1, n, f) != n) break;
                std::fgetc(f);
            }
        } else {
            break;
        }
        r.entries.push_back(std::move(e));
    }
    std::fclose(f);
    return ok;
}

}  // namespace pearl_h5stub

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5S_SCALAR 0
#define H5T_NATIVE_DOUBLE ((hid_t)1)
#define H5T_IEEE_F64LE ((hid_t)2)
#define H5T_C_S1 ((hid_t)3)
#define H5P_DATASET_CREATE ((hid_t)4)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_EXCL 4u
#define H5F_SCOPE_GLOBAL 1

static inline hid_t H5Screate(int) {
    pearl_h5stub::Obj o{pearl_h5stub::K_SPACE};
    o.rank = 0;
    return pearl_h5stub::add(o);
}
static inline hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t*) {
    pearl_h5stub::Obj o{pearl_h5stub::K_SPACE};
    o.rank = rank;
    for (int i = 0; i < rank && i < 2; ++i) o.dims[i] = dims[i];
    return pearl_h5stub::add(o);
}
static inline herr_t H5Sclose(hid_t id) { return pearl_h5stub::drop(id); }
static inline int H5Sget_simple_extent_ndims(hid_t id) {
    auto* o = pearl_h5stub::get(id);
    return o ? o->rank : -1;
}
static inline int H5Sget_simple_extent_dims(hid_t id, hsize_t* dims, hsize_t*) {
    auto* o = pearl_h5stub::get(id);
    if (!o) return -1;
    for (int i = 0; i < o->rank; ++i) dims[i] = o->dims[i];
    return o->rank;
}

static inline hid_t H5Tcopy(hid_t base) {
    pearl_h5stub::Obj o{pearl_h5stub::K_TYPE};
    o.is_string = (base == H5T_C_S1);
    o.str_size = 1;
    return pearl_h5stub::add(o);
}
static inline herr_t H5Tset_size(hid_t id, size_t n) {
    auto* o = pearl_h5stub::get(id);
    if (!o) return -1;
    o->str_size = n;
    return 0;
}
static inline size_t H5Tget_size(hid_t id) {
    auto* o = pearl_h5stub::get(id);
    return o ? o->str_size : 0;
}
static inline herr_t H5Tclose(hid_t id) { return pearl_h5stub::drop(id); }

static inline hid_t H5Pcreate(hid_t) {
    pearl_h5stub::Obj o{pearl_h5stub::K_PLIST};
    return pearl_h5stub::add(o);
}
static inline herr_t H5Pset_chunk(hid_t, int, const hsize_t*) { return 0; }
static inline herr_t H5Pset_fletcher32(hid_t) { return 0; }
static inline herr_t H5Pclose(hid_t id) { return pearl_h5stub::drop(id); }

static inline hid_t H5Fcreate(const char* path, unsigned flags, hid_t, hid_t) {
    struct stat st;
    if ((flags & H5F_ACC_EXCL) && ::stat(path, &st) == 0) return -1;
    auto rec = std::make_shared<pearl_h5stub::FileRec>();
    rec->path = path;
    rec->writable = true;
    if (!pearl_h5stub::write_container(*rec)) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_FILE};
    o.rec = rec;
    return pearl_h5stub::add(o);
}
static inline hid_t H5Fopen(const char* path, unsigned, hid_t) {
    auto rec = std::make_shared<pearl_h5stub::FileRec>();
    rec->path = path;
    if (!pearl_h5stub::read_container(*rec)) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_FILE};
    o.rec = rec;
    return pearl_h5stub::add(o);
}
static inline herr_t H5Fflush(hid_t id, int) {
    auto* o = pearl_h5stub::get(id);
    if (!o || !o->rec) return -1;
    return (o->rec->writable && !pearl_h5stub::write_container(*o->rec)) ? -1 : 0;
}
static inline herr_t H5Fclose(hid_t id) {
    auto* o = pearl_h5stub::get(id);
    if (!o || !o->rec) return -1;
    herr_t s = (o->rec->writable && !pearl_h5stub::write_container(*o->rec)) ? -1 : 0;
    pearl_h5stub::drop(id);
    return s;
}

static inline hid_t H5Acreate2(hid_t file, const char* name, hid_t type, hid_t, hid_t, hid_t) {
    auto* f = pearl_h5stub::get(file);
    if (!f || !f->rec) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_ATTR};
    o.rec = f->rec;
    o.name = name;
    auto* t = pearl_h5stub::get(type);
    o.is_string = t && t->is_string;
    o.str_size = t ? t->str_size : 0;
    return pearl_h5stub::add(o);
}
static inline herr_t H5Awrite(hid_t attr, hid_t, const void* buf) {
    auto* a = pearl_h5stub::get(attr);
    if (!a || !a->rec) return -1;
    pearl_h5stub::Entry e;
    e.name = a->name;
    if (a->is_string) {
        e.kind = 's';
        const char* s = static_cast<const char*>(buf);
        e.text.assign(s, strnlen(s, a->str_size));
    } else {
        e.kind = 'd';
        e.data.push_back(*static_cast<const double*>(buf));
    }
    a->rec->entries.push_back(e);
    return 0;
}
static inline hid_t H5Aopen(hid_t file, const char* name, hid_t) {
    auto* f = pearl_h5stub::get(file);
    if (!f || !f->rec) return -1;
    auto* e = f->rec->find(name, false);
    if (!e) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_ATTR};
    o.rec = f->rec;
    o.name = name;
    o.is_string = (e->kind == 's');
    o.str_size = e->text.size() + 1;
    return pearl_h5stub::add(o);
}
static inline hid_t H5Aget_type(hid_t attr) {
    auto* a = pearl_h5stub::get(attr);
    if (!a) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_TYPE};
    o.is_string = a->is_string;
    o.str_size = a->str_size;
    return pearl_h5stub::add(o);
}
static inline herr_t H5Aread(hid_t attr, hid_t, void* buf) {
    auto* a = pearl_h5stub::get(attr);
    if (!a || !a->rec) return -1;
    auto* e = a->rec->find(a->name, false);
    if (!e) return -1;
    if (e->kind == 's') {
        std::memcpy(buf, e->text.c_str(), e->text.size() + 1);
    } else {
        *static_cast<double*>(buf) = e->data.empty() ? 0.0 : e->data[0];
    }
    return 0;
}
static inline herr_t H5Aclose(hid_t id) { return pearl_h5stub::drop(id); }

static inline hid_t H5Dcreate2(hid_t file, const char* name, hid_t, hid_t space, hid_t, hid_t, hid_t) {
    auto* f = pearl_h5stub::get(file);
    auto* s = pearl_h5stub::get(space);
    if (!f || !f->rec || !s) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_DSET};
    o.rec = f->rec;
    o.name = name;
    o.rank = s->rank;
    o.dims[0] = s->dims[0];
    o.dims[1] = s->dims[1];
    return pearl_h5stub::add(o);
}
static inline herr_t H5Dwrite(hid_t set, hid_t, hid_t, hid_t, hid_t, const void* buf) {
    auto* d = pearl_h5stub::get(set);
    if (!d || !d->rec) return -1;
    pearl_h5stub::Entry e;
    e.kind = 'D';
    e.name = d->name;
    e.dims[0] = d->dims[0];
    e.dims[1] = d->dims[1];
    const double* v = static_cast<const double*>(buf);
    e.data.assign(v, v + static_cast<size_t>(d->dims[0] * d->dims[1]));
    d->rec->entries.push_back(std::move(e));
    return 0;
}
static inline hid_t H5Dopen2(hid_t file, const char* name, hid_t) {
    auto* f = pearl_h5stub::get(file);
    if (!f || !f->rec) return -1;
    auto* e = f->rec->find(name, true);
    if (!e) return -1;
    pearl_h5stub::Obj o{pearl_h5stub::K_DSET};
    o.rec = f->rec;
    o.name = name;
    o.rank = 2;
    o.dims[0] = e->dims[0];
    o.dims[1] = e->dims[1];
    return pearl_h5stub::add(o);
}
static inline hid_t H5Dget_space(hid_t set) {
    auto* d = pearl_h5stub::get(set);
    if (!d) return -1;
    return H5Screate_simple(d->rank, d->dims, nullptr);
}
static inline herr_t H5Dread(hid_t set, hid_t, hid_t, hid_t, hid_t, void* buf) {
    auto* d = pearl_h5stub::get(set);
    if (!d || !d->rec) return -1;
    auto* e = d->rec->find(d->name, true);
    if (!e) return -1;
    std::memcpy(buf, e->data.data(), e->data.size() * sizeof(double));
    return 0;
}
static inline herr_t H5Dclose(hid_t id) { return pearl_h5stub::drop(id); }

#endif  // PEARL_HDF5_STUB_H
