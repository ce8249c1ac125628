// Mesh ingest from the reference's HDF5 mesh files (MeshHDF5Source,
// src/geometry/mesh/implementation/source/MeshHDF5Source.cpp), without an
// HDF5 library: a small read-only reader of the HDF5 file format (as the HDF
// Group's published File Format Specification describes it) covering what
// those files use:
//   superblock version 0 or 1 with 8-byte offsets and lengths; groups held
//   in symbol tables (version 1 B-tree of group nodes, symbol table nodes,
//   local heap); version 1 object headers with continuation blocks;
//   dataspace (versions 1, 2), datatype (fixed point, IEEE floating point,
//   little-endian), data layout version 3 (compact, contiguous; an
//   unallocated contiguous dataset reads as its fill value, or zero), fill
//   value (versions 1-3) and attribute (version 1) messages.
// Anything else (chunked or filtered datasets, big-endian types, newer
// object headers) returns CUPCFD_E_INVALID_FILE_FORMAT.
//
// The mesh is then what MeshHDF5Source hands to UnstructuredMeshInterface::
// addData (UnstructuredMeshInterface.ipp:1464-1862) on one rank: labels are
// 1-based (MeshHDF5Source.cpp:42-47: gidBase 1) and local ids follow label
// order; a face whose cell2 is 0 is a boundary face (:397-431, :543-580)
// with boundary label /face/bnd; geometry is read as stored (/face/lambda,
// area, n, x; /cell/x, vol); boundaries take region /bnd/rid and distance
// /bnd/distance; regions are default regions (CupCfdSoAMesh.cpp:211-221).
//
// The writer produces the same layout in the same oldest structures (superblock
// version 0, one symbol-table node per group, version 1 object headers,
// contiguous little-endian int32 / float64 datasets, int32 root attributes),
// with every dataset MeshHDF5Source reads for the mesh's connectivity and
// geometry: /cell/{nfaces, cface, x, vol}, /face/{cell1, cell2, bnd, lambda,
// area, n, x}, /bnd/{face, rid, distance} and root attributes ncel, nfac,
// nbnd, nreg, nvrt. Vertices are not part of this library's meshes: nvrt is 0
// and the vertex datasets (/vert, /face/vertices, /bnd/vertices) are absent.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <string>
#include <vector>

#include "internal.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr uint64_t UNDEF = ~0ull;

struct H5Error {
    int code;
    std::string msg;
};

[[noreturn]] void fail(const std::string &m) { throw H5Error{CUPCFD_E_INVALID_FILE_FORMAT, m}; }

struct Dataset {
    std::vector<uint64_t> dims;
    int cls = -1;         // 0 fixed point, 1 floating point
    int size = 0;         // bytes per element
    bool isSigned = false;
    bool compact = false;
    uint64_t addr = UNDEF, bytes = 0;
    std::vector<uint8_t> inline_;  // compact data or attribute data
    std::vector<uint8_t> fill;     // fill value (empty: zero)
    uint64_t count() const {
        uint64_t n = 1;
        for (uint64_t d : dims) n *= d;
        return n;
    }
};

// The file's bytes, mapped read-only (the reader touches only the
// structures and datasets it needs; nothing is copied up front).
class FileBytes {
public:
    explicit FileBytes(const std::string &path) {
        int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) throw H5Error{CUPCFD_E_FILE_MISSING, "cannot open " + path};
        struct stat sb;
        if (::fstat(fd, &sb) != 0) {
            ::close(fd);
            throw H5Error{CUPCFD_E_FILE_MISSING, "cannot read " + path};
        }
        n_ = (size_t) std::max<off_t>(sb.st_size, 0);
        if (n_ > 0) {
            void *m = ::mmap(nullptr, n_, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED) {
                ::close(fd);
                throw H5Error{CUPCFD_E_FILE_MISSING, "cannot map " + path};
            }
            p_ = static_cast<const uint8_t *>(m);
        }
        ::close(fd);
    }
    ~FileBytes() {
        if (p_) ::munmap(const_cast<uint8_t *>(p_), n_);
    }
    FileBytes(const FileBytes &) = delete;
    FileBytes &operator=(const FileBytes &) = delete;
    size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }
    const uint8_t *data() const { return p_; }
    const uint8_t *begin() const { return p_; }
    const uint8_t &operator[](size_t i) const { return p_[i]; }

private:
    const uint8_t *p_ = nullptr;
    size_t n_ = 0;
};

class H5File {
public:
    explicit H5File(const std::string &path) : d_(path) {
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        if (d_.size() < 96 || std::memcmp(d_.data(), sig, 8) != 0) fail("not an HDF5 file");
        int ver = u8(8);
        if (ver > 1) fail("superblock version " + std::to_string(ver) + " (only 0 and 1 are read)");
        if (u8(13) != 8 || u8(14) != 8) fail("offsets and lengths must be 8 bytes");
        size_t o = 24 + (ver == 1 ? 4 : 0);  // group K values, flags [, indexed-storage K + reserved]
        base_ = u64(o);
        rootEntry_ = o + 32;                  // after base, free-space, end-of-file, driver addresses
        root_ = u64(rootEntry_ + 8) + base_;
    }

    // Dataset (or group when isGroup) at an absolute path such as "/face/n".
    uint64_t lookup(const std::string &path) const {
        uint64_t oh = root_;
        size_t p = 1;
        while (p < path.size()) {
            size_t q = path.find('/', p);
            std::string name = path.substr(p, q == std::string::npos ? std::string::npos : q - p);
            uint64_t bt, heap;
            if (!symbol_table(oh, bt, heap)) fail("'" + name + "': parent is not a group");
            oh = find_in_group(bt, heap, name);
            if (oh == UNDEF) fail("no object '" + path + "'");
            p = q == std::string::npos ? path.size() : q + 1;
        }
        return oh;
    }

    Dataset dataset(const std::string &path) const {
        Dataset ds;
        bool haveSpace = false, haveType = false, haveLayout = false;
        for (const Msg &m : messages(lookup(path))) {
            if (m.type == 0x01) { parse_space(m.off, ds); haveSpace = true; }
            else if (m.type == 0x03) { parse_type(m.off, ds); haveType = true; }
            else if (m.type == 0x05 || m.type == 0x04) parse_fill(m, ds);
            else if (m.type == 0x08) { parse_layout(m.off, ds); haveLayout = true; }
            else if (m.type == 0x0B) fail(path + ": filtered datasets are not read");
        }
        if (!haveSpace || !haveType || !haveLayout) fail(path + " is not a dataset");
        return ds;
    }

    // Attribute `name` of the root group.
    Dataset root_attribute(const std::string &name) const {
        for (const Msg &m : messages(root_)) {
            if (m.type != 0x0C) continue;
            size_t o = m.off;
            if (u8(o) != 1) fail("attribute message version " + std::to_string(u8(o)));
            uint16_t nl = u16(o + 2), tl = u16(o + 4), sl = u16(o + 6);
            o += 8;
            std::string an(reinterpret_cast<const char *>(&d_[o]), strnlen(reinterpret_cast<const char *>(&d_[o]), nl));
            o += pad8(nl);
            if (an != name) continue;
            Dataset ds;
            parse_type(o, ds);
            o += pad8(tl);
            parse_space(o, ds);
            o += pad8(sl);
            uint64_t bytes = ds.count() * ds.size;
            need(o, bytes);
            ds.compact = true;
            ds.inline_.assign(d_.begin() + o, d_.begin() + o + bytes);
            return ds;
        }
        fail("no root attribute '" + name + "'");
    }

    // Element values as doubles / int64.
    std::vector<double> real(const Dataset &ds) const {
        std::vector<double> out(ds.count());
        const uint8_t *p = raw(ds);
        if (p && ds.cls == 1 && ds.size == 8) {  // little-endian float64, as stored: one copy
            if (!out.empty()) std::memcpy(out.data(), p, out.size() * 8);
            return out;
        }
        for (size_t i = 0; i < out.size(); i++) out[i] = value_real(ds, p ? p + i * ds.size : nullptr);
        return out;
    }
    std::vector<int64_t> integer(const Dataset &ds) const {
        if (ds.cls != 0) fail("integer dataset expected");
        std::vector<int64_t> out(ds.count());
        const uint8_t *p = raw(ds);
        if (p && ds.size == 4 && ds.isSigned) {  // little-endian int32
            for (size_t i = 0; i < out.size(); i++) {
                int32_t v;
                std::memcpy(&v, p + 4 * i, 4);
                out[i] = v;
            }
            return out;
        }
        for (size_t i = 0; i < out.size(); i++) out[i] = value_int(ds, p ? p + i * ds.size : nullptr);
        return out;
    }

private:
    struct Msg {
        int type;
        size_t off, size;
    };
    FileBytes d_;
    uint64_t base_ = 0, root_ = 0;
    size_t rootEntry_ = 0;

    static size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }
    void need(uint64_t o, uint64_t n) const {
        if (o > d_.size() || n > d_.size() - o) fail("structure past the end of the file");
    }
    uint8_t u8(uint64_t o) const { need(o, 1); return d_[o]; }
    uint16_t u16(uint64_t o) const { need(o, 2); uint16_t v; std::memcpy(&v, &d_[o], 2); return v; }
    uint32_t u32(uint64_t o) const { need(o, 4); uint32_t v; std::memcpy(&v, &d_[o], 4); return v; }
    uint64_t u64(uint64_t o) const { need(o, 8); uint64_t v; std::memcpy(&v, &d_[o], 8); return v; }
    bool sig(uint64_t o, const char *s) const { need(o, 4); return std::memcmp(&d_[o], s, 4) == 0; }

    std::vector<Msg> messages(uint64_t oh) const {
        if (u8(oh) != 1) fail("object header version " + std::to_string(u8(oh)) + " (only 1 is read)");
        uint16_t n = u16(oh + 2);
        std::vector<std::pair<uint64_t, uint64_t>> blocks{{oh + 16, u32(oh + 8)}};
        std::vector<Msg> out;
        for (size_t b = 0; b < blocks.size() && out.size() < n; b++) {
            uint64_t o = blocks[b].first, end = o + blocks[b].second;
            need(blocks[b].first, blocks[b].second);
            while (o + 8 <= end && out.size() < n) {
                int t = u16(o);
                size_t s = u16(o + 2);
                need(o + 8, s);
                if (t == 0x10) blocks.push_back({u64(o + 8) + base_, u64(o + 16)});
                out.push_back({t, (size_t) o + 8, s});
                o += 8 + s;
            }
            if (blocks.size() > 64) fail("too many header continuation blocks");
        }
        return out;
    }

    bool symbol_table(uint64_t oh, uint64_t &bt, uint64_t &heap) const {
        if (oh == root_) {  // the root's symbol table entry caches it (cache type 1)
            if (u32(rootEntry_ + 16) == 1) {
                bt = u64(rootEntry_ + 24) + base_;
                heap = u64(rootEntry_ + 32) + base_;
                return true;
            }
        }
        for (const Msg &m : messages(oh))
            if (m.type == 0x11) {
                bt = u64(m.off) + base_;
                heap = u64(m.off + 8) + base_;
                return true;
            }
        return false;
    }

    std::string heap_name(uint64_t heap, uint64_t off) const {
        if (!sig(heap, "HEAP")) fail("local heap signature");
        uint64_t size = u64(heap + 8), data = u64(heap + 24) + base_;
        if (off >= size) fail("name offset past the heap");
        need(data, size);
        const char *s = reinterpret_cast<const char *>(&d_[data + off]);
        return std::string(s, strnlen(s, size - off));
    }

    uint64_t find_in_group(uint64_t node, uint64_t heap, const std::string &name, int depth = 0) const {
        if (depth > 32) fail("group B-tree too deep");
        if (!sig(node, "TREE") || u8(node + 4) != 0) fail("group B-tree node");
        int level = u8(node + 5), n = u16(node + 6);
        uint64_t o = node + 24;  // signature, type, level, entries, left / right siblings
        for (int i = 0; i < n; i++) {
            uint64_t child = u64(o + 8 + 16 * i) + base_;
            if (level > 0) {
                uint64_t r = find_in_group(child, heap, name, depth + 1);
                if (r != UNDEF) return r;
                continue;
            }
            if (!sig(child, "SNOD")) fail("symbol table node");
            int ns = u16(child + 6);
            for (int j = 0; j < ns; j++) {
                uint64_t e = child + 8 + 40 * (uint64_t) j;
                if (heap_name(heap, u64(e)) == name) return u64(e + 8) + base_;
            }
        }
        return UNDEF;
    }

    void parse_space(size_t o, Dataset &ds) const {
        int ver = u8(o), rank = u8(o + 1);
        size_t dimOff;
        if (ver == 1) dimOff = o + 8;
        else if (ver == 2) {
            if (u8(o + 3) == 2) rank = 0;  // null dataspace
            dimOff = o + 4;
        } else fail("dataspace version " + std::to_string(ver));
        ds.dims.assign(rank, 0);
        for (int i = 0; i < rank; i++) ds.dims[i] = u64(dimOff + 8 * i);
    }

    void parse_type(size_t o, Dataset &ds) const {
        int cls = u8(o) & 15;
        uint8_t bits0 = u8(o + 1);
        ds.size = (int) u32(o + 4);
        if (cls != 0 && cls != 1) fail("datatype class " + std::to_string(cls) + " (only fixed and floating point)");
        if (bits0 & 1) fail("big-endian data are not read");
        if (cls == 0 && ds.size != 1 && ds.size != 2 && ds.size != 4 && ds.size != 8) fail("integer size");
        if (cls == 1 && ds.size != 4 && ds.size != 8) fail("floating-point size");
        ds.cls = cls;
        ds.isSigned = cls == 0 && (bits0 & 8);
    }

    void parse_fill(const Msg &m, Dataset &ds) const {
        size_t o = m.off;
        if (m.type == 0x04) {  // old fill value message: size, value
            uint32_t s = u32(o);
            if (s) ds.fill.assign(d_.begin() + o + 4, d_.begin() + o + 4 + s);
            return;
        }
        int ver = u8(o);
        if (ver == 1 || ver == 2) {
            bool defined = u8(o + 3) != 0;
            if (defined) {
                uint32_t s = u32(o + 4);
                need(o + 8, s);
                if (s) ds.fill.assign(d_.begin() + o + 8, d_.begin() + o + 8 + s);
            }
        } else if (ver == 3) {
            uint8_t flags = u8(o + 1);
            if (flags & 0x20) {
                uint32_t s = u32(o + 2);
                need(o + 6, s);
                if (s) ds.fill.assign(d_.begin() + o + 6, d_.begin() + o + 6 + s);
            }
        } else fail("fill value version " + std::to_string(ver));
    }

    void parse_layout(size_t o, Dataset &ds) const {
        if (u8(o) != 3) fail("data layout version " + std::to_string(u8(o)) + " (only 3 is read)");
        int cls = u8(o + 1);
        if (cls == 0) {
            uint16_t s = u16(o + 2);
            need(o + 4, s);
            ds.compact = true;
            ds.inline_.assign(d_.begin() + o + 4, d_.begin() + o + 4 + s);
        } else if (cls == 1) {
            uint64_t a = u64(o + 2);
            ds.addr = a == UNDEF ? UNDEF : a + base_;
            ds.bytes = u64(o + 10);
        } else fail("chunked datasets are not read");
    }

    // Raw element bytes, or null when every element is the fill value.
    const uint8_t *raw(const Dataset &ds) const {
        uint64_t bytes = ds.count() * ds.size;
        if (ds.compact) {
            if (ds.inline_.size() < bytes) fail("compact data shorter than its dataspace");
            return ds.inline_.data();
        }
        if (ds.addr == UNDEF) return nullptr;
        if (ds.bytes < bytes) fail("contiguous data shorter than its dataspace");
        need(ds.addr, bytes);
        return &d_[ds.addr];
    }

    const uint8_t *fill_or_null(const Dataset &ds) const {
        if (ds.fill.empty()) return nullptr;
        if ((int) ds.fill.size() != ds.size) fail("fill value size");
        return ds.fill.data();
    }

    double value_real(const Dataset &ds, const uint8_t *p) const {
        if (!p) p = fill_or_null(ds);
        if (!p) return 0.0;
        if (ds.cls == 0) return (double) value_int(ds, p);
        if (ds.size == 4) { float v; std::memcpy(&v, p, 4); return (double) v; }
        double v;
        std::memcpy(&v, p, 8);
        return v;
    }
    int64_t value_int(const Dataset &ds, const uint8_t *p) const {
        if (!p) p = fill_or_null(ds);
        if (!p) return 0;
        uint64_t u = 0;
        std::memcpy(&u, p, ds.size);
        if (ds.isSigned && ds.size < 8 && (u >> (8 * ds.size - 1)) & 1) u |= ~0ull << (8 * ds.size);
        return (int64_t) u;
    }
};

struct HostMesh {
    int nC = 0, nF = 0, nB = 0, nR = 0;
    std::vector<int32_t> c1, c2, bnd, bndRegion;
    std::vector<double> lam, area, S, X, cc, vol, dist;
};

int64_t attr_int(const H5File &h, const char *name) {
    Dataset a = h.root_attribute(name);
    if (a.count() != 1) fail(std::string("root attribute '") + name + "' is not a scalar");
    return h.integer(a)[0];
}

std::vector<double> vec3(const H5File &h, const char *path, int n) {
    Dataset ds = h.dataset(path);
    if (ds.dims.size() != 2 || ds.dims[0] != (uint64_t) n || ds.dims[1] != 3)
        throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, std::string(path) + " is not [n][3]"};
    return h.real(ds);
}

std::vector<double> reals(const H5File &h, const char *path, int n) {
    Dataset ds = h.dataset(path);
    if (ds.count() != (uint64_t) n) throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, std::string(path) + " has the wrong length"};
    return h.real(ds);
}

std::vector<int64_t> ints(const H5File &h, const char *path, int n) {
    Dataset ds = h.dataset(path);
    if (ds.count() != (uint64_t) n) throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, std::string(path) + " has the wrong length"};
    return h.integer(ds);
}

// MeshHDF5Source's view of the file (see the file comment).
HostMesh read_mesh(const std::string &path) {
    H5File h(path);
    HostMesh m;
    int64_t nC = attr_int(h, "ncel"), nF = attr_int(h, "nfac"), nB = attr_int(h, "nbnd"), nR = attr_int(h, "nreg");
    if (nC < 1 || nF < 1 || nB < 0 || nR < 0 || nC > INT32_MAX || nF > INT32_MAX || nB > INT32_MAX || nR > INT32_MAX)
        fail("counts out of range");
    m.nC = (int) nC; m.nF = (int) nF; m.nB = (int) nB; m.nR = (int) nR;
    auto c1 = ints(h, "/face/cell1", m.nF), c2 = ints(h, "/face/cell2", m.nF), fb = ints(h, "/face/bnd", m.nF);
    m.c1.resize(m.nF); m.c2.resize(m.nF); m.bnd.resize(m.nF);
    for (int f = 0; f < m.nF; f++) {
        if (c1[f] < 1 || c1[f] > nC || c2[f] < 0 || c2[f] > nC)
            throw H5Error{CUPCFD_E_INVALID_INDEX, "a face's cell label is out of range"};
        m.c1[f] = (int32_t) (c1[f] - 1);
        m.c2[f] = c2[f] == 0 ? -1 : (int32_t) (c2[f] - 1);
        if (c2[f] == 0) {
            if (fb[f] < 1 || fb[f] > nB) throw H5Error{CUPCFD_E_INVALID_INDEX, "a boundary face's boundary label is out of range"};
            m.bnd[f] = (int32_t) (fb[f] - 1);
        } else {
            m.bnd[f] = -1;
        }
    }
    m.lam = reals(h, "/face/lambda", m.nF);
    m.area = reals(h, "/face/area", m.nF);
    m.S = vec3(h, "/face/n", m.nF);
    m.X = vec3(h, "/face/x", m.nF);
    m.cc = vec3(h, "/cell/x", m.nC);
    m.vol = reals(h, "/cell/vol", m.nC);
    m.bndRegion.assign(m.nB, 0);
    m.dist.assign(m.nB, 0.0);
    if (m.nB > 0) {
        auto rid = ints(h, "/bnd/rid", m.nB);
        for (int b = 0; b < m.nB; b++) {
            if (rid[b] < 1 || rid[b] > std::max<int64_t>(nR, 1))
                throw H5Error{CUPCFD_E_INVALID_INDEX, "a boundary's region label is out of range"};
            m.bndRegion[b] = (int32_t) (rid[b] - 1);
        }
        m.dist = reals(h, "/bnd/distance", m.nB);
    }
    return m;
}

// ---------------------------------------------------------------------------
// Writer (the structures of the file comment; field layouts as the HDF
// Group's File Format Specification gives them for these versions)
// ---------------------------------------------------------------------------
class H5Writer {
public:
    H5Writer() : b_(96, 0) {}  // superblock + root symbol-table entry, filled in by finish()
    void reserve(size_t bytes) { b_.reserve(bytes); }

    uint64_t dataset_i32(const int32_t *v, std::initializer_list<uint64_t> dims) {
        return dataset(v, dims, 4, type_i32());
    }
    uint64_t dataset_f64(const double *v, std::initializer_list<uint64_t> dims) {
        return dataset(v, dims, 8, type_f64());
    }

    // A group of named objects (at most 2K = 8, one symbol-table node) with
    // optional scalar int32 attributes; returns its object header address.
    uint64_t group(std::vector<std::pair<std::string, uint64_t>> ents,
                   const std::vector<std::pair<std::string, int32_t>> &attrs = {}) {
        std::sort(ents.begin(), ents.end());
        if (ents.size() > 2 * LEAF_K) throw H5Error{CUPCFD_E_ERROR, "group too large for one symbol-table node"};
        std::vector<uint8_t> heap(8, 0);  // offset 0: the empty name
        std::vector<uint64_t> off;
        for (auto &e : ents) {
            off.push_back(heap.size());
            heap.insert(heap.end(), e.first.begin(), e.first.end());
            heap.push_back(0);
            heap.resize(pad8(heap.size()), 0);
        }
        uint64_t heapData = alloc(heap);
        std::vector<uint8_t> hp;
        put_bytes(hp, "HEAP", 4); put_n(hp, 0, 4);
        put_n(hp, heap.size(), 8); put_n(hp, UNDEF, 8); put_n(hp, heapData, 8);
        uint64_t heapAddr = alloc(hp);
        std::vector<uint8_t> sn;
        put_bytes(sn, "SNOD", 4); put_n(sn, 1, 1); put_n(sn, 0, 1); put_n(sn, ents.size(), 2);
        for (size_t i = 0; i < ents.size(); i++) {
            put_n(sn, off[i], 8); put_n(sn, ents[i].second, 8); put_n(sn, 0, 4); put_n(sn, 0, 4);
            sn.resize(sn.size() + 16, 0);
        }
        sn.resize(8 + 40 * 2 * LEAF_K, 0);
        uint64_t snod = alloc(sn);
        std::vector<uint8_t> tr;
        put_bytes(tr, "TREE", 4); put_n(tr, 0, 1); put_n(tr, 0, 1); put_n(tr, 1, 2);
        put_n(tr, UNDEF, 8); put_n(tr, UNDEF, 8);
        put_n(tr, 0, 8); put_n(tr, snod, 8); put_n(tr, ents.empty() ? 0 : off.back(), 8);
        tr.resize(24 + 8 * (2 * NODE_K + 1) + 8 * 2 * NODE_K, 0);
        uint64_t tree = alloc(tr);
        std::vector<std::vector<uint8_t>> msgs;
        std::vector<uint8_t> stab;
        put_n(stab, tree, 8); put_n(stab, heapAddr, 8);
        msgs.push_back(message(0x11, stab));
        for (auto &a : attrs) {
            std::vector<uint8_t> nm(a.first.begin(), a.first.end());
            nm.push_back(0);
            std::vector<uint8_t> dt = type_i32(), sp = space({1}), body;
            put_n(body, 1, 1); put_n(body, 0, 1); put_n(body, nm.size(), 2); put_n(body, dt.size(), 2);
            put_n(body, sp.size(), 2);
            append_padded(body, nm); append_padded(body, dt); append_padded(body, sp);
            put_n(body, (uint32_t) a.second, 4);
            msgs.push_back(message(0x0C, body));
        }
        rootTree_ = tree;
        rootHeap_ = heapAddr;
        return object_header(msgs);
    }

    // Fills in the superblock with `root` (the last group() call's header)
    // as the root group and writes the file.
    void write(uint64_t root, const std::string &path) {
        std::vector<uint8_t> sb;
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        sb.insert(sb.end(), sig, sig + 8);
        const uint8_t vers[8] = {0, 0, 0, 0, 0, 8, 8, 0};  // superblock, free space, root table, -, shared header, offsets, lengths, -
        sb.insert(sb.end(), vers, vers + 8);
        put_n(sb, LEAF_K, 2); put_n(sb, NODE_K, 2); put_n(sb, 0, 4);
        put_n(sb, 0, 8); put_n(sb, UNDEF, 8); put_n(sb, b_.size(), 8); put_n(sb, UNDEF, 8);
        put_n(sb, 0, 8); put_n(sb, root, 8); put_n(sb, 1, 4); put_n(sb, 0, 4);  // root entry: cache type 1
        put_n(sb, rootTree_, 8); put_n(sb, rootHeap_, 8);
        std::memcpy(b_.data(), sb.data(), 96);
        FILE *f = std::fopen(path.c_str(), "wb");
        if (!f) throw H5Error{CUPCFD_E_FILE_MISSING, "cannot open " + path + " for writing"};
        bool ok = std::fwrite(b_.data(), 1, b_.size(), f) == b_.size();
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) throw H5Error{CUPCFD_E_ERROR, "writing " + path + " failed"};
    }

private:
    static constexpr int LEAF_K = 4, NODE_K = 16;
    std::vector<uint8_t> b_;
    uint64_t rootTree_ = UNDEF, rootHeap_ = UNDEF;

    static size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }
    static void put_n(std::vector<uint8_t> &v, uint64_t x, int n) {
        for (int i = 0; i < n; i++) v.push_back((uint8_t) (x >> (8 * i)));
    }
    static void put_bytes(std::vector<uint8_t> &v, const char *p, int n) { v.insert(v.end(), p, p + n); }
    static void append_padded(std::vector<uint8_t> &v, const std::vector<uint8_t> &a) {
        v.insert(v.end(), a.begin(), a.end());
        v.resize(v.size() + (pad8(a.size()) - a.size()), 0);
    }
    uint64_t alloc(const void *p, size_t n) {
        uint64_t a = b_.size();
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b_.insert(b_.end(), q, q + n);
        b_.resize(pad8(b_.size()), 0);
        return a;
    }
    uint64_t alloc(const std::vector<uint8_t> &v) { return alloc(v.data(), v.size()); }
    static std::vector<uint8_t> message(int type, std::vector<uint8_t> body) {
        body.resize(pad8(body.size()), 0);
        std::vector<uint8_t> m;
        put_n(m, type, 2); put_n(m, body.size(), 2); put_n(m, 0, 4);  // type, size, flags, reserved
        m.insert(m.end(), body.begin(), body.end());
        return m;
    }
    uint64_t object_header(const std::vector<std::vector<uint8_t>> &msgs) {
        std::vector<uint8_t> h;
        size_t body = 0;
        for (auto &m : msgs) body += m.size();
        put_n(h, 1, 1); put_n(h, 0, 1); put_n(h, msgs.size(), 2); put_n(h, 1, 4); put_n(h, body, 4); put_n(h, 0, 4);
        for (auto &m : msgs) h.insert(h.end(), m.begin(), m.end());
        return alloc(h);
    }
    static std::vector<uint8_t> space(std::initializer_list<uint64_t> dims) {
        std::vector<uint8_t> v;
        put_n(v, 1, 1); put_n(v, dims.size(), 1); put_n(v, 0, 2); put_n(v, 0, 4);
        for (uint64_t d : dims) put_n(v, d, 8);
        return v;
    }
    static std::vector<uint8_t> type_i32() {  // class 0 (fixed point), version 1, signed, little-endian
        std::vector<uint8_t> v = {0x10, 0x08, 0, 0};
        put_n(v, 4, 4); put_n(v, 0, 2); put_n(v, 32, 2);
        return v;
    }
    static std::vector<uint8_t> type_f64() {  // class 1 (IEEE), version 1, little-endian, sign at bit 63
        std::vector<uint8_t> v = {0x11, 0x20, 63, 0};
        put_n(v, 8, 4);
        put_n(v, 0, 2); put_n(v, 64, 2); put_n(v, 52, 1); put_n(v, 11, 1); put_n(v, 0, 1); put_n(v, 52, 1);
        put_n(v, 1023, 4);
        return v;
    }
    uint64_t dataset(const void *v, std::initializer_list<uint64_t> dims, int es, const std::vector<uint8_t> &dt) {
        uint64_t n = 1;
        for (uint64_t d : dims) n *= d;
        uint64_t data = alloc(v, (size_t) (n * es));  // the host is little-endian, as the datatypes state
        std::vector<uint8_t> layout = {3, 1};          // version 3, contiguous
        put_n(layout, data, 8); put_n(layout, n * es, 8);
        return object_header({message(0x01, space(dims)), message(0x03, dt), message(0x08, layout)});
    }
};

// The datasets of a mesh in MeshHDF5Source's layout (0-based arrays in;
// labels written 1-based), checked for consistency first.
void write_mesh(const std::string &path, int nC, int nF, int nB, int nR, const int32_t *c1, const int32_t *c2,
                const int32_t *fb, const double *lam, const double *area, const double *S, const double *X,
                const double *cc, const double *vol, const int32_t *breg, const double *bdist) {
    if (nC < 1 || nF < 1 || nB < 0 || nR < 1) throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, "counts out of range"};
    std::vector<int32_t> l1(nF), l2(nF), lb(nF), nfaces(nC, 0), bface(nB, 0), rid(nB, 1);
    for (int f = 0; f < nF; f++) {
        if (c1[f] < 0 || c1[f] >= nC || c2[f] < -1 || c2[f] >= nC)
            throw H5Error{CUPCFD_E_INVALID_INDEX, "a face's cell id is out of range"};
        l1[f] = c1[f] + 1;
        l2[f] = c2[f] + 1;  // 0 on a boundary face
        nfaces[c1[f]]++;
        if (c2[f] >= 0) {
            nfaces[c2[f]]++;
            lb[f] = 0;
        } else {
            if (fb[f] < 0 || fb[f] >= nB || bface[fb[f]] != 0)
                throw H5Error{CUPCFD_E_INVALID_INDEX, "boundary ids are not one per boundary face"};
            bface[fb[f]] = f + 1;
            lb[f] = fb[f] + 1;
        }
    }
    for (int b = 0; b < nB; b++) {
        if (bface[b] == 0) throw H5Error{CUPCFD_E_INVALID_INDEX, "a boundary id has no face"};
        if (breg) {
            if (breg[b] < 0 || breg[b] >= nR) throw H5Error{CUPCFD_E_INVALID_INDEX, "a boundary's region is out of range"};
            rid[b] = breg[b] + 1;
        }
    }
    // /cell/cface: each cell's faces, ascending face label, padded with 0
    const int maxF = *std::max_element(nfaces.begin(), nfaces.end());
    std::vector<int32_t> cface((size_t) nC * maxF, 0), fill(nC, 0);
    for (int f = 0; f < nF; f++) {
        cface[(size_t) c1[f] * maxF + fill[c1[f]]++] = f + 1;
        if (c2[f] >= 0) cface[(size_t) c2[f] * maxF + fill[c2[f]]++] = f + 1;
    }
    std::vector<double> dist(nB, 0.0);
    if (bdist) std::copy(bdist, bdist + nB, dist.begin());
    H5Writer w;
    w.reserve((size_t) nF * (3 * 4 + 8 * 8) + (size_t) nC * (4 + 4 * (size_t) maxF + 4 * 8) + (size_t) nB * 16 +
              (1u << 20));
    const uint64_t C = (uint64_t) nC, F = (uint64_t) nF, B = (uint64_t) nB;
    uint64_t cell = w.group({{"nfaces", w.dataset_i32(nfaces.data(), {C})},
                             {"cface", w.dataset_i32(cface.data(), {C, (uint64_t) maxF})},
                             {"x", w.dataset_f64(cc, {C, 3})},
                             {"vol", w.dataset_f64(vol, {C})}});
    uint64_t face = w.group({{"cell1", w.dataset_i32(l1.data(), {F})}, {"cell2", w.dataset_i32(l2.data(), {F})},
                             {"bnd", w.dataset_i32(lb.data(), {F})}, {"lambda", w.dataset_f64(lam, {F})},
                             {"area", w.dataset_f64(area, {F})}, {"n", w.dataset_f64(S, {F, 3})},
                             {"x", w.dataset_f64(X, {F, 3})}});
    uint64_t bnd = w.group({{"face", w.dataset_i32(bface.data(), {B})}, {"rid", w.dataset_i32(rid.data(), {B})},
                            {"distance", w.dataset_f64(dist.data(), {B})}});
    uint64_t root = w.group({{"cell", cell}, {"face", face}, {"bnd", bnd}},
                            {{"ncel", nC}, {"nfac", nF}, {"nbnd", nB}, {"nreg", nR}, {"nvrt", 0}});
    w.write(root, path);
}

template <class F>
int guarded(const char *what, F &&f) {
    try {
        return f();
    } catch (const H5Error &e) {
        set_error(std::string(what) + ": " + e.msg);
        return e.code;
    } catch (const std::exception &e) {
        set_error(std::string(what) + ": " + e.what());
        return CUPCFD_E_ERROR;
    }
}

}  // namespace

extern "C" int cupcfd_gpu_hdf5_mesh_counts(const char *path, int32_t *nCells, int32_t *nFaces, int32_t *nBoundaries,
                                           int32_t *nRegions) {
    clear_error();
    CG_RETURN_IF(!path || !nCells || !nFaces || !nBoundaries || !nRegions, CUPCFD_E_NULL_PTR, "hdf5_mesh_counts: null argument");
    return guarded("hdf5_mesh_counts", [&] {
        H5File h(path);
        *nCells = (int32_t) attr_int(h, "ncel");
        *nFaces = (int32_t) attr_int(h, "nfac");
        *nBoundaries = (int32_t) attr_int(h, "nbnd");
        *nRegions = (int32_t) attr_int(h, "nreg");
        return CUPCFD_E_SUCCESS;
    });
}

extern "C" int cupcfd_gpu_hdf5_mesh_read(const char *path, int32_t nCells, int32_t nFaces, int32_t nBoundaries,
                                         int32_t *faceCell1, int32_t *faceCell2, int32_t *faceBnd, double *faceLambda,
                                         double *faceArea, double *faceNorm, double *faceCenter, double *cellCenter,
                                         double *cellVolume, int32_t *bndRegion, double *bndDistance) {
    clear_error();
    CG_RETURN_IF(!path, CUPCFD_E_NULL_PTR, "hdf5_mesh_read: null path");
    return guarded("hdf5_mesh_read", [&] {
        HostMesh m = read_mesh(path);
        if (m.nC != nCells || m.nF != nFaces || m.nB != nBoundaries)
            throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, "counts differ from the file's"};
        auto put = [](auto *dst, const auto &src) {
            if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
        };
        put(faceCell1, m.c1); put(faceCell2, m.c2); put(faceBnd, m.bnd);
        put(faceLambda, m.lam); put(faceArea, m.area); put(faceNorm, m.S); put(faceCenter, m.X);
        put(cellCenter, m.cc); put(cellVolume, m.vol); put(bndRegion, m.bndRegion); put(bndDistance, m.dist);
        return CUPCFD_E_SUCCESS;
    });
}

extern "C" int cupcfd_gpu_mesh_load_hdf5(const char *path, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    clear_error();
    CG_RETURN_IF(!path || !out, CUPCFD_E_NULL_PTR, "mesh_load_hdf5: null argument");
    *out = nullptr;
    HostMesh m;
    int rc = guarded("mesh_load_hdf5", [&] {
        m = read_mesh(path);
        return CUPCFD_E_SUCCESS;
    });
    if (rc != CUPCFD_E_SUCCESS) return rc;
    cupcfd_mesh_view v;
    std::memset(&v, 0, sizeof(v));
    v.nCells = m.nC; v.nFaces = m.nF; v.nBoundaries = m.nB; v.real_size = sizeof(double);
    v.faceCell1 = m.c1.data(); v.faceCell2 = m.c2.data(); v.faceBnd = m.bnd.data();
    v.faceLambda = m.lam.data(); v.faceArea = m.area.data(); v.cellVolume = m.vol.data();
    v.faceNorm = {m.S.data(), (int32_t) (3 * sizeof(double)), 0};
    v.faceCenter = {m.X.data(), (int32_t) (3 * sizeof(double)), 0};
    v.cellCenter = {m.cc.data(), (int32_t) (3 * sizeof(double)), 0};
    cupcfd_gpu_mesh *g = nullptr;
    CG_TRY(cupcfd_gpu_mesh_create(&v, opt, &g));
    // default regions (every region the file names), boundaries' regions and distances
    const int nR = std::max(m.nR, 1);
    std::vector<int32_t> rtype(nR, CUPCFD_RTYPE_DEFAULT);
    std::vector<double> ruvw(3 * (size_t) nR, 0.0), rden(nR, 0.0);
    rc = cupcfd_gpu_mesh_set_regions(g, nR, rtype.data(), ruvw.data(), rden.data(), m.bndRegion.data(), m.nB);
    if (rc == CUPCFD_E_SUCCESS && m.nB > 0) rc = cupcfd_gpu_mesh_set_boundary_distance(g, m.dist.data(), m.nB);
    if (rc != CUPCFD_E_SUCCESS) {
        std::string msg = cupcfd_gpu_last_error();
        cupcfd_gpu_mesh_destroy(g);
        set_error("mesh_load_hdf5: " + msg);
        return rc;
    }
    *out = g;
    return CUPCFD_E_SUCCESS;
}

extern "C" int cupcfd_gpu_hdf5_mesh_write(const char *path, int32_t nCells, int32_t nFaces, int32_t nBoundaries,
                                          int32_t nRegions, const int32_t *faceCell1, const int32_t *faceCell2,
                                          const int32_t *faceBnd, const double *faceLambda, const double *faceArea,
                                          const double *faceNorm, const double *faceCenter, const double *cellCenter,
                                          const double *cellVolume, const int32_t *bndRegion,
                                          const double *bndDistance) {
    clear_error();
    CG_RETURN_IF(!path || !faceCell1 || !faceCell2 || !faceBnd || !faceLambda || !faceArea || !faceNorm ||
                     !faceCenter || !cellCenter || !cellVolume,
                 CUPCFD_E_NULL_PTR, "hdf5_mesh_write: null argument");
    return guarded("hdf5_mesh_write", [&] {
        write_mesh(path, nCells, nFaces, nBoundaries, nRegions, faceCell1, faceCell2, faceBnd, faceLambda, faceArea,
                   faceNorm, faceCenter, cellCenter, cellVolume, bndRegion, bndDistance);
        return CUPCFD_E_SUCCESS;
    });
}

extern "C" int cupcfd_gpu_mesh_save_hdf5(const cupcfd_gpu_mesh *m, const char *path) {
    clear_error();
    CG_RETURN_IF(!m || !path, CUPCFD_E_NULL_PTR, "mesh_save_hdf5: null argument");
    CG_TRY(make_device_current(m->device));
    const int nC = m->nC, nF = m->nF, nB = m->nB;
    std::vector<int32_t> c1(nF), c2(nF), bnd(nF), breg(nB, 0);
    std::vector<double> lam(nF), area(nF), S(3 * (size_t) nF), X(3 * (size_t) nF), cc(3 * (size_t) nC), vol(nC),
        dist(nB, 0.0);
    CG_TRY(cupcfd_gpu_mesh_get_geometry(m, c1.data(), c2.data(), bnd.data(), lam.data(), area.data(), S.data(),
                                        X.data(), cc.data(), vol.data()));
    CG_CHECK_CUDA(cudaStreamSynchronize(m->stream));
    if (nB > 0 && m->bndRegion)
        CG_CHECK_CUDA(cudaMemcpy(breg.data(), m->bndRegion, sizeof(int32_t) * nB, cudaMemcpyDeviceToHost));
    if (nB > 0 && m->bndDist)
        CG_CHECK_CUDA(cudaMemcpy(dist.data(), m->bndDist, sizeof(double) * nB, cudaMemcpyDeviceToHost));
    return guarded("mesh_save_hdf5", [&] {
        write_mesh(path, nC, nF, nB, std::max(m->nR, 1), c1.data(), c2.data(), bnd.data(), lam.data(), area.data(),
                   S.data(), X.data(), cc.data(), vol.data(), breg.data(), dist.data());
        return CUPCFD_E_SUCCESS;
    });
}

extern "C" int cupcfd_gpu_hdf5_dataset_shape(const char *path, const char *name, int32_t *ndims, int64_t *dims,
                                             int32_t *isReal) {
    clear_error();
    CG_RETURN_IF(!path || !name || !ndims || !dims || !isReal, CUPCFD_E_NULL_PTR, "hdf5_dataset_shape: null argument");
    return guarded("hdf5_dataset_shape", [&] {
        H5File h(path);
        Dataset ds = h.dataset(name);
        if (ds.dims.size() > 4) fail(std::string(name) + " has more than 4 dimensions");
        *ndims = (int32_t) ds.dims.size();
        for (size_t i = 0; i < ds.dims.size(); i++) dims[i] = (int64_t) ds.dims[i];
        *isReal = ds.cls == 1;
        return CUPCFD_E_SUCCESS;
    });
}

extern "C" int cupcfd_gpu_hdf5_dataset_read(const char *path, const char *name, double *out, int64_t n) {
    clear_error();
    CG_RETURN_IF(!path || !name || !out, CUPCFD_E_NULL_PTR, "hdf5_dataset_read: null argument");
    return guarded("hdf5_dataset_read", [&] {
        H5File h(path);
        Dataset ds = h.dataset(name);
        if ((int64_t) ds.count() != n) throw H5Error{CUPCFD_E_ARRAY_SIZE_MISMATCH, std::string(name) + " has another size"};
        std::vector<double> v = h.real(ds);
        std::copy(v.begin(), v.end(), out);
        return CUPCFD_E_SUCCESS;
    });
}
