// Read-only HDF5 subset and the two EMAN image layouts the reference reads.
//
// The reference reads HDF5 inputs through libhdf5 (EMReader/emhdf_.cpp,
// EMReader/emhdf2_.cpp), dispatched by EMReader/emdata_.cpp:174-199: a file
// whose first 8 bytes are the HDF5 signature is read as
//   - "old style" (EMhdf) when the root group has a `num_dataset` attribute:
//     image n is the root dataset named "n" (emhdf_.cpp:123-135, 233-265),
//     nx = dims[0], ny = dims[1] (, nz = dims[2]) of its dataspace, FLOAT data
//     only, and the image is refused unless its spacing_row / spacing_col /
//     spacing_sec attributes are equal (emdata_.cpp:216-262);
//   - "new style" (EMhdf2, EMAN2) otherwise: image n is dataset
//     /MDF/images/n/image, its size the EMAN.nx / EMAN.ny / EMAN.nz attributes
//     of group /MDF/images/n converted the way EMObject::operator int does
//     (emhdf2_.cpp:245-275, 348-362, emdata_.cpp:330-372, 693-710).
// libhdf5 is not available to this project, so the file format is parsed here
// from its published specification: superblock versions 0-3 (a user block in
// front of the superblock is searched at 512, 1024, ... bytes), object
// headers versions 1 and 2 with continuation blocks, symbol-table groups
// (version 1 B-tree, symbol nodes, local heap) and compact link messages,
// dataspace, datatype (integer, IEEE float, fixed-length string), data layout
// versions 1-4 (compact, contiguous, chunked with a version 1 B-tree index or a
// single chunk), the deflate / shuffle / Fletcher-32 filters and attribute
// messages versions 1-3.  Dense (fractal-heap) link or attribute storage,
// virtual datasets, variable-length types and the other chunk indexes of
// layout version 4 are reported as unsupported.
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gisspa.h"

namespace {

constexpr uint64_t kUndef = ~0ull;

struct H5Error : std::runtime_error {
    int status;
    H5Error(int st, const std::string& m) : std::runtime_error(m), status(st) {}
};
[[noreturn]] void fail_io(const std::string& m) { throw H5Error(GS_ERR_IO, m); }
[[noreturn]] void fail_unsupported(const std::string& m) { throw H5Error(GS_ERR_UNSUPPORTED, m); }

uint64_t le(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

// Bounds-checked little-endian cursor over one block of the file.
struct Cur {
    const std::vector<uint8_t>* b;
    size_t p;
    const uint8_t* at(uint64_t n) const {
        if (p > b->size() || n > b->size() - p) fail_io("HDF5 structure runs past its block");
        return b->data() + p;
    }
    uint64_t u(int n) {
        const uint64_t v = le(at((size_t)n), n);
        p += (size_t)n;
        return v;
    }
    void skip(uint64_t n) {
        at(n);
        p += (size_t)n;
    }
};

struct Msg {
    int type = 0;
    int flags = 0;
    std::vector<uint8_t> data;
};

struct DType {
    int cls = -1;  // 0 integer, 1 float, 3 string
    int size = 0;
    bool big = false;
    bool sgn = false;
};

struct Space {
    bool null = false;
    std::vector<uint64_t> dims;  // empty: scalar
    // number of elements, saturating at 2^62 (no wrap-around for corrupt dims)
    uint64_t count() const {
        if (null) return 0;
        uint64_t n = 1;
        for (uint64_t d : dims) {
            if (d == 0) return 0;
            n = (n > (1ull << 62) / d) ? (1ull << 62) : n * d;
        }
        return n;
    }
};

struct Attr {
    DType t;
    Space s;
    std::vector<uint8_t> raw;
};

struct Layout {
    int cls = -1;  // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = kUndef, size = 0;
    std::vector<uint8_t> compact;
    std::vector<uint64_t> chunk;  // chunk dims (dataset rank)
    int index = 0;                // chunked: 0 = version 1 B-tree, 1 = single chunk
    uint64_t single_size = 0;     // single chunk: filtered size (0 = unfiltered)
    uint32_t single_mask = 0;
};

struct Filter {
    int id;
    std::vector<uint32_t> cd;
};

class File {
  public:
    explicit File(const char* path) {
        f_ = fopen(path, "rb");
        if (!f_) fail_io(std::string("cannot open HDF5 file ") + path);
        find_superblock(path);
    }
    ~File() {
        if (f_) fclose(f_);
    }
    File(const File&) = delete;
    File& operator=(const File&) = delete;

    uint64_t root() const { return root_; }

    std::vector<uint8_t> read(uint64_t addr, uint64_t n) const {
        if (addr == kUndef) fail_io("HDF5 address is undefined");
        const uint64_t a = base_ + addr;
        if (n > (1ull << 40) || a + n > fsize_ || a + n < a) fail_io("HDF5 block lies outside the file");
        std::vector<uint8_t> v((size_t)n);
        if (n && (fseeko(f_, (off_t)a, SEEK_SET) != 0 || fread(v.data(), 1, (size_t)n, f_) != n))
            fail_io("short read in HDF5 file");
        return v;
    }

    // object header messages (both header versions, continuation blocks followed)
    std::vector<Msg> messages(uint64_t addr) const {
        std::vector<Msg> out;
        if (addr == kUndef || addr >= fsize_ - base_) fail_io("HDF5 object header outside the file");
        std::vector<uint8_t> pre = read(addr, std::min<uint64_t>(64, fsize_ - base_ - addr));
        struct Block {
            uint64_t addr, len;
            bool v2cont;
        };
        std::vector<Block> todo;
        bool v2 = false;
        int oflags = 0;
        if (pre.size() >= 4 && memcmp(pre.data(), "OHDR", 4) == 0) {
            v2 = true;
            Cur c{&pre, 4};
            if (c.u(1) != 2) fail_unsupported("HDF5 object header version");
            oflags = (int)c.u(1);
            if (oflags & 0x20) c.skip(16);
            if (oflags & 0x10) c.skip(4);
            const uint64_t len0 = c.u(1 << (oflags & 3));
            todo.push_back({addr + c.p, len0, false});
        } else if (pre.size() >= 16 && pre[0] == 1) {
            Cur c{&pre, 8};
            const uint64_t hsize = c.u(4);
            todo.push_back({addr + 16, hsize, false});
        } else {
            fail_io("not an HDF5 object header");
        }
        for (size_t k = 0; k < todo.size(); ++k) {
            if (todo.size() > 4096) fail_io("HDF5 object header continuation loop");
            Block bl = todo[k];
            std::vector<uint8_t> b;
            size_t end;
            Cur c{nullptr, 0};
            if (bl.v2cont) {
                b = read(bl.addr, bl.len);
                if (b.size() < 8 || memcmp(b.data(), "OCHK", 4) != 0) fail_io("bad HDF5 continuation block");
                c = Cur{&b, 4};
                end = b.size() - 4;  // checksum
            } else {
                b = read(bl.addr, bl.len);
                c = Cur{&b, 0};
                end = b.size();
            }
            const size_t hdr = v2 ? (4 + ((oflags & 0x04) ? 2 : 0)) : 8;
            while (c.p + hdr <= end) {
                Msg m;
                if (v2) {
                    m.type = (int)c.u(1);
                    const uint64_t sz = c.u(2);
                    m.flags = (int)c.u(1);
                    if (oflags & 0x04) c.skip(2);
                    if (c.p + sz > end) fail_io("HDF5 message runs past its header");
                    m.data.assign(b.data() + c.p, b.data() + c.p + sz);
                    c.p += sz;
                } else {
                    m.type = (int)c.u(2);
                    const uint64_t sz = c.u(2);
                    m.flags = (int)c.u(1);
                    c.skip(3);
                    if (c.p + sz > end) fail_io("HDF5 message runs past its header");
                    m.data.assign(b.data() + c.p, b.data() + c.p + sz);
                    c.p += sz;
                }
                if (m.type == 0x10) {  // continuation
                    Cur d{&m.data, 0};
                    const uint64_t ca = d.u(so_), cl = d.u(sl_);
                    todo.push_back({ca, cl, v2});
                } else if (m.type != 0) {
                    out.push_back(std::move(m));
                }
            }
        }
        return out;
    }

    // object header address of `path` (absolute, '/'-separated); false if absent
    bool lookup(const std::string& path, uint64_t* addr) const {
        uint64_t cur = root_;
        size_t i = 0;
        while (i < path.size()) {
            while (i < path.size() && path[i] == '/') ++i;
            if (i >= path.size()) break;
            size_t j = path.find('/', i);
            if (j == std::string::npos) j = path.size();
            if (!child(cur, path.substr(i, j - i), &cur)) return false;
            i = j;
        }
        *addr = cur;
        return true;
    }

    DType dtype(const uint8_t* p, size_t n) const {
        if (n < 8) fail_io("short HDF5 datatype message");
        DType t;
        t.cls = p[0] & 0x0f;
        t.size = (int)le(p + 4, 4);
        if (t.cls == 0) {
            t.big = p[1] & 1;
            t.sgn = (p[1] >> 3) & 1;
            if (t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8) fail_unsupported("HDF5 integer size");
        } else if (t.cls == 1) {
            if (p[1] & 0x40) fail_unsupported("VAX-order HDF5 floats");
            t.big = p[1] & 1;
            if (t.size != 4 && t.size != 8) fail_unsupported("HDF5 float size");
        } else if (t.cls != 3) {
            t.cls = -1 - t.cls;  // not readable here (compound, variable length, ...)
        }
        return t;
    }

    Space space(const uint8_t* p, size_t n) const {
        std::vector<uint8_t> b(p, p + n);
        Cur c{&b, 0};
        const int ver = (int)c.u(1), rank = (int)c.u(1), flags = (int)c.u(1);
        Space s;
        if (ver == 1) {
            c.skip(5);
        } else if (ver == 2) {
            const int type = (int)c.u(1);
            if (type == 2) s.null = true;
        } else {
            fail_unsupported("HDF5 dataspace version");
        }
        (void)flags;
        for (int k = 0; k < rank; ++k) s.dims.push_back(c.u(sl_));
        return s;
    }

    // attributes of the object at `addr`, by name
    std::map<std::string, Attr> attributes(uint64_t addr) const {
        std::map<std::string, Attr> out;
        for (const Msg& m : messages(addr)) {
            if (m.type == 0x15) {  // attribute info: dense storage not read here
                Cur c{&m.data, 0};
                c.skip(1);
                const int fl = (int)c.u(1);
                if (fl & 1) c.skip(2);
                if (c.u(so_) != kUndef) fail_unsupported("dense HDF5 attribute storage");
                continue;
            }
            if (m.type != 0x0C) continue;
            if (m.flags & 0x02) fail_unsupported("shared HDF5 attribute message");
            Cur c{&m.data, 0};
            const int ver = (int)c.u(1);
            const int aflags = (int)c.u(1);
            const uint64_t nlen = c.u(2), tlen = c.u(2), slen = c.u(2);
            if (ver == 3) c.skip(1);
            if (ver < 1 || ver > 3) fail_unsupported("HDF5 attribute message version");
            if (aflags & 0x03) fail_unsupported("shared HDF5 attribute type or space");
            auto pad = [&](uint64_t x) { return ver == 1 ? (x + 7) / 8 * 8 : x; };
            const uint8_t* np = c.at(nlen);
            std::string name((const char*)np, strnlen((const char*)np, nlen));
            c.skip(pad(nlen));
            Attr a;
            a.t = dtype(c.at(tlen), tlen);
            c.skip(pad(tlen));
            a.s = space(c.at(slen), slen);
            c.skip(pad(slen));
            // the element count is bounded by the bytes left in the message
            // before it is multiplied (a corrupt dataspace can claim 2^62)
            uint64_t bytes = 0;
            if (a.t.cls >= 0 && a.t.size > 0) {
                const uint64_t left = m.data.size() - c.p;
                const uint64_t n = a.s.count();
                if (n > left / (uint64_t)a.t.size) fail_io("HDF5 attribute " + name + " runs past its message");
                bytes = n * (uint64_t)a.t.size;
            }
            a.raw.assign(c.at(bytes), c.at(bytes) + bytes);
            out[name] = std::move(a);
        }
        return out;
    }

    struct Dataset {
        DType t;
        Space s;
        Layout lay;
        std::vector<Filter> filters;
    };
    Dataset dataset(uint64_t addr) const {
        Dataset d;
        bool have_t = false, have_s = false;
        for (const Msg& m : messages(addr)) {
            if ((m.type == 0x01 || m.type == 0x03 || m.type == 0x08) && (m.flags & 0x02))
                fail_unsupported("shared HDF5 dataset message");
            if (m.type == 0x01) {
                d.s = space(m.data.data(), m.data.size());
                have_s = true;
            } else if (m.type == 0x03) {
                d.t = dtype(m.data.data(), m.data.size());
                have_t = true;
            } else if (m.type == 0x08) {
                d.lay = layout(m.data);
            } else if (m.type == 0x0B) {
                d.filters = filters(m.data);
            }
        }
        if (!have_t || !have_s || d.lay.cls < 0) fail_io("HDF5 object is not a dataset");
        return d;
    }

    // raw bytes of a dataset in row-major element order
    std::vector<uint8_t> raw(const Dataset& d) const {
        const uint64_t es = (uint64_t)d.t.size;
        const uint64_t n = d.s.count();
        if (n > (1ull << 31) / std::max<uint64_t>(es, 1)) fail_unsupported("HDF5 dataset above 2 GB");
        const uint64_t bytes = n * es;
        if (d.lay.cls == 0) {
            if (d.lay.compact.size() < bytes) fail_io("short compact HDF5 dataset");
            return std::vector<uint8_t>(d.lay.compact.begin(), d.lay.compact.begin() + bytes);
        }
        if (d.lay.cls == 1) {
            if (d.lay.addr == kUndef) return std::vector<uint8_t>(bytes, 0);  // never written: fill value 0
            return read(d.lay.addr, bytes);
        }
        // chunked
        const int rank = (int)d.s.dims.size();
        if ((int)d.lay.chunk.size() != rank) fail_io("HDF5 chunk rank does not match the dataspace");
        uint64_t cbytes = es;
        for (uint64_t c : d.lay.chunk) {
            if (c == 0 || c > (1ull << 31) / cbytes) fail_io("bad HDF5 chunk dimensions");
            cbytes *= c;
        }
        std::vector<uint8_t> out(bytes, 0);
        auto place = [&](const std::vector<uint64_t>& off, std::vector<uint8_t> chunk, uint32_t mask) {
            chunk = unfilter(std::move(chunk), d.filters, mask, cbytes);
            if (chunk.size() < cbytes) fail_io("short HDF5 chunk");
            // copy the part of the chunk inside the dataspace, row by row of the last dimension
            std::vector<uint64_t> idx(rank, 0);
            const uint64_t last = d.lay.chunk[rank - 1];
            while (true) {
                bool inside = true;
                uint64_t dst = 0, src = 0;
                for (int k = 0; k < rank; ++k) {
                    const uint64_t g = off[k] + idx[k];
                    if (k < rank - 1 && g >= d.s.dims[k]) inside = false;
                    dst = dst * d.s.dims[k] + g;
                    src = src * d.lay.chunk[k] + idx[k];
                }
                if (inside && off[rank - 1] < d.s.dims[rank - 1]) {
                    const uint64_t cnt = std::min<uint64_t>(last, d.s.dims[rank - 1] - off[rank - 1]);
                    if (dst > n || cnt > n - dst || (src + cnt) * es > chunk.size())
                        fail_io("HDF5 chunk outside its dataset");
                    memcpy(out.data() + dst * es, chunk.data() + src * es, cnt * es);
                }
                int k = rank - 2;
                for (; k >= 0; --k) {
                    if (++idx[k] < d.lay.chunk[k]) break;
                    idx[k] = 0;
                }
                if (k < 0) break;
            }
        };
        if (rank == 0) fail_io("chunked scalar HDF5 dataset");
        if (d.lay.index == 1) {
            if (d.lay.addr == kUndef) return out;
            const uint64_t sz = d.lay.single_size ? d.lay.single_size : cbytes;
            place(std::vector<uint64_t>(rank, 0), read(d.lay.addr, sz), d.lay.single_mask);
            return out;
        }
        if (d.lay.addr == kUndef) return out;
        uint64_t budget = 1u << 20;  // B-tree nodes and chunks visited, against corrupt cycles
        walk_chunks(d.lay.addr, rank + 1, place, 0, &budget);
        return out;
    }

  private:
    FILE* f_ = nullptr;
    uint64_t fsize_ = 0, base_ = 0, root_ = kUndef;
    int so_ = 8, sl_ = 8;

    void find_superblock(const char* path) {
        fseeko(f_, 0, SEEK_END);
        fsize_ = (uint64_t)ftello(f_);
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        uint64_t at = kUndef;
        for (uint64_t off = 0; off + 8 <= fsize_; off = off ? off * 2 : 512) {
            uint8_t s[8];
            if (fseeko(f_, (off_t)off, SEEK_SET) != 0 || fread(s, 1, 8, f_) != 8) break;
            if (memcmp(s, sig, 8) == 0) {
                at = off;
                break;
            }
        }
        if (at == kUndef) fail_io(std::string("no HDF5 signature in ") + path);
        base_ = 0;
        std::vector<uint8_t> sb = read(at, std::min<uint64_t>(128, fsize_ - at));
        Cur c{&sb, 8};
        const int ver = (int)c.u(1);
        if (ver == 0 || ver == 1) {
            c.skip(3);  // free-space, root symbol table entry, reserved
            c.skip(1);  // shared header version
            so_ = (int)c.u(1);
            sl_ = (int)c.u(1);
            c.skip(1);
            c.skip(4);  // leaf / internal K
            c.skip(4);  // consistency flags
            if (ver == 1) c.skip(4);
            check_sizes();
            base_ = c.u(so_);
            c.skip((size_t)so_ * 3);  // free space, end of file, driver block
            c.skip(so_);              // root entry: link name offset
            root_ = c.u(so_);
        } else if (ver == 2 || ver == 3) {
            so_ = (int)c.u(1);
            sl_ = (int)c.u(1);
            c.skip(1);
            check_sizes();
            base_ = c.u(so_);
            c.skip((size_t)so_ * 2);  // superblock extension, end of file
            root_ = c.u(so_);
        } else {
            fail_unsupported("HDF5 superblock version " + std::to_string(ver));
        }
        // addresses are relative to the superblock's own position (a user
        // block may precede it), whatever base address it records
        base_ = at;
    }
    void check_sizes() const {
        if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) fail_unsupported("HDF5 offset / length size");
    }

    // name -> object header address in the group whose header is at `grp`
    bool child(uint64_t grp, const std::string& name, uint64_t* out) const {
        for (const Msg& m : messages(grp)) {
            if (m.type == 0x11) {  // symbol table: B-tree + local heap
                Cur c{&m.data, 0};
                const uint64_t bt = c.u(so_), heap = c.u(so_);
                const std::vector<uint8_t> names = heap_data(heap);
                return btree_find(bt, names, name, out, 0);
            }
            if (m.type == 0x02) {  // link info
                Cur c{&m.data, 0};
                c.skip(1);
                const int fl = (int)c.u(1);
                if (fl & 1) c.skip(8);
                if (c.u(so_) != kUndef) fail_unsupported("dense HDF5 link storage");
            }
            if (m.type == 0x06) {  // compact link
                Cur c{&m.data, 0};
                if (c.u(1) != 1) fail_unsupported("HDF5 link message version");
                const int fl = (int)c.u(1);
                const int ltype = (fl & 0x08) ? (int)c.u(1) : 0;
                if (fl & 0x04) c.skip(8);
                if (fl & 0x10) c.skip(1);
                const uint64_t nl = c.u(1 << (fl & 3));
                const std::string nm((const char*)c.at(nl), (size_t)nl);
                c.skip(nl);
                if (nm == name) {
                    if (ltype != 0) fail_unsupported("soft or external HDF5 link " + name);
                    *out = c.u(so_);
                    return true;
                }
            }
        }
        return false;
    }

    std::vector<uint8_t> heap_data(uint64_t addr) const {
        const std::vector<uint8_t> h = read(addr, 8 + 2 * (uint64_t)sl_ + so_);
        if (memcmp(h.data(), "HEAP", 4) != 0) fail_io("bad HDF5 local heap");
        Cur c{&h, 8};
        const uint64_t size = c.u(sl_);
        c.skip(sl_);
        const uint64_t data = c.u(so_);
        return read(data, size);
    }
    static std::string heap_name(const std::vector<uint8_t>& names, uint64_t off) {
        if (off >= names.size()) fail_io("HDF5 heap offset out of range");
        const char* s = (const char*)names.data() + off;
        return std::string(s, strnlen(s, names.size() - off));
    }

    // version 1 B-tree of a group: the child whose key range holds `name`
    bool btree_find(uint64_t node, const std::vector<uint8_t>& names, const std::string& name, uint64_t* out,
                    int depth) const {
        if (depth > 64) fail_io("HDF5 group B-tree too deep");
        const uint64_t hdr = 8 + 2 * (uint64_t)so_;
        std::vector<uint8_t> h = read(node, hdr);
        if (memcmp(h.data(), "TREE", 4) != 0 || h[4] != 0) fail_io("bad HDF5 group B-tree node");
        const int level = h[5];
        const uint64_t used = le(h.data() + 6, 2);
        const std::vector<uint8_t> b = read(node + hdr, used * (sl_ + so_) + sl_);
        Cur c{&b, 0};
        std::vector<uint64_t> keys, kids;
        for (uint64_t i = 0; i < used; ++i) {
            keys.push_back(c.u(sl_));
            kids.push_back(c.u(so_));
        }
        keys.push_back(c.u(sl_));
        for (uint64_t i = 0; i < used; ++i) {
            // child i holds names in (key i, key i+1]
            if (name.compare(heap_name(names, keys[i + 1])) > 0) continue;
            if (level > 0) return btree_find(kids[i], names, name, out, depth + 1);
            return snod_find(kids[i], names, name, out);
        }
        return false;
    }
    bool snod_find(uint64_t addr, const std::vector<uint8_t>& names, const std::string& name, uint64_t* out) const {
        const std::vector<uint8_t> h = read(addr, 8);
        if (memcmp(h.data(), "SNOD", 4) != 0) fail_io("bad HDF5 symbol table node");
        const uint64_t n = le(h.data() + 6, 2);
        const uint64_t es = 2 * (uint64_t)so_ + 24;
        const std::vector<uint8_t> b = read(addr + 8, n * es);
        for (uint64_t i = 0; i < n; ++i) {
            Cur c{&b, (size_t)(i * es)};
            const uint64_t noff = c.u(so_), ohdr = c.u(so_);
            if (heap_name(names, noff) == name) {
                *out = ohdr;
                return true;
            }
        }
        return false;
    }

    Layout layout(const std::vector<uint8_t>& m) const {
        Cur c{&m, 0};
        Layout L;
        const int ver = (int)c.u(1);
        if (ver == 1 || ver == 2) {
            const int nd = (int)c.u(1);
            L.cls = (int)c.u(1);
            c.skip(5);
            if (L.cls != 0) L.addr = c.u(so_);
            std::vector<uint64_t> dims;
            for (int k = 0; k < nd; ++k) dims.push_back(c.u(4));
            if (L.cls == 0) {
                const uint64_t sz = c.u(4);
                L.compact.assign(c.at(sz), c.at(sz) + sz);
            } else if (L.cls == 2) {
                if (nd < 2) fail_io("bad HDF5 chunk dimensions");
                L.chunk.assign(dims.begin(), dims.end() - 1);  // the last is the element size
            }
        } else if (ver == 3 || ver == 4) {
            L.cls = (int)c.u(1);
            if (L.cls == 0) {
                const uint64_t sz = c.u(2);
                L.compact.assign(c.at(sz), c.at(sz) + sz);
            } else if (L.cls == 1) {
                L.addr = c.u(so_);
                L.size = c.u(sl_);
            } else if (L.cls == 2 && ver == 3) {
                const int nd = (int)c.u(1);
                L.addr = c.u(so_);
                for (int k = 0; k < nd; ++k) L.chunk.push_back(c.u(4));
                if (nd < 2) fail_io("bad HDF5 chunk dimensions");
                L.chunk.pop_back();
            } else if (L.cls == 2) {
                const int fl = (int)c.u(1);
                const int nd = (int)c.u(1);
                const int w = (int)c.u(1);
                for (int k = 0; k < nd; ++k) L.chunk.push_back(c.u(w));
                if (nd < 2) fail_io("bad HDF5 chunk dimensions");
                L.chunk.pop_back();
                const int idx = (int)c.u(1);
                if (idx != 1) fail_unsupported("HDF5 chunk index type " + std::to_string(idx));
                L.index = 1;
                if (fl & 0x02) {
                    L.single_size = c.u(sl_);
                    L.single_mask = (uint32_t)c.u(4);
                }
                L.addr = c.u(so_);
            } else {
                fail_unsupported("HDF5 layout class " + std::to_string(L.cls));
            }
        } else {
            fail_unsupported("HDF5 layout version " + std::to_string(ver));
        }
        return L;
    }

    std::vector<Filter> filters(const std::vector<uint8_t>& m) const {
        Cur c{&m, 0};
        const int ver = (int)c.u(1), n = (int)c.u(1);
        if (ver == 1) c.skip(6);
        else if (ver != 2) fail_unsupported("HDF5 filter pipeline version");
        std::vector<Filter> out;
        for (int i = 0; i < n; ++i) {
            Filter f;
            f.id = (int)c.u(2);
            const uint64_t nl = (ver == 1 || f.id >= 256) ? c.u(2) : 0;
            c.skip(2);  // flags
            const int ncd = (int)c.u(2);
            c.skip(ver == 1 ? (nl + 7) / 8 * 8 : nl);
            for (int k = 0; k < ncd; ++k) f.cd.push_back((uint32_t)c.u(4));
            if (ver == 1 && (ncd & 1)) c.skip(4);
            out.push_back(f);
        }
        return out;
    }

    static std::vector<uint8_t> unfilter(std::vector<uint8_t> b, const std::vector<Filter>& fs, uint32_t mask,
                                         uint64_t nominal) {
        for (int i = (int)fs.size() - 1; i >= 0; --i) {
            if (mask & (1u << i)) continue;
            const Filter& f = fs[i];
            if (f.id == 1) {  // deflate
                std::vector<uint8_t> out((size_t)nominal);
                z_stream z;
                memset(&z, 0, sizeof z);
                if (inflateInit(&z) != Z_OK) fail_io("zlib initialisation failed");
                z.next_in = b.data();
                z.avail_in = (uInt)b.size();
                z.next_out = out.data();
                z.avail_out = (uInt)out.size();
                const int r = inflate(&z, Z_FINISH);
                const uint64_t got = z.total_out;
                inflateEnd(&z);
                if (r != Z_STREAM_END) fail_io("corrupt deflate-compressed HDF5 chunk");
                out.resize((size_t)got);
                b.swap(out);
            } else if (f.id == 2) {  // shuffle
                const size_t es = f.cd.empty() ? 1 : f.cd[0];
                if (es > 1) {
                    const size_t n = b.size() / es;
                    std::vector<uint8_t> out(b.size());
                    for (size_t k = 0; k < es; ++k)
                        for (size_t j = 0; j < n; ++j) out[j * es + k] = b[k * n + j];
                    memcpy(out.data() + n * es, b.data() + n * es, b.size() - n * es);
                    b.swap(out);
                }
            } else if (f.id == 3) {  // Fletcher-32: checksum appended
                if (b.size() < 4) fail_io("short Fletcher-32 HDF5 chunk");
                b.resize(b.size() - 4);
            } else {
                fail_unsupported("HDF5 filter " + std::to_string(f.id));
            }
        }
        return b;
    }

    template <class Place>
    void walk_chunks(uint64_t node, int nkey, Place& place, int depth, uint64_t* budget) const {
        if (depth > 64) fail_io("HDF5 chunk B-tree too deep");
        if ((*budget)-- == 0) fail_io("HDF5 chunk B-tree visits too many nodes");
        const uint64_t hdr = 8 + 2 * (uint64_t)so_;
        const std::vector<uint8_t> h = read(node, hdr);
        if (memcmp(h.data(), "TREE", 4) != 0 || h[4] != 1) fail_io("bad HDF5 chunk B-tree node");
        const int level = h[5];
        const uint64_t used = le(h.data() + 6, 2);
        const uint64_t ks = 8 + 8 * (uint64_t)nkey;
        const std::vector<uint8_t> b = read(node + hdr, used * (ks + so_) + ks);
        Cur c{&b, 0};
        for (uint64_t i = 0; i < used; ++i) {
            const uint64_t csize = c.u(4);
            const uint32_t mask = (uint32_t)c.u(4);
            std::vector<uint64_t> off;
            for (int k = 0; k < nkey; ++k) off.push_back(c.u(8));
            off.pop_back();
            const uint64_t kid = c.u(so_);
            if (level > 0) {
                walk_chunks(kid, nkey, place, depth + 1, budget);
            } else {
                if ((*budget)-- == 0) fail_io("HDF5 chunk B-tree visits too many chunks");
                place(off, read(kid, csize), mask);
            }
        }
    }
};

template <class T>
void convert(const DType& t, const std::vector<uint8_t>& raw, uint64_t n, T* out) {
    const int es = t.size;
    for (uint64_t i = 0; i < n; ++i) {
        uint8_t b[8];
        const uint8_t* p = raw.data() + i * es;
        for (int k = 0; k < es; ++k) b[k] = t.big ? p[es - 1 - k] : p[k];
        const uint64_t u = le(b, es);
        double v;
        if (t.cls == 1) {
            if (es == 4) {
                uint32_t w = (uint32_t)u;
                float f;
                memcpy(&f, &w, 4);
                v = f;
            } else {
                memcpy(&v, &u, 8);
            }
        } else if (t.sgn) {
            const int sh = 64 - 8 * es;
            v = (double)((int64_t)(u << sh) >> sh);
        } else {
            v = (double)u;
        }
        out[i] = (T)v;
    }
}

// EMObject::operator int of an attribute as EMhdf2::read_attr builds it
// (emhdf2_.cpp:191-236, emdata_.cpp:693-710): integers as int, a scalar
// 4-byte float truncated, an 8-byte float's first value truncated, anything
// else (strings, float arrays, a missing attribute) 0.
int eman_int(const std::map<std::string, Attr>& attrs, const std::string& key) {
    auto it = attrs.find(key);
    if (it == attrs.end()) return 0;
    const Attr& a = it->second;
    if (a.raw.empty()) return 0;
    if (a.t.cls == 0) {
        int64_t v;
        convert(a.t, a.raw, 1, &v);
        return (int)v;
    }
    if (a.t.cls == 1) {
        if (a.t.size == 4 && a.s.count() != 1) return 0;
        double v;
        convert(a.t, a.raw, 1, &v);
        return (int)v;
    }
    return 0;
}

// A float attribute read through H5T_NATIVE_FLOAT, 0 when absent
// (EMhdf::read_float_attr, emhdf_.cpp:289-298).
float float_attr(const std::map<std::string, Attr>& attrs, const std::string& key) {
    auto it = attrs.find(key);
    if (it == attrs.end() || it->second.raw.empty() || (it->second.t.cls != 0 && it->second.t.cls != 1)) return 0.0f;
    float v;
    convert(it->second.t, it->second.raw, 1, &v);
    return v;
}

int report(const H5Error& e, char* err, size_t err_len) {
    if (err && err_len) snprintf(err, err_len, "%s", e.what());
    return e.status;
}
int report_oom(char* err, size_t err_len) {
    if (err && err_len) snprintf(err, err_len, "out of host memory");
    return GS_ERR_OOM;
}
// any other exception (e.g. std::length_error) must not leave an extern "C"
// function: it is reported as an unreadable file
int report_other(const std::exception& e, char* err, size_t err_len) {
    if (err && err_len) snprintf(err, err_len, "HDF5 read failed: %s", e.what());
    return GS_ERR_IO;
}

}  // namespace

extern "C" int gs_hdf_read_image(const char* path, int index, float** host_data, int* nx, int* ny, int* nz,
                                 char* err, size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!path || !host_data || !nx || !ny || !nz) return GS_ERR_ARG;
    *host_data = nullptr;
    *nx = *ny = *nz = 0;
    try {
        {
            // is_valid (emhdf_.cpp:47-62): the signature at offset 0 only
            FILE* f = fopen(path, "rb");
            if (!f) fail_io(std::string("cannot open ") + path);
            uint8_t s[8] = {0};
            const size_t got = fread(s, 1, 8, f);
            fclose(f);
            static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
            if (got != 8 || memcmp(s, sig, 8) != 0) fail_io(std::string("not an HDF5 file: ") + path);
        }
        File h(path);
        if (index < 0) index = 0;
        const std::map<std::string, Attr> root_attrs = h.attributes(h.root());
        const bool old_style = root_attrs.count("num_dataset") != 0;  // EMhdf::init_test
        int w = 0, hgt = 0, d = 0;
        uint64_t ds_addr = 0;
        const std::string idx = std::to_string(index);
        if (old_style) {
            if (!h.lookup("/" + idx, &ds_addr)) fail_io("HDF5 file has no dataset " + idx + ": " + path);
        } else {
            uint64_t g = 0;
            if (!h.lookup("/MDF/images/" + idx, &g)) fail_io("HDF5 file has no image group /MDF/images/" + idx);
            const std::map<std::string, Attr> all = h.attributes(g);
            std::map<std::string, Attr> em;
            for (const auto& kv : all)
                if (kv.first.compare(0, 5, "EMAN.") == 0) em[kv.first.substr(5)] = kv.second;
            const int ax = eman_int(em, "nx"), ay = eman_int(em, "ny"), az = eman_int(em, "nz");
            // emdata_.cpp:347-360
            if (az > 1) { w = ax; hgt = ay; d = az; }
            else if (ay > 1) { w = ax; hgt = ay; d = 1; }
            else if (ax > 1) { w = ax; hgt = 1; d = 1; }
            else fail_io("EMAN image " + idx + " has no size attributes: " + path);
            if (!h.lookup("/MDF/images/" + idx + "/image", &ds_addr))
                fail_io("HDF5 image /MDF/images/" + idx + "/image does not exist: " + path);
        }
        const File::Dataset ds = h.dataset(ds_addr);
        if (old_style) {
            // read_dims + readHDF (emhdf_.cpp:123-160, emdata_.cpp:228-240)
            const auto& dm = ds.s.dims;
            if (dm.size() == 3) { w = (int)dm[0]; hgt = (int)dm[1]; d = (int)dm[2]; }
            else if (dm.size() == 2) { w = (int)dm[0]; hgt = (int)dm[1]; d = 1; }
            else fail_io("HDF5 dataset " + idx + " is not 2D or 3D: " + path);
            if (ds.t.cls != 1) fail_unsupported(std::string("old-style EMAN HDF data must be floating point: ") + path);
        } else if (ds.t.cls != 0 && ds.t.cls != 1) {
            fail_unsupported(std::string("EMAN HDF image of a non-numeric type: ") + path);
        }
        const uint64_t n = (uint64_t)w * hgt * d;
        if (w <= 0 || hgt <= 0 || d <= 0 || ds.s.count() != n)
            fail_io("EMAN HDF image " + idx + ": dataset size does not match nx * ny * nz: " + path);
        const std::vector<uint8_t> raw = h.raw(ds);
        if (old_style) {
            // the pixel size must be isotropic (emdata_.cpp:248-258)
            const std::map<std::string, Attr> da = h.attributes(ds_addr);
            const float px = float_attr(da, "spacing_row"), py = float_attr(da, "spacing_col"),
                        pz = float_attr(da, "spacing_sec");
            if (!(px == py && px == pz)) fail_io(std::string("old-style EMAN HDF image with anisotropic spacing: ") + path);
        }
        float* out = (float*)malloc(sizeof(float) * (size_t)n);
        if (!out) return report_oom(err, err_len);
        convert(ds.t, raw, n, out);
        *host_data = out;
        *nx = w;
        *ny = hgt;
        *nz = d;
        return GS_OK;
    } catch (const H5Error& e) {
        return report(e, err, err_len);
    } catch (const std::bad_alloc&) {
        return report_oom(err, err_len);
    } catch (const std::exception& e) {
        return report_other(e, err, err_len);
    }
}

extern "C" int gs_hdf_read_dataset(const char* path, const char* name, double** host_data, int64_t* dims,
                                   int* rank, char* err, size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!path || !name || !host_data || !dims || !rank) return GS_ERR_ARG;
    *host_data = nullptr;
    *rank = 0;
    try {
        File h(path);
        uint64_t a = 0;
        if (!h.lookup(name, &a)) fail_io(std::string("no HDF5 object ") + name + " in " + path);
        const File::Dataset ds = h.dataset(a);
        if (ds.t.cls != 0 && ds.t.cls != 1) fail_unsupported(std::string("non-numeric HDF5 dataset ") + name);
        if (ds.s.dims.size() > 8) fail_unsupported("HDF5 dataset rank above 8");
        const uint64_t n = ds.s.count();
        const std::vector<uint8_t> raw = h.raw(ds);
        double* out = (double*)malloc(sizeof(double) * (size_t)std::max<uint64_t>(n, 1));
        if (!out) return report_oom(err, err_len);
        convert(ds.t, raw, n, out);
        for (size_t k = 0; k < ds.s.dims.size(); ++k) dims[k] = (int64_t)ds.s.dims[k];
        *rank = (int)ds.s.dims.size();
        *host_data = out;
        return GS_OK;
    } catch (const H5Error& e) {
        return report(e, err, err_len);
    } catch (const std::bad_alloc&) {
        return report_oom(err, err_len);
    } catch (const std::exception& e) {
        return report_other(e, err, err_len);
    }
}

extern "C" int gs_hdf_read_attribute(const char* path, const char* object, const char* name, double* values,
                                     size_t max_values, size_t* n_values, char* text, size_t text_len, char* err,
                                     size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!path || !object || !name || !n_values) return GS_ERR_ARG;
    *n_values = 0;
    if (text && text_len) text[0] = 0;
    try {
        File h(path);
        uint64_t a = 0;
        if (!h.lookup(object, &a)) fail_io(std::string("no HDF5 object ") + object + " in " + path);
        const std::map<std::string, Attr> at = h.attributes(a);
        auto it = at.find(name);
        if (it == at.end()) fail_io(std::string("no attribute ") + name + " on " + object);
        const Attr& v = it->second;
        if (v.t.cls == 3) {
            if (text && text_len) {
                const size_t len = strnlen((const char*)v.raw.data(), v.raw.size());
                snprintf(text, text_len, "%.*s", (int)len, (const char*)v.raw.data());
            }
            return GS_OK;
        }
        if (v.t.cls != 0 && v.t.cls != 1) fail_unsupported(std::string("HDF5 attribute type of ") + name);
        const uint64_t n = v.s.count();
        *n_values = (size_t)n;
        if (values && max_values) {
            std::vector<double> all((size_t)n);
            convert(v.t, v.raw, n, all.data());
            for (size_t k = 0; k < std::min<size_t>(max_values, (size_t)n); ++k) values[k] = all[k];
        }
        return GS_OK;
    } catch (const H5Error& e) {
        return report(e, err, err_len);
    } catch (const std::bad_alloc&) {
        return report_oom(err, err_len);
    } catch (const std::exception& e) {
        return report_other(e, err, err_len);
    }
}

extern "C" void gs_host_free(void* p) { free(p); }
