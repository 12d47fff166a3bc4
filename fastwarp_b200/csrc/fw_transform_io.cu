// fw_transform_io.cu -- ITK transform files of a registration (host code, no device work).
//
// Composite.h5 / InverseComposite.h5: the reference writes its own HDF5 subset
// (transform/hdf5.rs:1127-1400), so these bytes follow that layout, not libhdf5's: a 48-byte
// version-2 superblock; one global heap collection right after it holding every string of the
// file in tree order; then the tree written depth first, each dataset as its raw data (8-byte
// aligned) followed by its object header (dataspace, datatype, fill value, contiguous layout),
// each group after its members as an object header of link-info, group-info and one link
// message per member. Object headers are version 2 without timestamps, closed by the lookup3
// checksum of their bytes. ITK's tree is transform/itk_h5.rs:108-190.
//
// 0GenericAffine.mat: per affine two MATLAB v4 column vectors, `AffineTransform_double_3_3`
// (12 parameters) and `fixed` (the centre) -- transform/itk_mat.rs:134-165.
//
// A field's displacements (float32, possibly hundreds of MB) are widened to f64 only while they
// are written: the metadata is laid out first with a gap for each, and the gaps are filled in
// blocks as the bytes go out.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fw_internal.cuh"
#include "../../include/fastwarp_transform_io.h"

namespace fw {
namespace {

constexpr uint64_t kUndef = ~uint64_t(0);

struct Bytes {
    std::vector<uint8_t> v;
    void u8(unsigned x) { v.push_back((uint8_t)x); }
    void le(uint64_t x, int width) {
        for (int i = 0; i < width; ++i) v.push_back((uint8_t)(x >> (8 * i)));
    }
    void raw(const void* p, size_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        v.insert(v.end(), b, b + n);
    }
    void str(const std::string& s) { raw(s.data(), s.size()); }
    void align8() { v.resize((v.size() + 7) / 8 * 8, 0); }
    size_t size() const { return v.size(); }
};

inline uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

// Bob Jenkins, lookup3.c (2006, public domain): hashlittle, byte-at-a-time reads.
uint32_t lookup3(const uint8_t* k, size_t length, uint32_t initval) {
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (uint32_t)length + initval;
    auto word = [](const uint8_t* p, size_t n) {
        uint32_t w = 0;
        for (size_t i = 0; i < n && i < 4; ++i) w |= (uint32_t)p[i] << (8 * i);
        return w;
    };
    while (length > 12) {
        a += word(k, 4);
        b += word(k + 4, 4);
        c += word(k + 8, 4);
        a -= c; a ^= rotl(c, 4);  c += b;
        b -= a; b ^= rotl(a, 6);  a += c;
        c -= b; c ^= rotl(b, 8);  b += a;
        a -= c; a ^= rotl(c, 16); c += b;
        b -= a; b ^= rotl(a, 19); a += c;
        c -= b; c ^= rotl(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    if (length == 0) return c;
    a += word(k, length);
    if (length > 4) b += word(k + 4, length - 4);
    if (length > 8) c += word(k + 8, length - 8);
    c ^= b; c -= rotl(b, 14);
    a ^= c; a -= rotl(c, 11);
    b ^= a; b -= rotl(a, 25);
    c ^= b; c -= rotl(b, 16);
    a ^= c; a -= rotl(c, 4);
    b ^= a; b -= rotl(a, 14);
    c ^= b; c -= rotl(b, 24);
    return c;
}

// ---- the HDF5 subset ------------------------------------------------------------------------

struct Node {
    enum Kind { Group, F64, F32Wide, Str } kind;
    std::string name;
    std::vector<Node> members;   // Group
    std::vector<double> d;       // F64
    const float* f = nullptr;    // F32Wide: float32 values written as f64
    size_t n = 0;
    std::string s;               // Str
};

Node group(std::string name, std::vector<Node> members) {
    Node x;
    x.kind = Node::Group;
    x.name = std::move(name);
    x.members = std::move(members);
    return x;
}
Node f64s(std::string name, std::vector<double> d) {
    Node x;
    x.kind = Node::F64;
    x.name = std::move(name);
    x.d = std::move(d);
    return x;
}
Node f32wide(std::string name, const float* f, size_t n) {
    Node x;
    x.kind = Node::F32Wide;
    x.name = std::move(name);
    x.f = f;
    x.n = n;
    return x;
}
Node text(std::string name, std::string s) {
    Node x;
    x.kind = Node::Str;
    x.name = std::move(name);
    x.s = std::move(s);
    return x;
}

struct Msg {
    uint8_t type, flags;
    Bytes body;
};

// Version-2 object header: "OHDR", version 2, the width flag of the chunk-size field (1, 2 or
// 4 bytes), the chunk size, the messages, the checksum.
Bytes object_header(const std::vector<Msg>& msgs) {
    size_t total = 0;
    for (const Msg& m : msgs) total += 4 + m.body.size();
    int flag = total <= 0xff ? 0 : (total <= 0xffff ? 1 : 2);
    Bytes h;
    h.str("OHDR");
    h.u8(2);
    h.u8((unsigned)flag);
    h.le(total, 1 << flag);
    for (const Msg& m : msgs) {
        h.u8(m.type);
        h.le(m.body.size(), 2);
        h.u8(m.flags);
        h.raw(m.body.v.data(), m.body.size());
    }
    h.le(lookup3(h.v.data(), h.size(), 0), 4);
    return h;
}

Msg msg(uint8_t type, uint8_t flags, std::initializer_list<uint8_t> b) {
    Msg m{type, flags, {}};
    m.body.v.assign(b.begin(), b.end());
    return m;
}

Msg dataspace1(uint64_t n) {  // version 2, rank 1, maximum dimensions present, simple
    Msg m = msg(0x01, 1, {2, 1, 1, 1});
    m.body.le(n, 8);
    m.body.le(n, 8);
    return m;
}

// IEEE f64, little-endian: class 1 version 1, size 8, offset 0, precision 64, exponent at 52
// (11 bits), mantissa at 0 (52 bits), exponent bias 1023.
Msg f64_type() {
    return msg(0x03, 1, {0x11, 0x20, 0x3f, 0x00, 8, 0, 0, 0, 0, 0, 64, 0, 52, 11, 0, 52, 0xff,
                         0x03, 0, 0});
}

// Variable-length string (class 9 version 1, string flag, null-terminated ASCII), 16-byte
// references, base type: 1-byte unsigned character.
Msg vlen_string_type() {
    return msg(0x03, 1, {0x19, 0x01, 0x00, 0x00, 16, 0, 0, 0, 0x10, 0x00, 0x00, 0x00, 1, 0, 0, 0,
                         0, 0, 8, 0});
}

struct Gap {
    size_t at;       // position in the metadata where the values go
    const float* f;  // float32 values widened to f64
    size_t n;
};

struct Layout {
    Bytes meta;             // the file without the gaps' bytes
    std::vector<Gap> gaps;  // in increasing position
    uint64_t skipped = 0;   // gap bytes before the end of `meta`
    uint64_t heap = 0;      // global heap collection address
    uint32_t next_string = 0;

    uint64_t pos() const { return meta.size() + skipped; }

    uint64_t header(Msg space, Msg type, uint64_t data_addr, uint64_t len) {
        uint64_t at = pos();
        Msg layout = msg(0x08, 0, {3, 1});  // layout version 3, contiguous
        layout.body.le(data_addr, 8);
        layout.body.le(len, 8);
        std::vector<Msg> msgs;
        msgs.push_back(std::move(space));
        msgs.push_back(std::move(type));
        msgs.push_back(msg(0x05, 1, {3, 2}));  // fill value version 3, fill time "if set"
        msgs.push_back(std::move(layout));
        Bytes h = object_header(msgs);
        meta.raw(h.v.data(), h.size());
        return at;
    }

    uint64_t dataset(Msg space, Msg type, const Bytes& raw) {
        meta.align8();
        uint64_t data_addr = pos();
        meta.raw(raw.v.data(), raw.size());
        meta.align8();
        return header(std::move(space), std::move(type), data_addr, raw.size());
    }

    int node(const Node& x, uint64_t* addr) {
        switch (x.kind) {
            case Node::F64: {
                Bytes raw;
                for (double v : x.d) {
                    uint64_t bits;
                    std::memcpy(&bits, &v, 8);
                    raw.le(bits, 8);
                }
                *addr = dataset(dataspace1(x.d.size()), f64_type(), raw);
                return 0;
            }
            case Node::F32Wide: {
                meta.align8();
                uint64_t data_addr = pos();
                gaps.push_back({meta.size(), x.f, x.n});
                skipped += 8 * (uint64_t)x.n;
                *addr = header(dataspace1(x.n), f64_type(), data_addr, 8 * (uint64_t)x.n);
                return 0;
            }
            case Node::Str: {
                // a global heap ID: the string's length, the collection's address, the object's
                // index (strings are numbered in the order the tree is written)
                Bytes raw;
                raw.le(x.s.size(), 4);
                raw.le(heap, 8);
                raw.le(++next_string, 4);
                *addr = dataset(dataspace1(1), vlen_string_type(), raw);
                return 0;
            }
            case Node::Group:
                return group(x.members, addr);
        }
        return fail(FW_ERR_INVALID, "hdf5: unknown node");
    }

    int group(const std::vector<Node>& members, uint64_t* addr) {
        std::vector<uint64_t> addrs(members.size());
        for (size_t i = 0; i < members.size(); ++i) FW_TRY(node(members[i], &addrs[i]));
        std::vector<Msg> msgs;
        Msg info = msg(0x02, 0, {0, 0});  // link info: no creation order, no dense storage
        info.body.le(kUndef, 8);
        info.body.le(kUndef, 8);
        msgs.push_back(std::move(info));
        msgs.push_back(msg(0x0a, 1, {0, 0}));  // group info, defaults
        for (size_t i = 0; i < members.size(); ++i) {
            const std::string& nm = members[i].name;
            if (nm.empty() || nm.size() > 0xffff)
                return fail(FW_ERR_INVALID,
                            "hdf5: bad member name length " + std::to_string(nm.size()));
            Msg link = msg(0x06, 0, {1});
            if (nm.size() <= 0xff) {
                link.body.u8(0);
                link.body.u8((unsigned)nm.size());
            } else {
                link.body.u8(1);
                link.body.le(nm.size(), 2);
            }
            link.body.str(nm);
            link.body.le(addrs[i], 8);
            msgs.push_back(std::move(link));
        }
        meta.align8();
        *addr = pos();
        Bytes h = object_header(msgs);
        meta.raw(h.v.data(), h.size());
        return 0;
    }
};

void collect_strings(const std::vector<Node>& members, std::vector<const std::string*>& out) {
    for (const Node& x : members) {
        if (x.kind == Node::Group) collect_strings(x.members, out);
        else if (x.kind == Node::Str) out.push_back(&x.s);
    }
}

int layout_file(const std::vector<Node>& root, Layout& L) {
    std::vector<const std::string*> strings;
    collect_strings(root, strings);
    L.meta.v.assign(48, 0);  // the superblock, written last
    if (!strings.empty()) {
        L.meta.align8();
        L.heap = L.meta.size();
        Bytes body;
        for (size_t i = 0; i < strings.size(); ++i) {  // heap objects 1..n, reference count 1
            body.le(i + 1, 2);
            body.le(1, 2);
            body.le(0, 4);
            body.le(strings[i]->size(), 8);
            body.str(*strings[i]);
            body.align8();
        }
        const size_t used = 16 + body.size();
        const size_t size = (std::max<size_t>(used, 4096) + 7) / 8 * 8;
        L.meta.str("GCOL");
        L.meta.u8(1);
        L.meta.le(0, 3);
        L.meta.le(size, 8);
        L.meta.raw(body.v.data(), body.size());
        if (size > used) {  // object 0: the free space up to the collection's size
            L.meta.le(0, 2);
            L.meta.le(0, 2);
            L.meta.le(0, 4);
            L.meta.le(size - used, 8);
            L.meta.v.resize(L.heap + size, 0);
        }
    }
    uint64_t root_addr = 0;
    FW_TRY(L.group(root, &root_addr));
    L.meta.align8();
    const uint64_t eof = L.pos();
    Bytes sb;
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', 0x0d, 0x0a, 0x1a, 0x0a};
    sb.raw(sig, 8);
    for (uint8_t b : {2, 8, 8, 0}) sb.u8(b);  // version 2, 8-byte offsets and lengths, no flags
    sb.le(0, 8);                               // base address
    sb.le(kUndef, 8);                          // no superblock extension
    sb.le(eof, 8);
    sb.le(root_addr, 8);
    sb.le(lookup3(sb.v.data(), sb.size(), 0), 4);
    std::memcpy(L.meta.v.data(), sb.v.data(), 48);
    return 0;
}

// Emits the file: metadata segments and the widened gap values, in blocks of 64 Ki values.
template <typename Sink>
int emit(const Layout& L, Sink&& sink) {
    size_t at = 0;
    std::vector<uint8_t> block;
    for (const Gap& g : L.gaps) {
        FW_TRY(sink(L.meta.v.data() + at, g.at - at));
        for (size_t i = 0; i < g.n; i += 65536) {
            const size_t m = std::min<size_t>(65536, g.n - i);
            block.resize(8 * m);
            for (size_t q = 0; q < m; ++q) {
                const double v = (double)g.f[i + q];
                std::memcpy(block.data() + 8 * q, &v, 8);  // little-endian host
            }
            FW_TRY(sink(block.data(), block.size()));
        }
        at = g.at;
    }
    return sink(L.meta.v.data() + at, L.meta.size() - at);
}

// ---- ITK's transform layout -----------------------------------------------------------------

const char* kAffineName = "AffineTransform_double_3_3";
const char* kFieldName = "DisplacementFieldTransform_double_3_3";
const char* kCompositeName = "CompositeTransform_double_3_3";

int check_elem(const fw_transform_elem& e, size_t* nvox) {
    if (e.kind == FW_ELEM_AFFINE) {
        for (double v : e.matrix) FW_CHECK(std::isfinite(v), "transform file: affine not finite");
        return 0;
    }
    FW_CHECK(e.kind == FW_ELEM_FIELD, "transform file: unknown element kind");
    FW_CHECK(e.field != nullptr, "transform file: null field data");
    HostGrid g;
    FW_TRY(make_grid(&e.grid, g));
    *nvox = (size_t)g.count();
    return 0;
}

// itk_params.rs:104-117 and grid.rs:158-169: type name, fixed parameters, parameters.
int elem_group(const fw_transform_elem& e, int index, Node* out) {
    size_t nvox = 0;
    FW_TRY(check_elem(e, &nvox));
    std::vector<Node> m;
    if (e.kind == FW_ELEM_AFFINE) {
        std::vector<double> p(e.matrix, e.matrix + 9);
        p.insert(p.end(), e.translation, e.translation + 3);
        m.push_back(text("TransformType", kAffineName));
        m.push_back(f64s("TransformFixedParameters", std::vector<double>(e.center, e.center + 3)));
        m.push_back(f64s("TransformParameters", std::move(p)));
    } else {
        std::vector<double> fixed(18);
        for (int a = 0; a < 3; ++a) {
            fixed[a] = (double)e.grid.size[a];
            fixed[3 + a] = e.grid.origin[a];
            fixed[6 + a] = e.grid.spacing[a];
        }
        for (int k = 0; k < 9; ++k) fixed[9 + k] = e.grid.direction[k];
        m.push_back(text("TransformType", kFieldName));
        m.push_back(f64s("TransformFixedParameters", std::move(fixed)));
        m.push_back(f32wide("TransformParameters", e.field, 3 * nvox));
    }
    *out = group(std::to_string(index), std::move(m));
    return 0;
}

int itk_h5_layout(const fw_transform_elem* chain, int32_t n, const char* os_name,
                  const char* os_version, Layout& L) {
    FW_CHECK(n >= 0 && (chain || n == 0), "null chain");
    if (n == 0) return fail(FW_ERR_INVALID, "ITK transform file: cannot write an empty chain");
    std::vector<Node> groups;
    groups.push_back(group("0", {text("TransformType", kCompositeName)}));
    for (int32_t i = 0; i < n; ++i) {
        Node g;
        FW_TRY(elem_group(chain[i], i + 1, &g));
        groups.push_back(std::move(g));
    }
    std::vector<Node> root;
    root.push_back(text("HDFVersion", "1.14.0"));
    root.push_back(text("ITKVersion", "5.4.4"));
    root.push_back(text("OSName", os_name ? os_name : "linux"));
    root.push_back(text("OSVersion", os_version ? os_version : "x86_64"));
    root.push_back(group("TransformGroup", std::move(groups)));
    return layout_file(root, L);
}

int mat_bytes(const fw_transform_elem* chain, int32_t n, Bytes& out) {
    FW_CHECK(n >= 0 && (chain || n == 0), "null chain");
    auto variable = [&](const std::string& name, const double* v, int count) {
        out.le(0, 4);  // type 0: f64, little-endian, full matrix
        out.le((uint64_t)count, 4);
        out.le(1, 4);  // one column
        out.le(0, 4);  // real
        out.le(name.size() + 1, 4);
        out.str(name);
        out.u8(0);
        for (int i = 0; i < count; ++i) {
            uint64_t bits;
            std::memcpy(&bits, &v[i], 8);
            out.le(bits, 8);
        }
    };
    for (int32_t i = 0; i < n; ++i) {
        const fw_transform_elem& e = chain[i];
        if (e.kind != FW_ELEM_AFFINE)
            return fail(FW_ERR_INVALID,
                        "ITK transform file: DisplacementFieldTransform_double_3_3 in a .mat file "
                        "is not supported");
        double p[12];
        std::memcpy(p, e.matrix, sizeof(e.matrix));
        std::memcpy(p + 9, e.translation, sizeof(e.translation));
        variable(kAffineName, p, 12);
        variable("fixed", e.center, 3);
    }
    return 0;
}

// Writes through `path`.tmp renamed to `path` once complete (fs_write.rs: write_complete).
template <typename Fill>
int write_complete(const char* path, Fill&& fill) {
    FW_CHECK(path && *path, "null path");
    const std::string tmp = std::string(path) + ".tmp";
    FILE* fh = std::fopen(tmp.c_str(), "wb");
    if (!fh) return fail(FW_ERR_INVALID, std::string("cannot open ") + tmp + " for writing");
    int rc = fill([&](const void* p, size_t n) -> int {
        if (n && std::fwrite(p, 1, n, fh) != n)
            return fail(FW_ERR_INVALID, std::string("write failed: ") + tmp);
        return 0;
    });
    if (std::fclose(fh) != 0 && !rc) rc = fail(FW_ERR_INVALID, std::string("close failed: ") + tmp);
    if (!rc && std::rename(tmp.c_str(), path) != 0)
        rc = fail(FW_ERR_INVALID, std::string("cannot rename ") + tmp + " to " + path);
    if (rc) std::remove(tmp.c_str());
    return rc;
}

int copy_out(const Bytes& b, uint8_t* out, size_t cap, size_t* len) {
    FW_CHECK(len, "null length");
    *len = b.size();
    if (out && cap >= b.size()) std::memcpy(out, b.v.data(), b.size());
    return 0;
}

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

uint32_t fw_lookup3(const uint8_t* data, size_t len) {
    return lookup3(data, data ? len : 0, 0);
}

int fw_format_itk_h5(const fw_transform_elem* chain, int32_t n, const char* os_name,
                     const char* os_version, uint8_t* out, size_t cap, size_t* len) {
    FW_CHECK(len, "null length");
    Layout L;
    FW_TRY(itk_h5_layout(chain, n, os_name, os_version, L));
    const size_t total = L.pos();
    *len = total;
    if (!out || cap < total) return 0;
    size_t at = 0;
    return emit(L, [&](const void* p, size_t k) {
        std::memcpy(out + at, p, k);
        at += k;
        return 0;
    });
}

int fw_write_itk_h5(const char* path, const fw_transform_elem* chain, int32_t n) {
    Layout L;
    FW_TRY(itk_h5_layout(chain, n, nullptr, nullptr, L));
    return write_complete(path, [&](auto&& sink) { return emit(L, sink); });
}

int fw_format_itk_mat(const fw_transform_elem* chain, int32_t n, uint8_t* out, size_t cap,
                      size_t* len) {
    Bytes b;
    FW_TRY(mat_bytes(chain, n, b));
    return copy_out(b, out, cap, len);
}

int fw_write_itk_mat(const char* path, const fw_transform_elem* chain, int32_t n) {
    Bytes b;
    FW_TRY(mat_bytes(chain, n, b));
    return write_complete(path, [&](auto&& sink) { return sink(b.v.data(), b.size()); });
}

}  // extern "C"
