// bgeo.cpp — Houdini binary geometry (BGEO version 5) particle files, the format the reference reads
// and writes through partio (Utilities/PartioReaderWriter.cpp:8-66 reading, :189-231 writing; the
// byte layout is partio's readBGEO / writeBGEO, extern/partio/src/lib/io/BGEO.cpp).
//
// Layout (big-endian): "Bgeo" magic, 'V', version 5, point / primitive / group / attribute counts;
// one definition per point attribute besides position (name, component count, Houdini type,
// default values); then per point: x y z w(=1) followed by the attribute values in definition
// order, 4 bytes per component; a writer appends the one particle primitive that lists every point
// (partio's "generator" = "papi" primitive attribute, tag 0x8000) and the end bytes 0x00 0xff.
// Files are gzip-compressed when written; the reader accepts compressed and plain files.
//
// Host code only; the library's C entry points (dfsph_bgeo_read, dfsph_bgeo_write,
// dfsph_export_bgeo) are thin wrappers over these functions.
#include "bgeo.h"

#include <zlib.h>

#include <cstring>
#include <memory>

namespace dfsph {
namespace {

constexpr int32_t kMagic = ('B' << 24) | ('g' << 16) | ('e' << 8) | 'o';
constexpr int32_t kHoudiniFloat = 0, kHoudiniInt = 1, kHoudiniString = 2, kHoudiniIndexed = 4,
                  kHoudiniVector = 5;

struct GzCloser {
    void operator()(gzFile_s* f) const {
        if (f) gzclose(f);
    }
};
using Gz = std::unique_ptr<gzFile_s, GzCloser>;

// Big-endian output into a byte buffer; the whole file is assembled and then deflated in one write.
struct Out {
    std::vector<uint8_t> b;
    void u8(uint8_t v) { b.push_back(v); }
    void u16(uint16_t v) {
        u8(uint8_t(v >> 8));
        u8(uint8_t(v));
    }
    void u32(uint32_t v) {
        u16(uint16_t(v >> 16));
        u16(uint16_t(v));
    }
    void f32(float v) {
        uint32_t u;
        std::memcpy(&u, &v, 4);
        u32(u);
    }
    void str(const char* s) {  // Houdini string: 16-bit length, bytes, no terminator
        const size_t n = std::strlen(s);
        u16(uint16_t(n));
        b.insert(b.end(), s, s + n);
    }
};

struct In {
    gzFile_s* f;
    bool ok = true;
    bool read(void* p, size_t n) {
        if (!ok) return false;
        size_t got = 0;
        while (got < n) {
            const unsigned chunk = (unsigned)std::min<size_t>(n - got, 1u << 30);
            const int r = gzread(f, (char*)p + got, chunk);
            if (r <= 0) return ok = false;
            got += (size_t)r;
        }
        return true;
    }
    uint16_t u16() {
        uint8_t c[2] = {0, 0};
        read(c, 2);
        return uint16_t((c[0] << 8) | c[1]);
    }
    uint32_t u32() {
        uint8_t c[4] = {0, 0, 0, 0};
        read(c, 4);
        return (uint32_t(c[0]) << 24) | (uint32_t(c[1]) << 16) | (uint32_t(c[2]) << 8) | uint32_t(c[3]);
    }
    std::string str() {
        const uint16_t n = u16();
        std::string s(n, '\0');
        if (n) read(&s[0], n);
        return s;
    }
};

inline float be_float(const uint8_t* p) {
    const uint32_t u = (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]);
    float v;
    std::memcpy(&v, &u, 4);
    return v;
}

}  // namespace

bool bgeo_write(const std::string& path, uint64_t n, const float* xyz, const float* vxyz, float radius,
                std::string& err) {
    if (n > (uint64_t)INT32_MAX) {
        err = "bgeo: more than 2^31-1 particles";
        return false;
    }
    if (n && !xyz) {
        err = "bgeo: null positions";
        return false;
    }
    const bool has_scale = radius != 0.0f;
    Out o;
    o.b.reserve(64 + (size_t)n * (16 + (vxyz ? 12 : 0) + (has_scale ? 4 : 0) + 4 + 4) + 64);
    o.u32((uint32_t)kMagic);
    o.u8('V');
    o.u32(5);                                                 // version
    o.u32((uint32_t)n);                                       // points
    o.u32(1);                                                 // primitives: the particle system
    o.u32(0);                                                 // point groups
    o.u32(0);                                                 // primitive groups
    o.u32(1u + (vxyz ? 1u : 0u) + (has_scale ? 1u : 0u));     // point attributes besides position
    o.u32(0);                                                 // vertex attributes
    o.u32(1);                                                 // primitive attributes
    o.u32(0);                                                 // detail attributes
    auto attr = [&](const char* name, uint16_t size, int32_t type) {
        o.str(name);
        o.u16(size);
        o.u32((uint32_t)type);
        for (uint16_t k = 0; k < size; ++k) o.u32(0);         // default value 0
    };
    if (vxyz) attr("velocity", 3, kHoudiniVector);
    if (has_scale) attr("pscale", 1, kHoudiniFloat);
    attr("id", 1, kHoudiniInt);
    for (uint64_t i = 0; i < n; ++i) {
        o.f32(xyz[3 * i]);
        o.f32(xyz[3 * i + 1]);
        o.f32(xyz[3 * i + 2]);
        o.f32(1.0f);  // homogeneous w
        if (vxyz) {
            o.f32(vxyz[3 * i]);
            o.f32(vxyz[3 * i + 1]);
            o.f32(vxyz[3 * i + 2]);
        }
        if (has_scale) o.f32(radius);
        o.u32((uint32_t)i);
    }
    // the primitive attribute "generator" (one indexed string, "papi") and the particle primitive
    o.str("generator");
    o.u16(1);
    o.u32((uint32_t)kHoudiniIndexed);
    o.u32(1);
    o.str("papi");
    o.u32(0x8000);
    o.u32((uint32_t)n);
    for (uint64_t i = 0; i < n; ++i) {
        if (n > (1u << 16))
            o.u32((uint32_t)i);
        else
            o.u16((uint16_t)i);
    }
    o.u32(0);  // value of the primitive attribute (index of "papi")
    o.u8(0x00);
    o.u8(0xff);

    Gz f(gzopen(path.c_str(), "wb"));
    if (!f) {
        err = "cannot open " + path + " for writing";
        return false;
    }
    size_t done = 0;
    while (done < o.b.size()) {
        const unsigned chunk = (unsigned)std::min<size_t>(o.b.size() - done, 1u << 30);
        if (gzwrite(f.get(), o.b.data() + done, chunk) != (int)chunk) {
            err = "write failed: " + path;
            return false;
        }
        done += chunk;
    }
    if (gzclose(f.release()) != Z_OK) {
        err = "write failed: " + path;
        return false;
    }
    return true;
}

bool bgeo_read(const std::string& path, std::vector<float>& xyz, std::vector<float>& vxyz, bool& has_velocity,
               std::string& err) {
    Gz f(gzopen(path.c_str(), "rb"));
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    In in{f.get()};
    const uint32_t magic = in.u32();
    uint8_t vchar = 0;
    in.read(&vchar, 1);
    const uint32_t version = in.u32();
    const uint32_t n_points = in.u32();
    in.u32();  // primitives
    in.u32();  // point groups
    in.u32();  // primitive groups
    const uint32_t n_point_attr = in.u32();
    in.u32();  // vertex attributes
    in.u32();  // primitive attributes
    in.u32();  // detail attributes
    if (!in.ok || magic != (uint32_t)kMagic) {
        err = path + ": not a bgeo file";
        return false;
    }
    if (version != 5) {
        err = path + ": bgeo version " + std::to_string(version) + " (only version 5 is read)";
        return false;
    }
    if (n_points > (uint32_t)INT32_MAX) {
        err = path + ": bad point count";
        return false;
    }
    // Per-point record: 4 words of position, then each attribute's components.
    size_t words = 4;
    long vel_offset = -1;
    for (uint32_t a = 0; a < n_point_attr && in.ok; ++a) {
        const std::string name = in.str();
        const uint16_t size = in.u16();
        const int32_t type = (int32_t)in.u32();
        if (type == kHoudiniFloat || type == kHoudiniInt || type == kHoudiniVector) {
            for (uint16_t k = 0; k < size; ++k) in.u32();  // defaults
        } else if (type == kHoudiniIndexed) {
            const uint32_t n_strings = in.u32();
            for (uint32_t k = 0; k < n_strings && in.ok; ++k) in.str();
        } else if (type == kHoudiniString) {
            err = path + ": attribute '" + name + "' has the unsupported type 'string'";
            return false;
        } else {
            err = path + ": attribute '" + name + "' has the unknown type " + std::to_string(type);
            return false;
        }
        if (name == "velocity" && size >= 3 && vel_offset < 0) vel_offset = (long)words;
        words += size;
    }
    if (!in.ok) {
        err = path + ": truncated header";
        return false;
    }
    has_velocity = vel_offset >= 0;
    xyz.assign((size_t)n_points * 3, 0.0f);
    vxyz.assign((size_t)n_points * 3, 0.0f);
    std::vector<uint8_t> rec(words * 4);
    for (uint32_t i = 0; i < n_points; ++i) {
        if (!in.read(rec.data(), rec.size())) {
            err = path + ": truncated point data";
            return false;
        }
        for (int c = 0; c < 3; ++c) xyz[3 * (size_t)i + c] = be_float(&rec[4 * c]);
        if (has_velocity)
            for (int c = 0; c < 3; ++c) vxyz[3 * (size_t)i + c] = be_float(&rec[4 * (vel_offset + c)]);
    }
    return true;
}

}  // namespace dfsph
