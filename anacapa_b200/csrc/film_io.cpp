// Film output (Film::writeEXR / Film::writePNG, src/film/Film.cpp:154-272)
// without OpenImageIO: a scanline OpenEXR file of 32-bit float channels with
// ZIP compression (blocks of 16 scanlines, the byte reordering and delta
// predictor of the OpenEXR ZIP codec, then zlib), and an 8-bit RGB PNG with
// the reference's exposure and sRGB transfer, written to a temporary name and
// renamed into place.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/anacapa_b200.h"

namespace {

struct Out {
    std::vector<unsigned char> b;
    void u8(uint8_t v) { b.push_back(v); }
    void u32(uint32_t v) {
        for (int k = 0; k < 4; ++k) b.push_back(uint8_t(v >> (8 * k)));
    }
    void i32(int32_t v) { u32(uint32_t(v)); }
    void u64(uint64_t v) {
        for (int k = 0; k < 8; ++k) b.push_back(uint8_t(v >> (8 * k)));
    }
    void f32(float v) {
        uint32_t u;
        std::memcpy(&u, &v, 4);
        u32(u);
    }
    void str(const char* s) {
        while (*s) b.push_back(uint8_t(*s++));
        b.push_back(0);
    }
    void bytes(const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        b.insert(b.end(), c, c + n);
    }
};

// An EXR header attribute: name, type name, size, value.
void attr(Out& o, const char* name, const char* type, const Out& value) {
    o.str(name);
    o.str(type);
    o.u32(uint32_t(value.b.size()));
    o.bytes(value.b.data(), value.b.size());
}

bool write_file(const std::string& path, const std::vector<unsigned char>& data) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data.data(), 1, data.size(), f) == data.size();
    return std::fclose(f) == 0 && ok;
}

// OpenEXR's ZIP block codec: interleave the even and odd bytes, replace each
// byte by its difference to the previous one (+128, modulo 256), deflate.
// Returns false when that would not be smaller (the block is then stored).
bool zip_block(const std::vector<unsigned char>& raw, std::vector<unsigned char>& out) {
    const size_t n = raw.size();
    std::vector<unsigned char> t(n);
    size_t i1 = 0, i2 = (n + 1) / 2;
    for (size_t i = 0; i < n; ++i) t[(i & 1) ? i2++ : i1++] = raw[i];
    for (size_t i = n; i-- > 1;) t[i] = uint8_t(int(t[i]) - int(t[i - 1]) + 128);
    uLongf cap = compressBound(uLong(n));
    out.resize(cap);
    if (compress(out.data(), &cap, t.data(), uLong(n)) != Z_OK) return false;
    out.resize(cap);
    return cap < n;
}

}  // namespace

extern "C" {

int ana_image_write_exr(const char* path, uint32_t w, uint32_t h, const float* rgb, const float* albedo,
                        const float* normal) {
    if (!path || !rgb || w == 0 || h == 0) return ANA_ERR_INVALID_ARG;
    // channels in the sorted order the file stores them: B G R, then the
    // AOV layers' B G R (Film::writeEXR names: R G B, albedo.*, normals.*)
    struct Ch {
        const char* name;
        const float* src;
        int comp;
    };
    std::vector<Ch> ch = {{"B", rgb, 2}, {"G", rgb, 1}, {"R", rgb, 0}};
    if (albedo) ch.insert(ch.end(), {{"albedo.B", albedo, 2}, {"albedo.G", albedo, 1}, {"albedo.R", albedo, 0}});
    if (normal) ch.insert(ch.end(), {{"normals.B", normal, 2}, {"normals.G", normal, 1}, {"normals.R", normal, 0}});
    Out o;
    o.u32(20000630u);  // magic
    o.u32(2u);         // version 2, scanline, single part
    Out chl;
    for (const Ch& c : ch) {
        chl.str(c.name);
        chl.i32(2);  // FLOAT
        chl.u8(0);   // pLinear
        chl.u8(0);
        chl.u8(0);
        chl.u8(0);
        chl.i32(1);  // x sampling
        chl.i32(1);  // y sampling
    }
    chl.u8(0);
    attr(o, "channels", "chlist", chl);
    Out cmp;
    cmp.u8(3);  // ZIP_COMPRESSION: 16 scanlines per block
    attr(o, "compression", "compression", cmp);
    Out box;
    box.i32(0);
    box.i32(0);
    box.i32(int32_t(w) - 1);
    box.i32(int32_t(h) - 1);
    attr(o, "dataWindow", "box2i", box);
    attr(o, "displayWindow", "box2i", box);
    Out lo;
    lo.u8(0);  // INCREASING_Y
    attr(o, "lineOrder", "lineOrder", lo);
    Out par;
    par.f32(1.f);
    attr(o, "pixelAspectRatio", "float", par);
    Out swc;
    swc.f32(0.f);
    swc.f32(0.f);
    attr(o, "screenWindowCenter", "v2f", swc);
    attr(o, "screenWindowWidth", "float", par);
    o.u8(0);  // end of header
    const uint32_t kLines = 16, nBlocks = (h + kLines - 1) / kLines;
    const size_t tableAt = o.b.size();
    for (uint32_t k = 0; k < nBlocks; ++k) o.u64(0);
    std::vector<unsigned char> raw, z;
    for (uint32_t k = 0; k < nBlocks; ++k) {
        const uint32_t y0 = k * kLines, y1 = std::min(h, y0 + kLines);
        raw.clear();
        for (uint32_t y = y0; y < y1; ++y)
            for (const Ch& c : ch)
                for (uint32_t x = 0; x < w; ++x) {
                    const float v = c.src[3 * (size_t(y) * w + x) + c.comp];
                    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
                    raw.insert(raw.end(), p, p + 4);
                }
        const uint64_t at = o.b.size();
        std::memcpy(o.b.data() + tableAt + 8 * k, &at, 8);
        o.i32(int32_t(y0));
        if (zip_block(raw, z)) {
            o.u32(uint32_t(z.size()));
            o.bytes(z.data(), z.size());
        } else {
            o.u32(uint32_t(raw.size()));
            o.bytes(raw.data(), raw.size());
        }
    }
    return write_file(path, o.b) ? ANA_OK : ANA_ERR_INVALID_ARG;
}

int ana_image_write_png(const char* path, uint32_t w, uint32_t h, const float* rgb, float exposure) {
    if (!path || !rgb || w == 0 || h == 0) return ANA_ERR_INVALID_ARG;
    const float evScale = std::pow(2.f, exposure);
    auto to_srgb = [](float x) -> float {  // clamp, then the sRGB transfer
        x = std::max(0.f, std::min(1.f, x));
        if (x <= 0.0031308f) return 12.92f * x;
        return 1.055f * std::pow(x, 1.f / 2.4f) - 0.055f;
    };
    std::vector<unsigned char> scan;
    scan.reserve(size_t(h) * (3 * size_t(w) + 1));
    for (uint32_t y = 0; y < h; ++y) {
        scan.push_back(0);  // filter: none
        for (uint32_t x = 0; x < w; ++x)
            for (int k = 0; k < 3; ++k) {
                const float c = rgb[3 * (size_t(y) * w + x) + k] * evScale;
                scan.push_back(static_cast<uint8_t>(to_srgb(c) * 255.f + 0.5f));
            }
    }
    uLongf cap = compressBound(uLong(scan.size()));
    std::vector<unsigned char> z(cap);
    if (compress2(z.data(), &cap, scan.data(), uLong(scan.size()), Z_DEFAULT_COMPRESSION) != Z_OK)
        return ANA_ERR_INVALID_ARG;
    z.resize(cap);
    std::vector<unsigned char> f = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    auto chunk = [&](const char* type, const std::vector<unsigned char>& data) {
        const uint32_t n = uint32_t(data.size());
        const unsigned char len[4] = {uint8_t(n >> 24), uint8_t(n >> 16), uint8_t(n >> 8), uint8_t(n)};
        f.insert(f.end(), len, len + 4);
        const size_t at = f.size();
        f.insert(f.end(), type, type + 4);
        f.insert(f.end(), data.begin(), data.end());
        const uint32_t crc = uint32_t(crc32(0L, f.data() + at, uInt(4 + n)));
        const unsigned char c[4] = {uint8_t(crc >> 24), uint8_t(crc >> 16), uint8_t(crc >> 8), uint8_t(crc)};
        f.insert(f.end(), c, c + 4);
    };
    std::vector<unsigned char> ihdr = {uint8_t(w >> 24), uint8_t(w >> 16), uint8_t(w >> 8), uint8_t(w),
                                       uint8_t(h >> 24), uint8_t(h >> 16), uint8_t(h >> 8), uint8_t(h),
                                       8, 2, 0, 0, 0};  // 8-bit RGB
    chunk("IHDR", ihdr);
    chunk("sRGB", {0});
    chunk("IDAT", z);
    chunk("IEND", {});
    const std::string tmp = std::string(path) + ".writing.png";
    if (!write_file(tmp, f)) return ANA_ERR_INVALID_ARG;
    return std::rename(tmp.c_str(), path) == 0 ? ANA_OK : ANA_ERR_INVALID_ARG;
}

}  // extern "C"
