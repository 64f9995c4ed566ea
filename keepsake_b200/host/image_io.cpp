// Image files of the small_pt task: OpenEXR (scanline; written ZIP-compressed), Radiance .hdr and
// PFM.  The OpenEXR layout follows the format's published file layout (magic and version,
// attribute header, chunk offset table, per-chunk scanline blocks, the ZIP and RLE codecs with
// their byte interleave and delta predictor); the Radiance reader follows the RGBE format with
// its run-length scanlines.
#include "image_io.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>

namespace fs = std::filesystem;

namespace ksb
{
namespace image
{

uint16_t float_to_half(float f)
{
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) // inf, nan (keeps the top payload bits, quiet)
        return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u | ((ax >> 13) & 0x3ffu) : 0u));
    if (ax >= 0x477ff000u) // at or above 65520: rounds past the largest half (65504)
        return (uint16_t)(sign | 0x7c00u);
    if (ax < 0x38800000u) { // below 2^-14: a subnormal half (or zero)
        if (ax <= 0x33000000u) // at most 2^-25: rounds to zero (2^-25 is a tie, zero is even)
            return (uint16_t)sign;
        const int e = (int)(ax >> 23);
        const uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        const int shift = 126 - e; // value / 2^-24 = m * 2^(e - 126)
        uint32_t q = m >> shift;
        const uint32_t rem = m & ((1u << shift) - 1u), half_way = 1u << (shift - 1);
        if (rem > half_way || (rem == half_way && (q & 1u)))
            ++q;
        return (uint16_t)(sign | q);
    }
    uint32_t h = ((((ax >> 23) - 127u + 15u)) << 10) | ((ax & 0x7fffffu) >> 13);
    const uint32_t rem = ax & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u)))
        ++h; // a carry moves into the exponent, as it should
    return (uint16_t)(sign | h);
}

float half_to_float(uint16_t h)
{
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t x;
    if (e == 0) {
        const float v = std::ldexp((float)m, -24);
        std::memcpy(&x, &v, 4);
        x |= sign;
    } else if (e == 31) {
        x = sign | 0x7f800000u | (m << 13);
    } else {
        x = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

namespace
{

std::vector<uint8_t> read_file(const fs::path &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot open " + path.string());
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void write_file(const fs::path &path, const std::vector<uint8_t> &bytes)
{
    std::ofstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot write " + path.string());
    f.write(reinterpret_cast<const char *>(bytes.data()), (std::streamsize)bytes.size());
    if (!f)
        throw Error("cannot write " + path.string());
}

template <class T>
void put(std::vector<uint8_t> &out, T v)
{
    uint8_t b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T)); // little-endian host
    out.insert(out.end(), b, b + sizeof(T));
}

void put_str(std::vector<uint8_t> &out, const std::string &s)
{
    out.insert(out.end(), s.begin(), s.end());
    out.push_back(0);
}

void attribute(std::vector<uint8_t> &out, const std::string &name, const std::string &type,
               const std::vector<uint8_t> &value)
{
    put_str(out, name);
    put_str(out, type);
    put<int32_t>(out, (int32_t)value.size());
    out.insert(out.end(), value.begin(), value.end());
}

// EXR compression codes and the scanlines one chunk holds
enum : int
{
    kNone = 0,
    kRle = 1,
    kZips = 2,
    kZip = 3,
    kPiz = 4
};

int lines_per_chunk(int compression)
{
    switch (compression) {
    case kNone:
    case kRle:
    case kZips:
        return 1;
    case kZip:
        return 16;
    default:
        return 0;
    }
}

// The ZIP and RLE codecs store the block's bytes split into even and odd positions, then as
// differences of consecutive bytes (offset by 128).
std::vector<uint8_t> interleave_predict(const std::vector<uint8_t> &raw)
{
    const size_t n = raw.size();
    std::vector<uint8_t> t(n);
    size_t a = 0, b = (n + 1) / 2;
    for (size_t i = 0; i < n; ++i)
        t[(i & 1) ? b++ : a++] = raw[i];
    int prev = n ? t[0] : 0;
    for (size_t i = 1; i < n; ++i) {
        const int cur = t[i];
        t[i] = (uint8_t)(cur - prev + 128 + 256);
        prev = cur;
    }
    return t;
}

std::vector<uint8_t> unpredict_deinterleave(std::vector<uint8_t> t)
{
    const size_t n = t.size();
    for (size_t i = 1; i < n; ++i)
        t[i] = (uint8_t)((int)t[i - 1] + (int)t[i] - 128);
    std::vector<uint8_t> raw(n);
    size_t a = 0, b = (n + 1) / 2;
    for (size_t i = 0; i < n; ++i)
        raw[i] = t[(i & 1) ? b++ : a++];
    return raw;
}

std::vector<uint8_t> rle_decode(const uint8_t *p, size_t size, size_t expect)
{
    std::vector<uint8_t> out;
    out.reserve(expect);
    size_t i = 0;
    while (i < size) {
        const int count = (int8_t)p[i++];
        if (count < 0) {
            const size_t n = (size_t)(-count);
            if (i + n > size || out.size() + n > expect)
                throw Error("EXR: corrupt RLE block");
            out.insert(out.end(), p + i, p + i + n);
            i += n;
        } else {
            const size_t n = (size_t)count + 1;
            if (i >= size || out.size() + n > expect)
                throw Error("EXR: corrupt RLE block");
            out.insert(out.end(), n, p[i++]);
        }
    }
    if (out.size() != expect)
        throw Error("EXR: RLE block of the wrong size");
    return out;
}

struct Channel
{
    std::string name;
    int type; // 0 UINT, 1 HALF, 2 FLOAT
    int bytes() const { return type == 1 ? 2 : 4; }
};

} // namespace

void write_exr(const fs::path &path, const float *pixels, int w, int h, int c, bool half)
{
    if (!pixels || w <= 0 || h <= 0 || c < 1 || c > 4)
        throw Error("write_exr: bad image size or channel count");
    // channels sorted by name; save_to_exr names them A, B, G, R (4), B, G, R (3), G, R (2), R (1)
    static const char *kNames[4] = {"R", "G", "B", "A"};
    const int vb = half ? 2 : 4;
    std::vector<uint8_t> out = {0x76, 0x2f, 0x31, 0x01};
    put<int32_t>(out, 2); // version 2, single-part scanline
    std::vector<uint8_t> chl;
    for (int k = 0; k < c; ++k) {
        put_str(chl, kNames[c - 1 - k]);
        put<int32_t>(chl, half ? 1 : 2);
        put<uint8_t>(chl, 0); // pLinear
        chl.insert(chl.end(), 3, 0);
        put<int32_t>(chl, 1);
        put<int32_t>(chl, 1);
    }
    chl.push_back(0);
    attribute(out, "channels", "chlist", chl);
    attribute(out, "compression", "compression", {(uint8_t)kZip});
    std::vector<uint8_t> box;
    for (int32_t v : {0, 0, w - 1, h - 1})
        put<int32_t>(box, v);
    attribute(out, "dataWindow", "box2i", box);
    attribute(out, "displayWindow", "box2i", box);
    attribute(out, "lineOrder", "lineOrder", {0});
    std::vector<uint8_t> one, center;
    put<float>(one, 1.0f);
    put<float>(center, 0.0f);
    put<float>(center, 0.0f);
    attribute(out, "pixelAspectRatio", "float", one);
    attribute(out, "screenWindowCenter", "v2f", center);
    attribute(out, "screenWindowWidth", "float", one);
    out.push_back(0); // end of header
    const int lpc = lines_per_chunk(kZip);
    const int n_chunks = (h + lpc - 1) / lpc;
    const size_t table = out.size();
    out.resize(table + 8 * (size_t)n_chunks);
    for (int ch = 0; ch < n_chunks; ++ch) {
        const int y0 = ch * lpc, y1 = std::min(h, y0 + lpc);
        std::vector<uint8_t> raw;
        raw.reserve((size_t)(y1 - y0) * w * c * vb);
        for (int y = y0; y < y1; ++y)
            for (int k = 0; k < c; ++k)
                for (int x = 0; x < w; ++x) {
                    const float v = pixels[((size_t)y * w + x) * c + (c - 1 - k)];
                    if (half)
                        put<uint16_t>(raw, float_to_half(v));
                    else
                        put<float>(raw, v);
                }
        const std::vector<uint8_t> pre = interleave_predict(raw);
        uLongf zsize = compressBound((uLong)pre.size());
        std::vector<uint8_t> z(zsize);
        if (compress(z.data(), &zsize, pre.data(), (uLong)pre.size()) != Z_OK)
            throw Error("write_exr: zlib failed");
        const uint64_t offset = out.size();
        std::memcpy(&out[table + 8 * (size_t)ch], &offset, 8);
        put<int32_t>(out, y0);
        if (zsize < raw.size()) {
            put<int32_t>(out, (int32_t)zsize);
            out.insert(out.end(), z.begin(), z.begin() + zsize);
        } else { // incompressible: the raw block
            put<int32_t>(out, (int32_t)raw.size());
            out.insert(out.end(), raw.begin(), raw.end());
        }
    }
    write_file(path, out);
}

// RGBA as tinyexr's LoadEXR returns it: R, G, B and A (1 without an A channel); a file of one
// channel gives that channel in all four.
std::vector<float> read_exr_rgba(const fs::path &path, int &width, int &height)
{
    const std::vector<uint8_t> f = read_file(path);
    const std::string where = path.string() + ": ";
    size_t pos = 0;
    auto need = [&](size_t n) {
        if (pos + n > f.size())
            throw Error(where + "truncated EXR file");
    };
    auto get32 = [&]() {
        need(4);
        int32_t v;
        std::memcpy(&v, &f[pos], 4);
        pos += 4;
        return v;
    };
    auto get_str = [&]() {
        const size_t end = std::find(f.begin() + (long)pos, f.end(), (uint8_t)0) - f.begin();
        if (end >= f.size())
            throw Error(where + "truncated EXR header");
        std::string s(f.begin() + (long)pos, f.begin() + (long)end);
        pos = end + 1;
        return s;
    };
    need(8);
    if (!(f[0] == 0x76 && f[1] == 0x2f && f[2] == 0x31 && f[3] == 0x01))
        throw Error(where + "not an OpenEXR file");
    pos = 4;
    const int32_t version = get32();
    if ((version & 0xff) != 2)
        throw Error(where + "unknown OpenEXR version", true);
    if (version & (0x200 | 0x800 | 0x1000))
        throw Error(where + "tiled, deep or multi-part OpenEXR files are not supported", true);
    std::vector<Channel> chans;
    int compression = -1;
    int32_t win[4] = {0, 0, -1, -1};
    bool have_win = false;
    for (;;) {
        const std::string name = get_str();
        if (name.empty())
            break;
        const std::string type = get_str();
        const int32_t size = get32();
        if (size < 0)
            throw Error(where + "bad EXR attribute size");
        need((size_t)size);
        const size_t vend = pos + (size_t)size;
        if (name == "channels" && type == "chlist") {
            while (pos < vend && f[pos] != 0) {
                Channel c;
                c.name = get_str();
                c.type = get32();
                pos += 4; // pLinear + reserved
                const int32_t xs = get32(), ys = get32();
                if (c.type < 0 || c.type > 2)
                    throw Error(where + "unknown EXR channel type");
                if (xs != 1 || ys != 1)
                    throw Error(where + "sub-sampled EXR channels are not supported", true);
                chans.push_back(c);
            }
        } else if (name == "compression" && size == 1) {
            compression = f[pos];
        } else if (name == "dataWindow" && size == 16) {
            for (int k = 0; k < 4; ++k)
                std::memcpy(&win[k], &f[pos + 4 * k], 4);
            have_win = true;
        }
        pos = vend;
    }
    if (chans.empty() || !have_win || compression < 0)
        throw Error(where + "EXR header without channels, dataWindow or compression");
    const int lpc = lines_per_chunk(compression);
    if (lpc == 0)
        throw Error(where + "EXR compression " + std::to_string(compression) +
                        " is not supported (NONE, RLE, ZIPS and ZIP are)",
                    true);
    const int64_t w = (int64_t)win[2] - win[0] + 1, h = (int64_t)win[3] - win[1] + 1;
    if (w <= 0 || h <= 0 || w * h > (1ll << 31))
        throw Error(where + "bad EXR data window");
    int ri = -1, gi = -1, bi = -1, yi = -1, ai = -1;
    size_t line_bytes = 0;
    for (size_t k = 0; k < chans.size(); ++k) {
        const std::string &n = chans[k].name;
        if (n == "R")
            ri = (int)k;
        else if (n == "G")
            gi = (int)k;
        else if (n == "B")
            bi = (int)k;
        else if (n == "Y")
            yi = (int)k;
        else if (n == "A")
            ai = (int)k;
        line_bytes += (size_t)w * chans[k].bytes();
    }
    if (!(ri >= 0 && gi >= 0 && bi >= 0)) {
        if (yi < 0 && chans.size() == 1)
            yi = 0;
        if (chans.size() == 1)
            ai = yi;
        if (yi < 0)
            throw Error(where + "EXR file without R, G, B (or a single) channel", true);
        ri = gi = bi = yi;
    }
    const int64_t n_chunks = (h + lpc - 1) / lpc;
    need(8 * (size_t)n_chunks);
    std::vector<uint64_t> offsets((size_t)n_chunks);
    std::memcpy(offsets.data(), &f[pos], 8 * (size_t)n_chunks);
    std::vector<float> rgba((size_t)(w * h * 4), 0.0f);
    std::vector<float> line((size_t)w * chans.size());
    for (int64_t ch = 0; ch < n_chunks; ++ch) {
        pos = (size_t)offsets[(size_t)ch];
        if (offsets[(size_t)ch] > f.size())
            throw Error(where + "EXR chunk offset out of range");
        const int64_t y0 = (int64_t)get32() - win[1];
        const int32_t size = get32();
        if (y0 < 0 || y0 >= h || size < 0)
            throw Error(where + "bad EXR chunk");
        need((size_t)size);
        const int64_t lines = std::min<int64_t>(lpc, h - y0);
        const size_t expect = (size_t)lines * line_bytes;
        std::vector<uint8_t> raw;
        if ((size_t)size == expect) {
            raw.assign(f.begin() + (long)pos, f.begin() + (long)pos + size);
        } else if (compression == kZip || compression == kZips) {
            std::vector<uint8_t> t(expect);
            uLongf got = (uLongf)expect;
            if (uncompress(t.data(), &got, &f[pos], (uLong)size) != Z_OK || got != expect)
                throw Error(where + "corrupt EXR ZIP block");
            raw = unpredict_deinterleave(std::move(t));
        } else if (compression == kRle) {
            raw = unpredict_deinterleave(rle_decode(&f[pos], (size_t)size, expect));
        } else {
            throw Error(where + "EXR block of the wrong size");
        }
        size_t q = 0;
        for (int64_t l = 0; l < lines; ++l) {
            for (size_t k = 0; k < chans.size(); ++k)
                for (int64_t x = 0; x < w; ++x) {
                    float v;
                    if (chans[k].type == 1) {
                        uint16_t hv;
                        std::memcpy(&hv, &raw[q], 2);
                        v = half_to_float(hv);
                    } else if (chans[k].type == 2) {
                        std::memcpy(&v, &raw[q], 4);
                    } else {
                        uint32_t u;
                        std::memcpy(&u, &raw[q], 4);
                        v = (float)u;
                    }
                    q += (size_t)chans[k].bytes();
                    line[k * (size_t)w + (size_t)x] = v;
                }
            float *row = &rgba[(size_t)((y0 + l) * w * 4)];
            for (int64_t x = 0; x < w; ++x) {
                row[4 * x] = line[(size_t)ri * w + x];
                row[4 * x + 1] = line[(size_t)gi * w + x];
                row[4 * x + 2] = line[(size_t)bi * w + x];
                row[4 * x + 3] = ai >= 0 ? line[(size_t)ai * w + x] : 1.0f;
            }
        }
    }
    width = (int)w;
    height = (int)h;
    return rgba;
}

std::vector<float> read_exr(const fs::path &path, int &width, int &height)
{
    const std::vector<float> rgba = read_exr_rgba(path, width, height);
    std::vector<float> rgb((size_t)width * height * 3);
    for (size_t i = 0; i < (size_t)width * height; ++i)
        for (int c = 0; c < 3; ++c)
            rgb[3 * i + c] = rgba[4 * i + c];
    return rgb;
}

std::vector<float> read_hdr(const fs::path &path, int &width, int &height)
{
    const std::vector<uint8_t> f = read_file(path);
    const std::string where = path.string() + ": ";
    size_t pos = 0;
    auto line = [&]() {
        const size_t end = std::find(f.begin() + (long)pos, f.end(), (uint8_t)'\n') - f.begin();
        if (end >= f.size())
            throw Error(where + "truncated Radiance header");
        std::string s(f.begin() + (long)pos, f.begin() + (long)end);
        pos = end + 1;
        return s;
    };
    const std::string magic = line();
    if (magic != "#?RADIANCE" && magic != "#?RGBE")
        throw Error(where + "not a Radiance .hdr file");
    bool rgbe = false;
    for (;;) {
        const std::string l = line();
        if (l.empty())
            break;
        if (l.rfind("FORMAT=", 0) == 0) {
            if (l != "FORMAT=32-bit_rle_rgbe")
                throw Error(where + "only the 32-bit_rle_rgbe format is supported", true);
            rgbe = true;
        }
    }
    (void)rgbe; // files without a FORMAT line are RGBE too
    const std::string res = line();
    int w = 0, h = 0;
    char ya[3] = {0}, xa[3] = {0};
    if (std::sscanf(res.c_str(), "%2s %d %2s %d", ya, &h, xa, &w) != 4 || std::string(ya) != "-Y" ||
        std::string(xa) != "+X")
        throw Error(where + "only the -Y H +X W orientation is supported", true);
    if (w <= 0 || h <= 0 || (int64_t)w * h > (1ll << 30))
        throw Error(where + "bad Radiance image size");
    std::vector<float> rgb((size_t)w * h * 3);
    std::vector<uint8_t> scan((size_t)w * 4);
    auto need = [&](size_t n) {
        if (pos + n > f.size())
            throw Error(where + "truncated Radiance data");
    };
    for (int y = 0; y < h; ++y) {
        need(4);
        const bool rle = w >= 8 && w < 0x8000 && f[pos] == 2 && f[pos + 1] == 2 && ((f[pos + 2] << 8) | f[pos + 3]) == w;
        if (!rle) {
            need((size_t)w * 4); // flat scanline
            std::memcpy(scan.data(), &f[pos], (size_t)w * 4);
            pos += (size_t)w * 4;
        } else {
            pos += 4;
            for (int c = 0; c < 4; ++c) { // the four components, one run-length stream each
                int x = 0;
                while (x < w) {
                    need(1);
                    int n = f[pos++];
                    if (n > 128) {
                        n -= 128;
                        need(1);
                        if (x + n > w)
                            throw Error(where + "corrupt Radiance scanline");
                        const uint8_t v = f[pos++];
                        for (int k = 0; k < n; ++k)
                            scan[4 * (size_t)(x++) + c] = v;
                    } else {
                        if (n == 0 || x + n > w)
                            throw Error(where + "corrupt Radiance scanline");
                        need((size_t)n);
                        for (int k = 0; k < n; ++k)
                            scan[4 * (size_t)(x++) + c] = f[pos++];
                    }
                }
            }
        }
        for (int x = 0; x < w; ++x) {
            const uint8_t *p = &scan[4 * (size_t)x];
            float *o = &rgb[((size_t)y * w + x) * 3];
            if (p[3] == 0) {
                o[0] = o[1] = o[2] = 0.0f;
            } else {
                const float s = std::ldexp(1.0f, (int)p[3] - (128 + 8));
                o[0] = p[0] * s;
                o[1] = p[1] * s;
                o[2] = p[2] * s;
            }
        }
    }
    width = w;
    height = h;
    return rgb;
}

// Portable float map: little-endian RGB, bottom row first.
void write_pfm(const fs::path &path, int w, int h, const float *rgb)
{
    std::ofstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot write " + path.string());
    f << "PF\n" << w << " " << h << "\n-1.0\n";
    for (int y = h - 1; y >= 0; --y)
        f.write(reinterpret_cast<const char *>(rgb + (size_t)y * w * 3), (std::streamsize)(sizeof(float) * 3 * w));
    if (!f)
        throw Error("cannot write " + path.string());
}

std::vector<float> read_pfm(const fs::path &path, int &w, int &h)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot open " + path.string());
    std::string magic;
    double scale;
    f >> magic >> w >> h >> scale;
    f.get();
    if (magic != "PF" || !f || w <= 0 || h <= 0 || (int64_t)w * h > (1ll << 30))
        throw Error(path.string() + ": not an RGB PFM file");
    std::vector<float> top_first((size_t)w * h * 3), rows((size_t)w * h * 3);
    f.read(reinterpret_cast<char *>(rows.data()), (std::streamsize)(sizeof(float) * rows.size()));
    if (!f)
        throw Error(path.string() + ": truncated");
    if (scale > 0.0)
        for (float &v : rows) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            u = __builtin_bswap32(u);
            std::memcpy(&v, &u, 4);
        }
    for (int y = 0; y < h; ++y)
        std::memcpy(&top_first[(size_t)y * w * 3], &rows[(size_t)(h - 1 - y) * w * 3], sizeof(float) * 3 * w);
    return top_first;
}

std::vector<float> read_float_texture(const fs::path &path, int channels, int &w, int &h)
{
    if (channels < 1 || channels > 4)
        throw Error(path.string() + ": a texture has 1 to 4 channels");
    const std::string ext = path.extension().string();
    std::vector<float> out;
    if (ext == ".exr") {
        // load_from_exr (image_util.cpp:71-100): the first `channels` of LoadEXR's RGBA
        const std::vector<float> rgba = read_exr_rgba(path, w, h);
        out.resize((size_t)w * h * channels);
        for (size_t i = 0; i < (size_t)w * h; ++i)
            for (int c = 0; c < channels; ++c)
                out[i * channels + c] = rgba[4 * i + c];
        return out;
    }
    // load_from_hdr (image_util.cpp:54-63): stb_image's float loader with a requested channel
    // count converts RGB to one or two channels as the mean of R, G and B (then alpha 1), and to
    // four with alpha 1
    const std::vector<float> rgb = ext == ".hdr" ? read_hdr(path, w, h) : ext == ".pfm" ? read_pfm(path, w, h)
                                  : throw Error(path.string() + ": float textures are read from .exr, .hdr or .pfm "
                                                                "files",
                                                true);
    out.resize((size_t)w * h * channels);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        const float *p = &rgb[3 * i];
        float *o = &out[i * channels];
        if (channels <= 2) {
            o[0] = (p[0] + p[1] + p[2]) / 3.0f;
            if (channels == 2)
                o[1] = 1.0f;
        } else {
            o[0] = p[0], o[1] = p[1], o[2] = p[2];
            if (channels == 4)
                o[3] = 1.0f;
        }
    }
    return out;
}

std::vector<float> read_rgb(const fs::path &path, int &w, int &h)
{
    const std::string ext = path.extension().string();
    if (ext == ".exr")
        return read_exr(path, w, h);
    if (ext == ".hdr")
        return read_hdr(path, w, h);
    if (ext == ".pfm")
        return read_pfm(path, w, h);
    throw Error(path.string() + ": images are read from .exr, .hdr or .pfm files", true);
}

} // namespace image
} // namespace ksb
