// PNG images for textures: the keepsake loaders read 8-bit images through stb_image (load_from_ldr,
// image_util.cpp:15-25, with a requested channel count) and glTF images through tinygltf (its
// default forces four channels and keeps 16-bit PNGs at 16 bits: create_texture_from_gltf,
// mesh_asset.cpp:370-388).  Neither library is in the reference tree; this reader follows the PNG
// specification (ISO/IEC 15948: chunk layout, zlib stream, the five scanline filters, Adam7
// interlacing, palette and tRNS transparency), and the channel conversions follow the ones stb_image
// documents for a requested channel count (grey replicated to RGB, RGB to grey as the integer
// luminance (77 R + 150 G + 29 B) >> 8, a missing alpha opaque, 16-bit samples reduced to 8 bits
// by their high byte).
#include "image_io.h"

#include <zlib.h>

#include <cstring>
#include <fstream>

namespace fs = std::filesystem;

namespace ksb
{
namespace image
{

namespace
{

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

uint8_t paeth(int a, int b, int c)
{
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc)
        return (uint8_t)a;
    return (uint8_t)(pb <= pc ? b : c);
}

// Reverses the scanline filters of one (sub-)image of `h` rows of `row_bytes` bytes (after the
// filter byte); `bpp` is the filter's byte distance (whole bytes per pixel, at least 1).
void unfilter(const uint8_t *in, size_t in_size, size_t &pos, uint8_t *out, uint32_t h, size_t row_bytes, size_t bpp,
              const std::string &where)
{
    std::vector<uint8_t> prev(row_bytes, 0);
    for (uint32_t y = 0; y < h; ++y) {
        if (pos + 1 + row_bytes > in_size)
            throw Error(where + "truncated PNG image data");
        const uint8_t type = in[pos++];
        uint8_t *row = out + (size_t)y * row_bytes;
        const uint8_t *src = in + pos;
        pos += row_bytes;
        for (size_t i = 0; i < row_bytes; ++i) {
            const int a = i >= bpp ? row[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
            int v;
            switch (type) {
            case 0: v = src[i]; break;
            case 1: v = src[i] + a; break;
            case 2: v = src[i] + b; break;
            case 3: v = src[i] + ((a + b) >> 1); break;
            case 4: v = src[i] + paeth(a, b, c); break;
            default: throw Error(where + "bad PNG filter type " + std::to_string(type));
            }
            row[i] = (uint8_t)v;
        }
        std::memcpy(prev.data(), row, row_bytes);
    }
}

} // namespace

Png read_png(const uint8_t *data, size_t size, const std::string &name)
{
    const std::string where = name + ": ";
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (size < 8 || std::memcmp(data, sig, 8) != 0)
        throw Error(where + "not a PNG file");
    size_t pos = 8;
    uint32_t w = 0, h = 0;
    int depth = 0, color = -1, interlace = 0;
    std::vector<uint8_t> idat, palette, trns;
    bool have_ihdr = false, have_iend = false;
    while (pos + 12 <= size && !have_iend) {
        const uint32_t len = be32(data + pos);
        if (len > size - pos - 12)
            throw Error(where + "truncated PNG chunk");
        const std::string type((const char *)data + pos + 4, 4);
        const uint8_t *body = data + pos + 8;
        if (type == "IHDR") {
            if (len != 13)
                throw Error(where + "bad PNG IHDR");
            w = be32(body);
            h = be32(body + 4);
            depth = body[8];
            color = body[9];
            if (body[10] != 0 || body[11] != 0)
                throw Error(where + "unknown PNG compression or filter method");
            interlace = body[12];
            have_ihdr = true;
        } else if (type == "PLTE") {
            palette.assign(body, body + len);
        } else if (type == "tRNS") {
            trns.assign(body, body + len);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), body, body + len);
        } else if (type == "IEND") {
            have_iend = true;
        } else if (type == "CgBI") {
            throw Error(where + "Apple CgBI PNG files are not supported", true);
        } else if (!(type[0] & 0x20)) {
            throw Error(where + "unknown critical PNG chunk " + type, true);
        }
        pos += 12 + (size_t)len;
    }
    if (!have_ihdr || idat.empty())
        throw Error(where + "PNG file without IHDR or image data");
    if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 28))
        throw Error(where + "bad PNG image size");
    if (interlace > 1)
        throw Error(where + "unknown PNG interlace method");
    // samples per pixel by colour type: 0 grey, 2 RGB, 3 palette, 4 grey + alpha, 6 RGBA
    int spp;
    switch (color) {
    case 0: spp = 1; break;
    case 2: spp = 3; break;
    case 3: spp = 1; break;
    case 4: spp = 2; break;
    case 6: spp = 4; break;
    default: throw Error(where + "bad PNG colour type");
    }
    const bool depth_ok = color == 0 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)
                          : color == 3 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8)
                                       : (depth == 8 || depth == 16);
    if (!depth_ok)
        throw Error(where + "bad PNG bit depth");
    if (color == 3 && (palette.empty() || palette.size() % 3 != 0 || palette.size() > 768))
        throw Error(where + "PNG palette image without a valid PLTE");

    // the zlib stream's size is fixed by the image: sum over passes of rows * (1 + row bytes)
    struct Pass
    {
        uint32_t x0, y0, dx, dy, w, h;
    };
    std::vector<Pass> passes;
    if (interlace == 0) {
        passes.push_back({0, 0, 1, 1, w, h});
    } else {
        static const uint32_t a7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                          {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
        for (const auto &p : a7) {
            const uint32_t pw = w > p[0] ? (w - p[0] + p[2] - 1) / p[2] : 0;
            const uint32_t ph = h > p[1] ? (h - p[1] + p[3] - 1) / p[3] : 0;
            passes.push_back({p[0], p[1], p[2], p[3], pw, ph});
        }
    }
    const size_t bits_pp = (size_t)spp * depth;
    size_t raw_size = 0;
    for (const Pass &p : passes)
        if (p.w && p.h)
            raw_size += (size_t)p.h * (1 + (p.w * bits_pp + 7) / 8);
    std::vector<uint8_t> raw(raw_size);
    uLongf got = (uLongf)raw_size;
    const int zs = uncompress(raw.data(), &got, idat.data(), (uLong)idat.size());
    if ((zs != Z_OK && zs != Z_BUF_ERROR) || got != raw_size)
        throw Error(where + "corrupt PNG image data");

    // samples of the full image before any palette / tRNS expansion, one uint16 per sample
    const int out_depth = depth == 16 ? 16 : 8;
    std::vector<uint16_t> samples((size_t)w * h * spp);
    size_t rpos = 0;
    const size_t bpp = std::max<size_t>(1, bits_pp / 8);
    for (const Pass &p : passes) {
        if (!p.w || !p.h)
            continue;
        const size_t row_bytes = (p.w * bits_pp + 7) / 8;
        std::vector<uint8_t> img((size_t)p.h * row_bytes);
        unfilter(raw.data(), raw.size(), rpos, img.data(), p.h, row_bytes, bpp, where);
        for (uint32_t y = 0; y < p.h; ++y) {
            const uint8_t *row = img.data() + (size_t)y * row_bytes;
            for (uint32_t x = 0; x < p.w; ++x) {
                uint16_t *dst = &samples[((size_t)(p.y0 + y * p.dy) * w + p.x0 + x * p.dx) * spp];
                for (int s = 0; s < spp; ++s) {
                    const size_t k = (size_t)x * spp + s;
                    uint16_t v;
                    if (depth == 16) {
                        v = (uint16_t)(row[2 * k] << 8 | row[2 * k + 1]);
                    } else if (depth == 8) {
                        v = row[k];
                    } else {
                        const size_t bit = k * depth;
                        v = (uint16_t)((row[bit >> 3] >> (8 - depth - (bit & 7))) & ((1 << depth) - 1));
                    }
                    dst[s] = v;
                }
            }
        }
    }

    Png out;
    out.width = (int)w;
    out.height = (int)h;
    out.depth = out_depth;
    if (color == 3) {
        // palette indices to RGB, or RGBA when tRNS gives alpha entries
        const size_t n_pal = palette.size() / 3;
        const bool alpha = !trns.empty();
        out.channels = alpha ? 4 : 3;
        out.samples.resize((size_t)w * h * out.channels);
        for (size_t i = 0; i < (size_t)w * h; ++i) {
            const size_t idx = samples[i];
            if (idx >= n_pal)
                throw Error(where + "PNG palette index out of range");
            for (int c = 0; c < 3; ++c)
                out.samples[i * out.channels + c] = palette[3 * idx + c];
            if (alpha)
                out.samples[i * 4 + 3] = idx < trns.size() ? trns[idx] : 255;
        }
        return out;
    }
    if (color == 0 && depth < 8) {
        // low bit-depth grey scaled to 8 bits (1 -> 255, 2 -> 85, 4 -> 17 per step)
        const uint16_t scale = (uint16_t)(255 / ((1 << depth) - 1));
        for (uint16_t &v : samples)
            v = (uint16_t)(v * scale);
    }
    const bool key = !trns.empty() && (color == 0 || color == 2);
    if (!key) {
        out.channels = spp;
        out.samples = std::move(samples);
        return out;
    }
    // tRNS colour key: an alpha channel, transparent where the pixel equals the key
    if ((color == 0 && trns.size() < 2) || (color == 2 && trns.size() < 6))
        throw Error(where + "bad PNG tRNS chunk");
    uint16_t keyv[3];
    for (int c = 0; c < (color == 0 ? 1 : 3); ++c) {
        uint16_t k = (uint16_t)(trns[2 * c] << 8 | trns[2 * c + 1]);
        if (color == 0 && depth < 8)
            k = (uint16_t)(k * (255 / ((1 << depth) - 1)));
        keyv[c] = k;
    }
    out.channels = spp + 1;
    out.samples.resize((size_t)w * h * out.channels);
    const uint16_t opaque = out_depth == 16 ? 0xffff : 0xff;
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        bool eq = true;
        for (int c = 0; c < spp; ++c) {
            out.samples[i * out.channels + c] = samples[i * spp + c];
            eq = eq && samples[i * spp + c] == keyv[c];
        }
        out.samples[i * out.channels + spp] = eq ? 0 : opaque;
    }
    return out;
}

Png read_png(const fs::path &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw Error(path.string() + ": cannot open");
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return read_png(bytes.data(), bytes.size(), path.string());
}

std::vector<uint16_t> convert_channels(const Png &png, int channels, int depth)
{
    const int n = png.channels;
    const size_t px = (size_t)png.width * png.height;
    const uint32_t opaque = depth == 16 ? 0xffffu : 0xffu;
    std::vector<uint16_t> out(px * channels);
    for (size_t i = 0; i < px; ++i) {
        uint32_t s[4];
        for (int c = 0; c < n; ++c) {
            uint32_t v = png.samples[i * n + c];
            if (png.depth == 16 && depth == 8)
                v >>= 8;
            s[c] = v;
        }
        const bool grey_in = n <= 2;
        const uint32_t a = (n == 2 || n == 4) ? s[n - 1] : opaque;
        const uint32_t grey = grey_in ? s[0] : (s[0] * 77 + s[1] * 150 + s[2] * 29) >> 8;
        uint16_t *d = &out[i * channels];
        switch (channels) {
        case 1: d[0] = (uint16_t)grey; break;
        case 2: d[0] = (uint16_t)grey, d[1] = (uint16_t)a; break;
        default:
            for (int c = 0; c < 3; ++c)
                d[c] = (uint16_t)(grey_in ? s[0] : s[c]);
            if (channels == 4)
                d[3] = (uint16_t)a;
        }
    }
    return out;
}

} // namespace image
} // namespace ksb
