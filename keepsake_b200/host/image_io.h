// Image files of keepsake's small_pt task: the interval images it writes
// (RenderTarget2::composite_and_save_to_exr, render_target.cpp:181-208, through save_to_exr,
// image_util.cpp:101-190) and the sky maps SkyLight reads (.exr and .hdr, light.cpp:19-31).
//
//   OpenEXR   single-part scanline files.  Written with ZIP compression (the reference's tinyexr
//             call asks for PIZ; both are lossless, so the pixels are the same), channels named
//             and ordered as save_to_exr names them (R, G, B, A sorted by name), FLOAT or HALF.
//             Read: NONE, RLE, ZIPS and ZIP compression, HALF / FLOAT / UINT channels; other
//             compressions, tiled, multi-part and deep files are reported as unsupported.
//   Radiance  .hdr (RGBE, flat or run-length scanlines, -Y H +X W orientation), converted as
//             stb_image converts it (m * 2^(e - 136)).
//   PFM       little- or big-endian RGB portable float maps (an extension of this build).
#pragma once
#include <cstdint>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

namespace ksb
{
namespace image
{

struct Error : std::runtime_error
{
    bool unsupported; // a valid file of a variant this reader does not handle
    Error(const std::string &what, bool unsupported = false) : std::runtime_error(what), unsupported(unsupported) {}
};

// `pixels`: width * height * channels floats, rows top first, channels interleaved (R, G, B[, A]).
void write_exr(const std::filesystem::path &path, const float *pixels, int width, int height, int channels,
               bool half);
// RGB, rows top first: load_from_exr's first three channels of its RGBA (one-channel files are
// grey).
std::vector<float> read_exr(const std::filesystem::path &path, int &width, int &height);
std::vector<float> read_hdr(const std::filesystem::path &path, int &width, int &height);
void write_pfm(const std::filesystem::path &path, int width, int height, const float *rgb);
std::vector<float> read_pfm(const std::filesystem::path &path, int &width, int &height);
// By extension: .exr, .hdr or .pfm.
std::vector<float> read_rgb(const std::filesystem::path &path, int &width, int &height);

// RGBA of an OpenEXR file as tinyexr's LoadEXR gives it: alpha 1 without an A channel, the one
// channel of a single-channel file in all four.
std::vector<float> read_exr_rgba(const std::filesystem::path &path, int &width, int &height);
// Float texels of a texture file (create_texture_from_image, texture.cpp:922-944): .exr through
// load_from_exr (the first `channels` of the RGBA), .hdr (and .pfm) through stb_image's float
// loader's channel conversion.
std::vector<float> read_float_texture(const std::filesystem::path &path, int channels, int &width, int &height);

// PNG (8- or 16-bit samples, all colour types, Adam7): samples row-major, top row first, channels
// interleaved; palette images expanded to RGB (RGBA with a tRNS chunk), grey / RGB with a tRNS
// colour key given an alpha channel, 1-, 2- and 4-bit grey scaled to 8 bits.
struct Png
{
    int width = 0, height = 0, channels = 0, depth = 8; // depth 8 or 16
    std::vector<uint16_t> samples;
};
Png read_png(const uint8_t *data, size_t size, const std::string &name);
Png read_png(const std::filesystem::path &path);
// The samples converted to `channels` (1-4) at `depth` (8 or 16; 16-bit samples reduced to 8 by
// their high byte), as stb_image converts for a requested channel count.
std::vector<uint16_t> convert_channels(const Png &png, int channels, int depth);

// IEEE binary16 conversions (round to nearest even; exact widening).
uint16_t float_to_half(float f);
float half_to_float(uint16_t h);

} // namespace image
} // namespace ksb
