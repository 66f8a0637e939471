// Image files: Radiance .hdr (RGBE, flat and run-length scanlines) and 8-bit PNG.
//
// Decoding follows what the reference's Image::load_from_file produces
// (src/engine/src/image/image.cpp:129-147): HDR texels are RGBE-decoded as
// byte * 2^(e - 136) (the stb reader's rule); 8-bit images are byte / 255 followed by
// SrgbToLinear (core/utils.h:120-125).  Writing mirrors Image::save_to_file
// (image.cpp:81-109): PNG bytes are round(255 * clamp(c, 0, 1)).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace fmhost {

struct ImageF {
    int width = 0, height = 0;
    std::vector<float> rgb;   // width*height*3, row 0 = top
};

// Reads .hdr (when `is_hdr`) or PNG.  Throws std::runtime_error on failure.
ImageF read_image(const std::string& path, bool is_hdr);
void write_png(const std::string& path, int w, int h, const float* rgb);
// 8-bit RGB PNG of already quantized values (row-major, top row first).
void write_png_u8(const std::string& path, int w, int h, const uint8_t* rgb8);
void write_hdr(const std::string& path, int w, int h, const float* rgb);

float srgb_to_linear(float c);
float linear_to_srgb(float c);

}  // namespace fmhost
