// PNG, binary PNM, BMP, TGA, JPEG, GIF, Radiance HDR, RGB PSD and Softimage PIC input, 8-bit grey / RGB / RGBA PNG output, for the command-line front end.
// Decoding always yields RGBA8 like the reference's stbi_load(..., 4) (src/main.cpp:37-57):
// grey -> R=G=B, missing alpha -> 255, 16-bit samples -> their high byte, palettes expanded.
#ifndef IQM_HOST_PNG_IO_H
#define IQM_HOST_PNG_IO_H

#include <string>
#include <vector>

#include "input_image.h"

namespace IQM {
// Throws std::runtime_error("Failed to load image '<path>', reason: ...") on failure.
InputImage load_image(const std::string &path);
// 8-bit single-channel PNG; returns false on failure.
bool write_grey_png(const std::string &path, int width, int height, const std::vector<unsigned char> &pixels);
// 8-bit PNG of 1 (grey), 3 (RGB) or 4 (RGBA) interleaved channels; returns false on failure.
bool write_png(const std::string &path, int width, int height, int channels, const std::vector<unsigned char> &pixels);
std::vector<unsigned char> encode_png(int width, int height, int channels, const std::vector<unsigned char> &pixels);
// Decoders exposed for tests: whole file contents in, RGBA8 out.
InputImage decode_png(const std::vector<unsigned char> &file);
InputImage decode_pnm(const std::vector<unsigned char> &file);
InputImage decode_bmp(const std::vector<unsigned char> &file);  // image_formats.cpp
InputImage decode_tga(const std::vector<unsigned char> &file);  // image_formats.cpp
InputImage decode_jpeg(const std::vector<unsigned char> &file); // jpeg_decode.cpp (baseline)
InputImage decode_gif(const std::vector<unsigned char> &file);  // image_formats.cpp (first frame)
InputImage decode_hdr(const std::vector<unsigned char> &file);  // image_formats.cpp (to 8 bits)
InputImage decode_psd(const std::vector<unsigned char> &file);  // image_formats.cpp (RGB)
InputImage decode_pic(const std::vector<unsigned char> &file);  // image_formats.cpp (Softimage)
std::vector<unsigned char> encode_grey_png(int width, int height, const std::vector<unsigned char> &pixels);
}  // namespace IQM

#endif
