// Test harness: decodes an image file with the command line's decoder and writes the RGBA8 pixels
// (width, height as two little-endian uint32 values, then the bytes) to stdout; with "--encode W H"
// it reads W*H grey bytes from stdin and writes a PNG to stdout ("--encode W H C": W*H*C bytes of C
// interleaved channels, C = 1, 3 or 4).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "png_io.h"

int main(int argc, char **argv) {
    try {
        if ((argc == 4 || argc == 5) && std::strcmp(argv[1], "--encode") == 0) {
            const int w = std::atoi(argv[2]), h = std::atoi(argv[3]), c = argc == 5 ? std::atoi(argv[4]) : 1;
            std::vector<unsigned char> px(size_t(w) * h * c);
            if (std::fread(px.data(), 1, px.size(), stdin) != px.size()) return 2;
            const auto png = c == 1 ? IQM::encode_grey_png(w, h, px) : IQM::encode_png(w, h, c, px);
            std::fwrite(png.data(), 1, png.size(), stdout);
            return 0;
        }
        if (argc != 2) return 2;
        const InputImage img = IQM::load_image(argv[1]);
        const uint32_t dims[2] = {uint32_t(img.width), uint32_t(img.height)};
        std::fwrite(dims, sizeof(dims), 1, stdout);
        std::fwrite(img.data.data(), 1, img.data.size(), stdout);
        return 0;
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
}
