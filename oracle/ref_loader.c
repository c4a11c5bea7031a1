/* Test infrastructure: the reference's own image loader, to check the command line's decoders
 * against.  cadik/IQM reads every input with stbi_load(path, &w, &h, &channels, 4) from the
 * stb_image.h it vendors (src/main.cpp:37-57, lib/stb/stb_image.h, compiled with
 * STB_IMAGE_IMPLEMENTATION and STBI_FAILURE_USERMSG as src/main.cpp:9-10 do).  This program makes
 * that one call, with the header taken from the reference's tree by oracle/Makefile's `ref` target
 * (output oracle/_ref/ref_loader; nothing of it is copied here), and writes the result as the test
 * loader tests/native/png_check.cpp writes this repository's: width and height as little-endian
 * 32-bit words, then the RGBA8 bytes.  On failure it prints the loader's reason and exits 1. */
#define STB_IMAGE_IMPLEMENTATION
#define STBI_FAILURE_USERMSG
#include "stb_image.h"

#include <stdint.h>
#include <stdio.h>

int main(int argc, char **argv) {
    if (argc != 2) {
        fprintf(stderr, "usage: ref_loader IMAGE\n");
        return 2;
    }
    int w = 0, h = 0, n = 0;
    unsigned char *px = stbi_load(argv[1], &w, &h, &n, 4);
    if (!px) {
        fprintf(stderr, "%s\n", stbi_failure_reason());
        return 1;
    }
    const uint32_t dims[2] = {(uint32_t)w, (uint32_t)h};
    unsigned char le[8];
    for (int i = 0; i < 2; i++)
        for (int b = 0; b < 4; b++) le[4 * i + b] = (unsigned char)(dims[i] >> (8 * b));
    fwrite(le, 1, 8, stdout);
    fwrite(px, 1, (size_t)w * h * 4, stdout);
    stbi_image_free(px);
    return 0;
}
