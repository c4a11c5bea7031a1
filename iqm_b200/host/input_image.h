// Decoded image handed to the metrics: always RGBA8, tightly packed (src/input_image.h).
#ifndef IQM_HOST_INPUT_IMAGE_H
#define IQM_HOST_INPUT_IMAGE_H

#include <vector>

struct InputImage {
    int width;
    int height;
    std::vector<unsigned char> data;
};

#endif
