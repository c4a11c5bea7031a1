// IQM command line on the B200 backend, with the reference's flags and output (src/main.cpp):
//   IQM --method {SSIM,SVD,FSIM,FLIP,CW_SSIM_CPU} --input A --ref B [--output P] [-v] [KEY VALUE]...
// Prints "MSSIM: x", "M-SVD: x", "FSIM: x\nFSIMc: y" like the reference, and "FLIP: x" (the
// reference computes the FLIP map but prints no score).  Errors go to stderr with exit code -1.
#include <chrono>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "args.h"
#include "iqm_cuda.hpp"
#include "png_io.h"

namespace {

using clk = std::chrono::high_resolution_clock;

// src/main.cpp:59-67: map values in [0,1] to bytes by truncating v * 255
std::vector<unsigned char> convertFloatToChar(const std::vector<float> &data) {
    std::vector<unsigned char> out(data.size());
    for (size_t i = 0; i < data.size(); i++) out[i] = static_cast<unsigned char>(data[i] * 255.0f);
    return out;
}

void load_pair(const IQM::Args &args, InputImage &input, InputImage &ref) {
    input = IQM::load_image(args.inputPath);
    ref = IQM::load_image(args.refPath);
    if (input.width != ref.width || input.height != ref.height)
        throw std::runtime_error("Compared images must have the same size");
}

void save_map(const IQM::Args &args, unsigned w, unsigned h, const std::vector<float> &map) {
    if (!args.outputPath.has_value()) return;
    if (!IQM::write_grey_png(args.outputPath.value(), int(w), int(h), convertFloatToChar(map)))
        throw std::runtime_error("Failed to save output image");
}

void ssim(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    if (args.verbose) std::cout << "Selected device: " << rt.selectedDevice << std::endl;
    IQM::CUDA::SSIM metric(rt);
    const auto start = clk::now();
    auto result = metric.computeMetric(rt, input, ref);
    const auto end = clk::now();
    std::cout << "MSSIM: " << result.mssim << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
    save_map(args, result.width, result.height, result.imageData);
}

void svd(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    IQM::CUDA::SVD metric(rt);
    if (args.verbose) std::cout << "Selected device: " << rt.selectedDevice << std::endl;
    const auto start = clk::now();
    auto result = metric.computeMetric(rt, input, ref);
    const auto end = clk::now();
    std::cout << "M-SVD: " << result.msvd << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
    save_map(args, result.width, result.height, result.imageData);
}

void fsim(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    IQM::CUDA::FSIM metric(rt);
    if (args.verbose) std::cout << "Selected device: " << rt.selectedDevice << std::endl;
    const auto start = clk::now();
    auto result = metric.computeMetric(rt, input, ref);
    const auto end = clk::now();
    std::cout << "FSIM: " << result.fsim << std::endl << "FSIMc: " << result.fsimc << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
}

void flip(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    IQM::CUDA::FLIP metric(rt);
    IQM::CUDA::FLIPArguments flip_args;
    if (args.options.count("FLIP_WIDTH")) flip_args.monitor_width = std::stof(args.options.at("FLIP_WIDTH"));
    if (args.options.count("FLIP_RES")) flip_args.monitor_resolution_x = std::stof(args.options.at("FLIP_RES"));
    if (args.options.count("FLIP_DISTANCE")) flip_args.monitor_distance = std::stof(args.options.at("FLIP_DISTANCE"));
    if (args.verbose) {
        std::cout << "Selected device: " << rt.selectedDevice << std::endl
                  << "FLIP monitor resolution: " << flip_args.monitor_resolution_x << std::endl
                  << "FLIP monitor distance: " << flip_args.monitor_distance << std::endl
                  << "FLIP monitor width: " << flip_args.monitor_width << std::endl;
    }
    const auto start = clk::now();
    auto result = metric.computeMetric(rt, input, ref, flip_args);
    const auto end = clk::now();
    std::cout << "FLIP: " << result.mean_flip << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
}

}  // namespace

int main(int argc, const char **argv) {
    auto args = IQM::Args(argc, argv);
    if (args.verbose) std::cout << "Selected method: " << IQM::method_name(args.method) << std::endl;
    try {
        switch (args.method) {
            case IQM::Method::SSIM: ssim(args); break;
            case IQM::Method::CW_SSIM_CPU: break;  // the reference's CW-SSIM is an empty stub
            case IQM::Method::SVD: svd(args); break;
            case IQM::Method::FSIM: fsim(args); break;
            case IQM::Method::FLIP: flip(args); break;
        }
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        exit(-1);
    }
    return 0;
}
