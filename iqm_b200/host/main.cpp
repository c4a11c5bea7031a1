// IQM command line on the B200 backend, with the reference's flags and output (src/main.cpp):
//   IQM --method {SSIM,SVD,FSIM,FLIP,CW_SSIM_CPU} --input A --ref B [--output P] [-v] [KEY VALUE]...
// Prints "MSSIM: x", "M-SVD: x", "FSIM: x\nFSIMc: y" like the reference, and "FLIP: x" (the
// reference computes the FLIP map but prints no score).  Errors go to stderr with exit code -1.
// Two additions for throughput work:
//   --repeat N   evaluate the pair N times (headless stand-in for the reference's windowed profile
//                loop, src/profile.cpp:227-283), each iteration inside an NVTX range
//                "IQM <method> <i>" for Nsight Systems; with -v, per-iteration times to stdout;
//   --batch LIST evaluate every pair of a list file (batch_pipeline.h).
#include <chrono>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>

#include "args.h"
#include "batch_pipeline.h"
#include "iqm_cuda.hpp"
#include "png_io.h"
#include "viridis_table.h"

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

int repeat_count(const IQM::Args &args) {
    auto it = args.options.find("--repeat");
    if (it == args.options.end()) return 1;
    const int n = std::stoi(it->second);
    if (n < 1) throw std::runtime_error("--repeat must be >= 1");
    return n;
}

// Runs `compute` --repeat times, each in an NVTX range; returns the last result.
template <class F>
auto repeated(const IQM::Args &args, F &&compute) {
    const int n = repeat_count(args);
    std::vector<double> ms;
    decltype(compute()) result = {};
    for (int i = 0; i < n; i++) {
        const std::string range = std::string("IQM ") + IQM::method_name(args.method) + " " + std::to_string(i);
        nvtxRangePushA(range.c_str());
        const auto t0 = clk::now();
        result = compute();
        ms.push_back(std::chrono::duration<double, std::milli>(clk::now() - t0).count());
        nvtxRangePop();
    }
    if (n > 1 && args.verbose) {
        std::vector<double> s = ms;
        std::sort(s.begin(), s.end());
        std::cout << "Iterations: " << n << ", min " << s.front() << " ms, median " << s[s.size() / 2]
                  << " ms, max " << s.back() << " ms" << std::endl;
    }
    return result;
}

void save_map(const IQM::Args &args, unsigned w, unsigned h, const std::vector<float> &map) {
    if (!args.outputPath.has_value()) return;
    if (!IQM::write_grey_png(args.outputPath.value(), int(w), int(h), convertFloatToChar(map)))
        throw std::runtime_error("Failed to save output image");
}

// FLIP --output: each pixel's FLIP value v in [0, 1] shown as viridis entry floor(v * 255), as the
// reference's combine pass colours its output image (shaders/flip/combine_error_maps.glsl:28-32);
// written as RGBA8 (alpha 255, the map's 1.0).
void save_flip_map(const IQM::Args &args, unsigned w, unsigned h, const std::vector<float> &map) {
    if (!args.outputPath.has_value()) return;
    std::vector<unsigned char> rgba(size_t(w) * h * 4);
    for (size_t i = 0; i < map.size(); i++) {
        const int idx = std::clamp(int(std::floor(map[i] * 255.0f)), 0, 255);
        rgba[4 * i] = IQM::kViridisRGB[idx][0];
        rgba[4 * i + 1] = IQM::kViridisRGB[idx][1];
        rgba[4 * i + 2] = IQM::kViridisRGB[idx][2];
        rgba[4 * i + 3] = 255;
    }
    if (!IQM::write_png(args.outputPath.value(), int(w), int(h), 4, rgba))
        throw std::runtime_error("Failed to save output image");
}

void ssim(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    if (args.verbose) std::cout << "Selected device: " << rt.selectedDevice << std::endl;
    IQM::CUDA::SSIM metric(rt);
    metric.precision = IQM::precision_option(args);
    const auto start = clk::now();
    auto result = repeated(args, [&] { return metric.computeMetric(rt, input, ref); });
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
    auto result = repeated(args, [&] { return metric.computeMetric(rt, input, ref); });
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
    metric.precision = IQM::precision_option(args);
    metric.energyMode = IQM::energy_option(args);
    if (args.verbose) std::cout << "Selected device: " << rt.selectedDevice << std::endl;
    const auto start = clk::now();
    auto result = repeated(args, [&] { return metric.computeMetric(rt, input, ref); });
    const auto end = clk::now();
    std::cout << "FSIM: " << result.fsim << std::endl << "FSIMc: " << result.fsimc << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
}

void flip(const IQM::Args &args) {
    InputImage input, ref;
    load_pair(args, input, ref);
    const IQM::CUDA::Runtime rt;
    IQM::CUDA::FLIP metric(rt);
    metric.wantMap = args.outputPath.has_value();
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
    auto result = repeated(args, [&] { return metric.computeMetric(rt, input, ref, flip_args); });
    const auto end = clk::now();
    std::cout << "FLIP: " << result.mean_flip << std::endl;
    if (args.verbose) result.timestamps.print(start, end);
    save_flip_map(args, result.width, result.height, result.imageData);
}

}  // namespace

int main(int argc, const char **argv) {
    auto args = IQM::Args(argc, argv);
    if (args.verbose) std::cout << "Selected method: " << IQM::method_name(args.method) << std::endl;
    try {
        IQM::precision_option(args);  // reject a bad value before any work
        IQM::energy_option(args);
        if (args.options.count("--batch")) return IQM::run_batch(args);
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
