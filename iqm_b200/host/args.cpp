#include "args.h"

#include <cstring>
#include <stdexcept>

namespace {
bool parse_method(const char *name, IQM::Method &m) {
    struct Entry {
        const char *name;
        IQM::Method m;
    };
    static const Entry table[] = {{"SSIM", IQM::Method::SSIM},
                                  {"CW_SSIM_CPU", IQM::Method::CW_SSIM_CPU},
                                  {"SVD", IQM::Method::SVD},
                                  {"FSIM", IQM::Method::FSIM},
                                  {"FLIP", IQM::Method::FLIP}};
    for (const Entry &e : table)
        if (std::strcmp(name, e.name) == 0) {
            m = e.m;
            return true;
        }
    return false;
}
}  // namespace

IQM::Args::Args(const unsigned argc, const char *argv[]) {
    bool have_method = false, have_input = false, have_ref = false;
    for (unsigned i = 0; i < argc; i++) {
        const char *a = argv[i];
        if (i + 1 < argc) {
            const char *v = argv[i + 1];
            if (std::strcmp(a, "--method") == 0) {
                if (!parse_method(v, method)) throw std::runtime_error("Unknown method");
                have_method = true;
            } else if (std::strcmp(a, "--input") == 0) {
                inputPath = v;
                have_input = true;
            } else if (std::strcmp(a, "--ref") == 0) {
                refPath = v;
                have_ref = true;
            } else if (std::strcmp(a, "--output") == 0) {
                outputPath = std::string(v);
            } else {
                options.emplace(std::string(a), std::string(v));
            }
        }
        if (std::strcmp(a, "-v") == 0) verbose = true;
    }
    if (!have_method) throw std::runtime_error("missing method");
    const bool batch = options.count("--batch") != 0;  // pairs come from the list file
    if (!have_input && !batch) throw std::runtime_error("missing input");
    if (!have_ref && !batch) throw std::runtime_error("missing reference");
}
