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

// --precision fp32 | mixed | mixed_fast (the forms of FSIM and SSIM; FLIP and M-SVD compute in FP32).
iqm_precision IQM::precision_option(const Args &args) {
    auto it = args.options.find("--precision");
    if (it == args.options.end() || it->second == "fp32") return IQM_FP32;
    if (it->second == "mixed") return IQM_MIXED;
    if (it->second == "mixed_fast") return IQM_MIXED_FAST;
    throw std::runtime_error("--precision must be fp32, mixed or mixed_fast");
}

// FSIM_ENERGY_SUM reference | full: how FSIM pools its noise-energy estimates (the reference's
// shader fills the first ceil(N/2) pixels only; "full" pools all N).
int IQM::energy_option(const Args &args) {
    auto it = args.options.find("FSIM_ENERGY_SUM");
    if (it == args.options.end() || it->second == "reference") return 0;
    if (it->second == "full") return 1;
    throw std::runtime_error("FSIM_ENERGY_SUM must be reference or full");
}
