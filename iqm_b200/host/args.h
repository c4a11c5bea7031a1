// Command-line arguments with the reference's rules (src/args.h:15-24, src/args.cpp:9-61):
// `--method M --input A --ref B [--output P] [-v]`; every other `KEY VALUE` pair is kept in
// `options` (FLIP reads FLIP_WIDTH, FLIP_RES, FLIP_DISTANCE from there; the batch and repeat modes
// of this front end read --batch, --chunk, --threads, --repeat).  A missing method, input or
// reference (input and reference are not needed with --batch), or an unknown method name, throws
// std::runtime_error.
#ifndef IQM_HOST_ARGS_H
#define IQM_HOST_ARGS_H

#include <optional>
#include <string>
#include <unordered_map>

#include "methods.h"

namespace IQM {
class Args {
public:
    Args(unsigned argc, const char *argv[]);
    Method method;
    std::string inputPath;
    std::string refPath;
    std::optional<std::string> outputPath;
    std::unordered_map<std::string, std::string> options;
    bool verbose = false;
};
}  // namespace IQM

#endif
