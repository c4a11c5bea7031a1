// Batch mode of the command line: evaluate every pair of a list file with one metric, decoding the
// images of the next chunk on worker threads (into page-locked staging buffers) while the GPU
// evaluates the current chunk.  The reference evaluates one pair per process (src/main.cpp:37-57
// decodes with stbi_load on the calling thread, then src/main.cpp:271-286 runs one metric).
//
// List file: one pair per line, "<input path> <reference path>" (whitespace separated; empty lines
// and lines starting with '#' are skipped).  Output: one line per pair, in list order,
//   "<input> <ref> MSSIM: x" | "M-SVD: x" | "FSIM: x FSIMc: y" | "FLIP: x"
// or "<input> <ref> error: <reason>" for a pair that cannot be evaluated (the others still are);
// the exit status is non-zero if any pair failed.
#ifndef IQM_HOST_BATCH_PIPELINE_H
#define IQM_HOST_BATCH_PIPELINE_H

#include <string>

#include "args.h"

namespace IQM {
// Options (KEY VALUE pairs of the command line): --batch LIST, --chunk N (pairs per GPU call,
// default 32), --threads N (decode threads, default: hardware threads), FLIP_RES / FLIP_DISTANCE /
// FLIP_WIDTH as in single-pair mode.  With -v a summary line goes to stderr.
int run_batch(const Args &args);
}  // namespace IQM

#endif
