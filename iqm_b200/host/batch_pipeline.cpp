#include "batch_pipeline.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <vector>

#include "iqm_cuda.h"
#include "iqm_cuda.hpp"
#include "png_io.h"

namespace {

struct Job {
    std::string input, ref;
};

// Page-locked buffer owned by one staging slot entry (grow-only).
struct Pinned {
    void *ptr = nullptr;
    size_t cap = 0;
    Pinned() = default;
    Pinned(const Pinned &) = delete;
    Pinned &operator=(const Pinned &) = delete;
    Pinned(Pinned &&o) noexcept : ptr(o.ptr), cap(o.cap) {
        o.ptr = nullptr;
        o.cap = 0;
    }
    void ensure(size_t bytes) {
        if (bytes <= cap) return;
        if (ptr) iqm_host_free(ptr);
        ptr = nullptr;
        cap = 0;
        if (iqm_host_alloc(bytes, &ptr) != IQM_OK) throw std::runtime_error("page-locked allocation failed");
        cap = bytes;
    }
    ~Pinned() {
        if (ptr) iqm_host_free(ptr);
    }
};

// One chunk's decoded pairs.
struct Chunk {
    size_t first = 0, count = 0;
    std::vector<Pinned> img;         // 2 per pair
    std::vector<iqm_pair> pairs;     // per pair (valid only where ok)
    std::vector<std::string> error;  // per pair, empty when decoded
};

std::vector<Job> read_list(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("Failed to open batch list '" + path + "'");
    std::vector<Job> jobs;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        Job j;
        if (!(is >> j.input) || j.input[0] == '#') continue;
        if (!(is >> j.ref)) throw std::runtime_error("Batch list line without a reference image: " + line);
        jobs.push_back(j);
    }
    return jobs;
}

// Decodes jobs [first, first + count) into `c` with `threads` workers.
void decode_chunk(const std::vector<Job> &jobs, size_t first, size_t count, int threads, Chunk &c) {
    c.first = first;
    c.count = count;
    if (c.img.size() < 2 * count) c.img.resize(2 * count);
    c.pairs.assign(count, iqm_pair{});
    c.error.assign(count, std::string());
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i = next++; i < count; i = next++) {
            const Job &j = jobs[first + i];
            try {
                const InputImage a = IQM::load_image(j.input);
                const InputImage b = IQM::load_image(j.ref);
                if (a.width != b.width || a.height != b.height)
                    throw std::runtime_error("Compared images must have the same size");
                const size_t bytes = size_t(a.width) * a.height * 4;
                c.img[2 * i].ensure(bytes);
                c.img[2 * i + 1].ensure(bytes);
                std::memcpy(c.img[2 * i].ptr, a.data.data(), bytes);
                std::memcpy(c.img[2 * i + 1].ptr, b.data.data(), bytes);
                c.pairs[i] = iqm_pair{static_cast<const uint8_t *>(c.img[2 * i].ptr),
                                      static_cast<const uint8_t *>(c.img[2 * i + 1].ptr), int(a.width),
                                      int(a.height), size_t(a.width) * 4};
            } catch (const std::exception &e) {
                c.error[i] = e.what();
            }
        }
    };
    std::vector<std::thread> pool;
    const int n = std::max(1, std::min<int>(threads, int(count)));
    for (int t = 1; t < n; t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
}

const char *label(IQM::Method m) {
    switch (m) {
        case IQM::Method::SSIM: return "MSSIM";
        case IQM::Method::SVD: return "M-SVD";
        case IQM::Method::FSIM: return "FSIM";
        case IQM::Method::FLIP: return "FLIP";
        default: return "";
    }
}

// Evaluates n decoded pairs with one batch call; k scores per pair (k = 2 for FSIM).
int evaluate(const IQM::CUDA::Runtime &rt, IQM::Method m, const iqm_flip_params &flip, iqm_precision precision,
             int energy_mode, const iqm_pair *pairs, int n, double *scores) {
    switch (m) {
        case IQM::Method::SSIM: {
            iqm_ssim_params p;
            iqm_ssim_default_params(&p);
            p.precision = int(precision);
            return iqm_ssim_batch(rt.ctx, pairs, n, &p, scores);
        }
        case IQM::Method::SVD: return iqm_msvd_batch(rt.ctx, pairs, n, scores);
        case IQM::Method::FSIM: return iqm_fsim_batch(rt.ctx, pairs, n, precision, energy_mode, scores);
        case IQM::Method::FLIP: return iqm_flip_batch(rt.ctx, pairs, n, &flip, scores);
        default: return IQM_OK;
    }
}

int option_int(const IQM::Args &args, const char *key, int def) {
    auto it = args.options.find(key);
    if (it == args.options.end()) return def;
    const int v = std::stoi(it->second);
    if (v < 1) throw std::runtime_error(std::string(key) + " must be >= 1");
    return v;
}

}  // namespace

int IQM::run_batch(const Args &args) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const std::vector<Job> jobs = read_list(args.options.at("--batch"));
    const int chunk = option_int(args, "--chunk", 32);
    const int threads = option_int(args, "--threads", int(std::max(1u, std::thread::hardware_concurrency())));
    iqm_flip_params flip;
    iqm_flip_default_params(&flip);
    if (args.options.count("FLIP_WIDTH")) flip.monitor_width = std::stof(args.options.at("FLIP_WIDTH"));
    if (args.options.count("FLIP_RES")) flip.monitor_resolution_x = std::stof(args.options.at("FLIP_RES"));
    if (args.options.count("FLIP_DISTANCE")) flip.monitor_distance = std::stof(args.options.at("FLIP_DISTANCE"));
    const iqm_precision precision = precision_option(args);
    const int energy_mode = energy_option(args);
    if (args.method == Method::CW_SSIM_CPU) return 0;  // the reference's CW-SSIM is an empty stub
    const CUDA::Runtime rt;
    const int k = args.method == Method::FSIM ? 2 : 1;
    int failed = 0;
    double gpu_s = 0.0;
    Chunk bufs[2];
    std::future<void> pending;
    if (!jobs.empty())
        pending = std::async(std::launch::async, decode_chunk, std::cref(jobs), size_t(0),
                             std::min<size_t>(chunk, jobs.size()), threads, std::ref(bufs[0]));
    for (size_t first = 0, c = 0; first < jobs.size(); first += chunk, c ^= 1) {
        pending.get();
        Chunk &cur = bufs[c];
        const size_t nxt = first + chunk;
        if (nxt < jobs.size())  // decode the next chunk while this one runs on the GPU
            pending = std::async(std::launch::async, decode_chunk, std::cref(jobs), nxt,
                                 std::min<size_t>(chunk, jobs.size() - nxt), threads, std::ref(bufs[c ^ 1]));
        std::vector<iqm_pair> ok;
        std::vector<size_t> where;
        for (size_t i = 0; i < cur.count; i++)
            if (cur.error[i].empty()) {
                ok.push_back(cur.pairs[i]);
                where.push_back(i);
            }
        std::vector<double> scores(k * ok.size());
        std::vector<std::string> err(cur.count);
        for (size_t i = 0; i < cur.count; i++) err[i] = cur.error[i];
        if (!ok.empty()) {
            const auto g0 = clk::now();
            int rc = evaluate(rt, args.method, flip, precision, energy_mode, ok.data(), int(ok.size()), scores.data());
            if (rc != IQM_OK) {  // find the pairs the call rejects, evaluate the rest one by one
                for (size_t q = 0; q < ok.size(); q++)
                    if (evaluate(rt, args.method, flip, precision, energy_mode, &ok[q], 1, &scores[k * q]) != IQM_OK)
                        err[where[q]] = iqm_last_error(rt.ctx);
            }
            gpu_s += std::chrono::duration<double>(clk::now() - g0).count();
        }
        for (size_t q = 0, i = 0; i < cur.count; i++) {
            const Job &j = jobs[cur.first + i];
            std::cout << j.input << ' ' << j.ref << ' ';
            if (!err[i].empty()) {
                std::cout << "error: " << err[i] << '\n';
                failed++;
                if (q < where.size() && where[q] == i) q++;
                continue;
            }
            const double *s = &scores[k * q++];
            std::cout << label(args.method) << ": " << float(s[0]);
            if (k == 2) std::cout << " FSIMc: " << float(s[1]);
            std::cout << '\n';
        }
        std::cout.flush();
    }
    if (args.verbose) {
        const double wall = std::chrono::duration<double>(clk::now() - t0).count();
        std::fprintf(stderr, "batch: %zu pairs, %d failed, %.3f s wall, %.3f s in GPU calls, %.1f pairs/s, %d decode threads\n",
                     jobs.size(), failed, wall, gpu_s, wall > 0 ? double(jobs.size()) / wall : 0.0, threads);
    }
    return failed ? 1 : 0;
}
