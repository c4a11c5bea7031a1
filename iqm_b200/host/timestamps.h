// Named wall-clock marks printed with -v, in the reference's format (src/timestamps.h):
// "<name>: <since start> | <since previous>" in microseconds, then "TOTAL: <duration>".
#ifndef IQM_HOST_TIMESTAMPS_H
#define IQM_HOST_TIMESTAMPS_H

#include <algorithm>
#include <chrono>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

class Timestamps {
public:
    using clock = std::chrono::high_resolution_clock;
    std::vector<std::pair<std::string, clock::time_point>> inner;

    void mark(const std::string &name) { inner.emplace_back(name, clock::now()); }

    void print(clock::time_point start, clock::time_point end) const {
        using std::chrono::duration_cast;
        using us = std::chrono::microseconds;
        const auto total = duration_cast<us>(end - start);
        int longest = 0;
        for (const auto &m : inner) longest = std::max(longest, int(m.first.size()));
        const int pad = int(std::ceil(std::log10(double(std::max<long long>(1, total.count()))))) + 2;
        auto prev = start;
        for (const auto &m : inner) {
            std::cout << std::setw(longest) << m.first << ": " << std::setw(pad) << duration_cast<us>(m.second - start)
                      << " | " << std::setw(pad) << duration_cast<us>(m.second - prev) << std::endl;
            prev = m.second;
        }
        std::cout << std::setw(longest) << "TOTAL" << ": " << std::setw(pad) << total << std::endl;
    }
};

#endif
