// Prints the host FFT planner's choice for every length given on the command line:
//   "<n> direct <radices...>"  or  "<n> bluestein <m> <radices of m...>"
// Built and run by tests/test_fft_planner.py (host code only, no device needed).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fft_plan.cuh"

int main(int argc, char **argv) {
    for (int i = 1; i < argc; i++) {
        const int n = std::atoi(argv[i]);
        std::vector<int> r, rm;
        int m = 0;
        if (iqm::plan_length(n, r, m, rm)) {
            std::printf("%d direct", n);
            for (int p : r) std::printf(" %d", p);
        } else {
            std::printf("%d bluestein %d", n, m);
            for (int p : rm) std::printf(" %d", p);
        }
        std::printf("\n");
    }
    return 0;
}
