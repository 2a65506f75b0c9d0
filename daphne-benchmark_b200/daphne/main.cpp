// DAPHNE-style harness main: `kernel [-p N]` runs the linked kernel object,
// timing run() with the kernel's I/O and checking paused, then prints the
// elapsed time, the average per test case and "result ok" / "error: wrong
// result" (exit 0 / 1), as the reference harness does
// (src/CPU/common/main.cpp:47-97).  Exit codes 2-4 for bad arguments.
#include <cerrno>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>

#include "benchmark.h"

extern kernel &myKernel;

namespace {
using clock_type = std::chrono::high_resolution_clock;
clock_type::time_point t_start;
std::chrono::duration<double> t_elapsed{0};
bool t_paused = false;

void pause_timer() {
    t_elapsed += clock_type::now() - t_start;
    t_paused = true;
}

void unpause_timer() {
    t_paused = false;
    t_start = clock_type::now();
}

void usage(const char *exe) {
    std::cout << "Usage: \n" << exe << " [-p N]\nOptions:\n  -p N   executes N invocations in sequence,"
              << "before taking time and check the result.\n         Default: N=1\n";
}
}  // namespace

int main(int argc, char **argv) {
    int pipelined = 1;
    if (argc != 1 && argc != 3) {
        usage(argv[0]);
        return 2;
    }
    if (argc == 3) {
        if (std::strcmp(argv[1], "-p") != 0) {
            usage(argv[0]);
            return 3;
        }
        errno = 0;
        pipelined = (int)std::strtol(argv[2], nullptr, 10);
        if (errno || pipelined < 1) {
            usage(argv[0]);
            return 4;
        }
        std::cout << "Invoking kernel " << pipelined << " time(s) per measure/checking step\n";
    }
    myKernel.set_timer_functions(pause_timer, unpause_timer);
    myKernel.init();
    t_start = clock_type::now();
    myKernel.run(pipelined);
    if (!t_paused) t_elapsed += clock_type::now() - t_start;
    std::cout << "elapsed time: " << t_elapsed.count() << " seconds, average time per testcase (#"
              << myKernel.testcases << "): " << t_elapsed.count() / (double)myKernel.testcases << " seconds"
              << std::endl;
    if (myKernel.check_output()) {
        std::cout << "result ok\n";
        return 0;
    }
    std::cout << "error: wrong result\n";
    return 1;
}
