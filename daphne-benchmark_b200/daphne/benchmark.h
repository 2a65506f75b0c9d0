// The DAPHNE benchmark harness interface, restated so that this front end
// links into the harness the same way the reference kernels do
// (src/CPU/include/benchmark.h:11-55): an abstract `kernel` with
// init / run(p) / check_output, a test-case count, pause/resume timer hooks,
// and read_next_testcases.
//
// The class must be layout-identical to the reference's, because the
// reference harness (src/CPU/common/main.cpp:72-80) calls init / run /
// check_output through the vtable of the `myKernel` object that this front
// end defines: the same virtual functions in the same order (no virtual
// destructor: one would shift every vtable slot), the same data members in
// the same order.  The default member initialisers only affect the
// constructor, which runs in this front end's translation unit.
#ifndef NDT_B200_DAPHNE_BENCHMARK_H
#define NDT_B200_DAPHNE_BENCHMARK_H

#include <cstdint>

class kernel {
public:
    // number of test cases in the input (at least 1)
    uint32_t testcases = 1;
    // pre-run set-up: opens the data files, reads the test-case count
    virtual void init() = 0;
    // runs all test cases in blocks of p (read, align, compare per block)
    virtual void run(int p = 1) = 0;
    // true when every result matched the reference data
    virtual bool check_output() = 0;
    // hooks that pause / resume the harness timer around I/O and checking
    void set_timer_functions(void (*pause_function)(), void (*unpause_function)()) {
        unpause_func = unpause_function;
        pause_func = pause_function;
    }

protected:
    void (*unpause_func)() = nullptr;
    void (*pause_func)() = nullptr;
    // reads up to count test cases; returns how many were read
    virtual int read_next_testcases(int count) = 0;
};

#endif
