// Command-line driver, the counterpart of the reference's `fdfault file.in`
// (src/main.cpp:8-72): builds the problem, runs problem::solve, and writes
// the output units and fronts.
// Usage: fdfault_b200 [--fp32] [--device N] [--plastic-every-node] file.in
// (--plastic-every-node: fdf_set_plastic_rule FDF_PLASTIC_EVERY_NODE)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#include "../../include/fdfault_b200.h"

static void stamp(const char* what) {
    std::time_t t = std::time(nullptr);
    std::printf("%s %s", what, std::asctime(std::localtime(&t)));
}

int main(int argc, char** argv) {
    int precision = FDF_PRECISION_FP64, device = 0, plastic_rule = FDF_PLASTIC_REFERENCE;
    const char* infile = nullptr;
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--fp32"))
            precision = FDF_PRECISION_FP32;
        else if (!std::strcmp(argv[i], "--plastic-every-node"))
            plastic_rule = FDF_PLASTIC_EVERY_NODE;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else
            infile = argv[i];
    }
    if (!infile) {
        std::fprintf(stderr, "usage: %s [--fp32] [--device N] [--plastic-every-node] file.in\n", argv[0]);
        return 2;
    }
    std::printf("fdfault_b200 on device %d\nReading from input file %s\n", device, infile);
    fdf_handle* h = nullptr;
    int rc = fdf_create(infile, precision, device, &h);
    if (rc) {
        std::fprintf(stderr, "error: %s\n", fdf_last_error(nullptr));
        return 1;
    }
    if (plastic_rule != FDF_PLASTIC_REFERENCE && (rc = fdf_set_plastic_rule(h, plastic_rule))) {
        std::fprintf(stderr, "error: %s\n", fdf_last_error(h));
        fdf_destroy(h);
        return 1;
    }
    stamp("Initialization finished");
    auto t0 = std::chrono::steady_clock::now();
    rc = fdf_solve(h);
    auto t1 = std::chrono::steady_clock::now();
    if (rc) {
        std::fprintf(stderr, "error: %s\n", fdf_last_error(h));
        fdf_destroy(h);
        return 1;
    }
    stamp("Problem finished");
    std::printf("solve_seconds %.6f\n", std::chrono::duration<double>(t1 - t0).count());
    fdf_destroy(h);
    return 0;
}
