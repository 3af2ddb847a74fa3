// adapter_check.cpp — the drop-in check of the reference-side binding (test infrastructure only).
//
// oracle/Makefile links this file with simple-hpc's own C++ sources (read in place), the binding
// simple-hpc_b200/adapter/sgpu_backend.cpp and libsgpu.so. It reads one config file, runs it through
// the reference's run_simple (its CPU path, src/solver.cpp:95-104) and through run_simple_sgpu (the
// binding, which a simple-hpc main calls in place of run_simple_hip), and compares the iteration
// count, the converged flag, the residual log and u, v, p bit for bit. Exit status 0 and the line
// "adapter ok" when they are identical, 1 otherwise.
#include "simple/config.hpp"
#include "simple/params.hpp"
#include "simple/solver.hpp"

#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>

RunResult run_simple_sgpu(const Params& p, State& s);

static bool same(const Field2D& a, const Field2D& b) {
    const std::size_t n = static_cast<std::size_t>(a.rows()) * a.cols();
    return a.rows() == b.rows() && a.cols() == b.cols() && std::memcmp(a.data(), b.data(), n * sizeof(double)) == 0;
}

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: adapter_check <config>\n");
        return 2;
    }
    try {
        std::ifstream f(argv[1]);
        const Params p = make_params(parse_config(f));
        State cpu(p), gpu(p);
        const RunResult rc = run_simple(p, cpu);
        const RunResult rg = run_simple_sgpu(p, gpu);
        bool ok = rc.iterations == rg.iterations && rc.converged == rg.converged &&
                  rc.log.size() == rg.log.size();
        for (std::size_t k = 0; ok && k < rc.log.size(); ++k)
            ok = std::memcmp(rc.log[k].data(), rg.log[k].data(), sizeof(double) * 4) == 0;
        const bool fields = same(cpu.u, gpu.u) && same(cpu.v, gpu.v) && same(cpu.p, gpu.p);
        std::printf("reference CPU: %d iterations, converged %d; adapter: %d iterations, converged %d; "
                    "log %s, fields %s\n", rc.iterations, rc.converged ? 1 : 0, rg.iterations,
                    rg.converged ? 1 : 0, ok ? "identical" : "DIFFERENT", fields ? "identical" : "DIFFERENT");
        double phase_sum = 0.0;
        for (double t : rg.timers.seconds) phase_sum += t;
        std::printf("adapter phase seconds sum %.6f, run seconds %.6f\n", phase_sum, rg.seconds);
        if (!(ok && fields && phase_sum > 0.0)) return 1;
        std::printf("adapter ok\n");
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
