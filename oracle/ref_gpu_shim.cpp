// ref_gpu_shim.cpp — C entry points into simple-hpc's own GPU backend (benchmark baseline only).
//
// oracle/Makefile compiles the reference's src/hip/solver_hip.hip as CUDA for sm_100a (nvcc -x cu
// -DSIMPLE_CUDA --fmad=false, the flags of its own CUDA build, CMakeLists.txt:69-84), read in place,
// and links it with its CPU sources and this file into oracle/_ref/libsimpleref_gpu.so. bench.py
// loads it to time the reference's GPU outer iteration (HipSolver::outer_iteration, one launch per
// colour and a device synchronisation per phase, solver_hip.hip:501-523) on the same B200 as this
// repository's solver, and to check that both give the same fields. Nothing from the reference is
// copied into this repository.
#include "simple/config.hpp"
#include "simple/params.hpp"
#include "simple/solver.hpp"
#include "simple/solver_hip.hpp"
#include "simple/timer.hpp"

#include <chrono>
#include <cstring>
#include <exception>
#include <memory>
#include <sstream>
#include <string>

namespace {
thread_local std::string g_err;

struct RefGpu {
    Params p;
    State s;
    std::unique_ptr<HipSolver> g;
    explicit RefGpu(const Params& prm) : p(prm), s(prm) { g = std::make_unique<HipSolver>(p, s); }
};

Field2D* field(State& s, int id) {
    if (id == 0) return &s.u;
    if (id == 1) return &s.v;
    if (id == 2) return &s.p;
    if (id == 27) return &s.pw.pc;
    return nullptr;
}
} // namespace

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// HipSolver for the parameters of config text (make_params(parse_config(text))), on device 0, from
// the reference's initial State (u = v = p = 0). Null on failure (message in refgpu_last_error).
void* refgpu_create(const char* text) {
    try {
        std::istringstream in(text);
        return new RefGpu(make_params(parse_config(in)));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void refgpu_destroy(void* h) { delete static_cast<RefGpu*>(h); }

// n outer iterations through HipSolver::outer_iteration; res receives 3 residuals per iteration
// (may be null); *seconds the wall time of the n iterations (each phase ends in a device
// synchronisation, so the wall time is the device time plus launch gaps).
int refgpu_iterations(void* h, int n, double* res, double* seconds) {
    try {
        RefGpu& r = *static_cast<RefGpu*>(h);
        PhaseTimers t;
        const auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < n; ++k) {
            const Residuals rr = r.g->outer_iteration(t);
            if (res) {
                res[3 * k + 0] = rr.u;
                res[3 * k + 1] = rr.v;
                res[3 * k + 2] = rr.p;
            }
        }
        if (seconds)
            *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The reference's own outer loop (run_outer_loop, src/solver.cpp:106-132: its stopping rule, its
// "iter k" lines) around HipSolver::outer_iteration, at most p.maxit iterations from the current
// state. *seconds is the loop's wall time as run_outer_loop measures it.
int refgpu_run(void* h, int* iterations, int* converged, double* seconds) {
    try {
        RefGpu& r = *static_cast<RefGpu*>(h);
        const RunResult out = run_outer_loop(r.p, [&](PhaseTimers& t) { return r.g->outer_iteration(t); });
        if (iterations) *iterations = out.iterations;
        if (converged) *converged = out.converged ? 1 : 0;
        if (seconds) *seconds = out.seconds;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Field id 0 / 1 / 2 / 27 (u, v, p, p'): the full nrows x ncols array after HipSolver::download.
int refgpu_download(void* h, int id, double* out) {
    try {
        RefGpu& r = *static_cast<RefGpu*>(h);
        r.g->download(r.s);
        Field2D* f = field(r.s, id);
        if (!f) {
            g_err = "bad field id";
            return -1;
        }
        std::memcpy(out, f->data(), sizeof(double) * static_cast<std::size_t>(f->rows()) * f->cols());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

} // extern "C"
