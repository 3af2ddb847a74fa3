// sgpu_backend.cpp — the reference-side binding: run_simple_hip's replacement over the C ABI.
//
// A simple-hpc maintainer adds this file to simple-hpc's src/ and calls run_simple_sgpu(p, s) where
// main (src/main.cpp:40-46) calls run_simple_hip(p, s) (include/simple/solver_hip.hpp:40). It is
// compiled with simple-hpc's own headers and linked against libsgpu.so; nothing of the reference
// is needed to build this repository.
#include "simple/solver.hpp"
#include "sgpu.h"                       // include/ of this repository
#include <stdexcept>
#include <string>
#include <vector>

static void check(int rc) {
    if (rc != SGPU_OK) throw std::runtime_error(std::string("GPU error: ") + sgpu_last_error());
}

RunResult run_simple_sgpu(const Params& p, State& s) {
    sgpu_params_t q{};
    check(sgpu_params_default(&q));
    q.NX = p.NX; q.NY = p.NY; q.N_halo_x = p.N_halo_x; q.N_halo_y = p.N_halo_y; q.Re = p.Re;
    q.maxit_inner_u = p.maxit_inner_u; q.maxit_inner_v = p.maxit_inner_v;
    q.maxit_inner_p = p.maxit_inner_p; q.error_tolerance = p.error_tolerance; q.maxit = p.maxit;
    q.relaxation_factor_u = p.relaxation_factor_u; q.relaxation_factor_v = p.relaxation_factor_v;
    q.relaxation_factor_p = p.relaxation_factor_p;
    q.convection_scheme = p.convection_scheme == Convection::UDS ? SGPU_UDS : SGPU_QUICK;
    q.diffusion_order = p.diffusion_order;
    q.residual_normalisation = p.residual_normalisation == ResidualNorm::Absolute
                                   ? SGPU_NORM_ABSOLUTE : SGPU_NORM_RUNNING_MAX;
    q.backend = SGPU_BACKEND_GPU;
    q.momentum_solver = static_cast<int>(p.momentum_solver);   // same enum order
    q.pressure_solver = static_cast<int>(p.pressure_solver);   // same enum order
    q.pressure_tolerance = p.pressure_tolerance; q.pressure_maxit = p.pressure_maxit;
    q.mg_cycles = p.mg_cycles; q.mg_pre = p.mg_pre; q.mg_post = p.mg_post; q.mg_omega = p.mg_omega;
    check(sgpu_params_finalize(&q));    // nrows, ncols, dx, dy, nu exactly as make_params

    sgpu_handle* h = nullptr;
    check(sgpu_create(&q, s.u.data(), s.v.data(), s.p.data(), &h));
    std::vector<double> log(4 * static_cast<size_t>(p.maxit));
    sgpu_result_t r{};
    // Sampled timers: the first iterations are timed per phase for timing.csv, the rest replay the
    // captured iteration graph (the fast path). A diverged run (SGPU_E_NONFINITE) still returns
    // its fields, as the reference returns those of a run that reached maxit.
    int rc = sgpu_set_profiling(h, 2);
    if (rc == SGPU_OK) rc = sgpu_run(h, p.maxit, log.data(), 100, &r);
    const bool diverged = rc == SGPU_E_NONFINITE;
    if (diverged) rc = SGPU_OK;
    if (rc == SGPU_OK) rc = sgpu_download(h, SGPU_F_U, s.u.data());
    if (rc == SGPU_OK) rc = sgpu_download(h, SGPU_F_V, s.v.data());
    if (rc == SGPU_OK) rc = sgpu_download(h, SGPU_F_P, s.p.data());
    sgpu_destroy(h);
    check(rc);

    RunResult out;
    out.iterations = r.iterations;
    out.converged = r.converged != 0;
    out.seconds = r.seconds;
    out.cg_iterations = r.cg_iterations;
    for (int k = 0; k < r.iterations; ++k)
        out.log.push_back({log[4 * k], log[4 * k + 1], log[4 * k + 2], log[4 * k + 3]});
    for (int ph = 0; ph < SGPU_PH_COUNT; ++ph) out.timers.seconds[ph] = r.phase_seconds[ph];
    return out;
}
