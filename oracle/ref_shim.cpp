// ref_shim.cpp — C entry points into simple-hpc's own C++ sources (test infrastructure only).
//
// oracle/Makefile compiles this file together with the reference's src/*.cpp (all but main.cpp),
// read in place, into oracle/_ref/libsimpleref.so. Tests load it to pin the C restatement in
// oracle.c against the reference itself, phase by phase, and bench.py's reference arm times its
// OpenMP outer iteration. Nothing from the reference is copied into this repository.
#include "simple/config.hpp"
#include "simple/io.hpp"
#include "simple/momentum_u.hpp"
#include "simple/momentum_v.hpp"
#include "simple/multigrid.hpp"
#include "simple/params.hpp"
#include "simple/pressure.hpp"
#include "simple/solver.hpp"

#include <cstring>
#include <exception>
#include <sstream>
#include <string>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

struct Ref {
    Params p;
    State s;
    explicit Ref(const Params& prm) : p(prm), s(prm) {}
};

Field2D* field(Ref* r, int id) {
    State& s = r->s;
    Field2D* cu[9] = {&s.cu.AE, &s.cu.AW, &s.cu.AN, &s.cu.AS, &s.cu.AEE,
                      &s.cu.AWW, &s.cu.ANN, &s.cu.ASS, &s.cu.AP};
    Field2D* cv[9] = {&s.cv.AE, &s.cv.AW, &s.cv.AN, &s.cv.AS, &s.cv.AEE,
                      &s.cv.AWW, &s.cv.ANN, &s.cv.ASS, &s.cv.AP};
    Field2D* pw[7] = {&s.pw.AEP, &s.pw.AWP, &s.pw.ANP, &s.pw.ASP, &s.pw.APP, &s.pw.b, &s.pw.pc};
    if (id == 0) return &s.u;
    if (id == 1) return &s.v;
    if (id == 2) return &s.p;
    if (id >= 3 && id < 12) return cu[id - 3];
    if (id >= 12 && id < 21) return cv[id - 12];
    if (id >= 21 && id < 28) return pw[id - 21];
    return nullptr;
}
} // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// make_params(parse_config(text)); fills the scalar fields the tests compare. Returns 0 or -1.
int ref_make_params(const char* text, int* ints, double* dbls) {
    try {
        std::istringstream in(text);
        const Params p = make_params(parse_config(in));
        const int iv[] = {p.NX, p.NY, p.H, p.N_halo_x, p.N_halo_y, p.maxit_inner_u, p.maxit_inner_v,
                          p.maxit_inner_p, p.maxit, static_cast<int>(p.convection_scheme),
                          p.diffusion_order, p.Hybrid_switch ? 1 : 0,
                          static_cast<int>(p.residual_normalisation), static_cast<int>(p.backend),
                          static_cast<int>(p.momentum_solver), static_cast<int>(p.pressure_solver),
                          p.pressure_maxit, p.mg_cycles, p.mg_pre, p.mg_post,
                          p.halo_overlap ? 1 : 0, p.write_fields ? 1 : 0, p.grid_rows_cfg,
                          p.grid_cols_cfg, p.nrows, p.ncols};
        const double dv[] = {p.Re, p.error_tolerance, p.relaxation_factor_u, p.relaxation_factor_v,
                             p.relaxation_factor_p, p.pressure_tolerance, p.mg_omega, p.dx, p.dy,
                             p.nu};
        std::memcpy(ints, iv, sizeof iv);
        std::memcpy(dbls, dv, sizeof dv);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void* ref_create(const char* text) {
    try {
        std::istringstream in(text);
        return new Ref(make_params(parse_config(in)));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_destroy(void* h) { delete static_cast<Ref*>(h); }

void ref_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int ref_get(void* h, int id, double* out) {
    Field2D* f = field(static_cast<Ref*>(h), id);
    if (!f) return -1;
    std::memcpy(out, f->data(), sizeof(double) * f->rows() * f->cols());
    return 0;
}

int ref_set(void* h, int id, const double* in) {
    Field2D* f = field(static_cast<Ref*>(h), id);
    if (!f) return -1;
    std::memcpy(f->data(), in, sizeof(double) * f->rows() * f->cols());
    return 0;
}

void ref_assemble_u(void* h) { Ref* r = static_cast<Ref*>(h); assemble_u(r->p, r->s.u, r->s.v, r->s.cu); }
void ref_bc_u(void* h) { Ref* r = static_cast<Ref*>(h); apply_bc_u(r->p, r->s.u); }
double ref_residual_u(void* h) { Ref* r = static_cast<Ref*>(h); return residual_u(r->p, r->s.cu, r->s.u, r->s.p); }
void ref_sweep_u(void* h, int n) { Ref* r = static_cast<Ref*>(h); sweep_u_batch(r->p, r->s.cu, r->s.u, r->s.p, r->s.scratch, n); }
void ref_assemble_v(void* h) { Ref* r = static_cast<Ref*>(h); assemble_v(r->p, r->s.u, r->s.v, r->s.cv); }
void ref_bc_v(void* h) { Ref* r = static_cast<Ref*>(h); apply_bc_v(r->p, r->s.v); }
double ref_residual_v(void* h) { Ref* r = static_cast<Ref*>(h); return residual_v(r->p, r->s.cv, r->s.v, r->s.p); }
void ref_sweep_v(void* h, int n) { Ref* r = static_cast<Ref*>(h); sweep_v_batch(r->p, r->s.cv, r->s.v, r->s.p, r->s.scratch, n); }
double ref_assemble_p(void* h) {
    Ref* r = static_cast<Ref*>(h);
    return assemble_p(r->p, r->s.cu.AP, r->s.cv.AP, r->s.u, r->s.v, r->s.pw);
}
void ref_solve_p(void* h) {
    Ref* r = static_cast<Ref*>(h);
    const Params& p = r->p;
    State& s = r->s;
    if (p.pressure_solver == PressureSolver::Jacobi) solve_pc_jacobi(p, s.pw, s.scratch);
    else if (p.pressure_solver == PressureSolver::GsRedBlack) solve_pc_redblack(p, s.pw);
    else if (p.pressure_solver == PressureSolver::CG) solve_pc_cg(p, s.pw, s.cg);
    else if (p.pressure_solver == PressureSolver::MG) solve_pc_mg(p, s.pw, s.mg);
    else solve_pc_gs_lex(p, s.pw);
}
void ref_correct(void* h) {
    Ref* r = static_cast<Ref*>(h);
    correct(r->p, r->s.pw, r->s.cu.AP, r->s.cv.AP, r->s.u, r->s.v, r->s.p);
}

void ref_outer_iteration(void* h, double* res) {
    Ref* r = static_cast<Ref*>(h);
    PhaseTimers t;
    const Residuals x = outer_iteration(r->p, r->s, t);
    res[0] = x.u;
    res[1] = x.v;
    res[2] = x.p;
}

// run_simple with maxit replaced; log gets 4 doubles per iteration. Returns the iteration count.
int ref_run(void* h, int maxit, double* log, int* converged, double* seconds) {
    Ref* r = static_cast<Ref*>(h);
    Params p = r->p;
    p.maxit = maxit;
    const RunResult out = run_simple(p, r->s);
    for (std::size_t k = 0; k < out.log.size(); ++k)
        for (int m = 0; m < 4; ++m)
            if (log) log[4 * k + m] = out.log[k][static_cast<std::size_t>(m)];
    *converged = out.converged ? 1 : 0;
    if (seconds) *seconds = out.seconds;
    return out.iterations;
}

int ref_cg_last_iterations(void* h) { return static_cast<Ref*>(h)->s.cg.last_iterations; }
int ref_mg_last_coarse_sweeps(void* h) { return static_cast<Ref*>(h)->s.mg.last_coarse_sweeps; }

// Write the reference's output files for the current state into dir (write_outputs, io.cpp:43).
int ref_write_outputs(void* h, const char* dir, int iterations, const double* log) {
    try {
        Ref* r = static_cast<Ref*>(h);
        Params p = r->p;
        p.output_dir = dir;
        RunResult res;
        res.iterations = iterations;
        for (int k = 0; k < iterations; ++k)
            res.log.push_back({log[4 * k], log[4 * k + 1], log[4 * k + 2], log[4 * k + 3]});
        write_outputs(p, r->s.u, r->s.v, r->s.p, res, "ref.cfg");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

} // extern "C"
