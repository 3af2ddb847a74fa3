/*
 * oracle.h — CPU restatement of simple-hpc's SIMPLE outer iteration, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it, and only as the checker or the timed CPU baseline; the GPU solver never calls it.
 *
 * Parity pin: the restatement is checked against the reference's committed snapshots
 * (tests/snapshots/short_16, converged_32x40, kept as fixtures in tests/golden/) and, in this
 * container, live against the reference's own C++ sources built into oracle/_ref/.
 */
#ifndef SIMPLE_ORACLE_H
#define SIMPLE_ORACLE_H

#include "../include/sgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

orc_state* orc_create(const sgpu_params_t* p);
void orc_destroy(orc_state* s);
int orc_get(orc_state* s, int field_id, double* out);
int orc_set(orc_state* s, int field_id, const double* in);

void orc_assemble_u(orc_state* s);
void orc_bc_u(orc_state* s);
double orc_residual_u(orc_state* s);
void orc_sweep_u(orc_state* s, int nsweeps);
void orc_assemble_v(orc_state* s);
void orc_bc_v(orc_state* s);
double orc_residual_v(orc_state* s);
void orc_sweep_v(orc_state* s, int nsweeps);
double orc_assemble_p(orc_state* s);
void orc_solve_p(orc_state* s);
void orc_correct(orc_state* s);
void orc_outer_iteration(orc_state* s, double res[3]);
/* Outer loop with the reference's stopping rule; log holds 4 doubles per iteration. */
int orc_run(orc_state* s, int maxit, double* log, int* converged);

/* Multigrid / CG introspection for the unit tests. */
int orc_mg_level_dims(int nx, int ny, int* dims /* 2 * 64 */);
int orc_mg_nlevels(orc_state* s);
int orc_mg_last_coarse_sweeps(orc_state* s);
int orc_cg_last_iterations(orc_state* s);
double orc_cg_last_rel_residual(orc_state* s);
/* One V-cycle on the current pc / b (mg_build must have run: orc_mg_build). */
void orc_mg_build(orc_state* s);
void orc_mg_vcycle(orc_state* s);
/* Copy level l's interior (nx x ny) of array k (0 AE, 1 AW, 2 AN, 3 AS, 4 AP, 5 b, 6 x, 7 r). */
int orc_mg_get_level(orc_state* s, int l, int k, double* out);

/* Ordered sum of a row-major nr x nc block: rows left to right from 0.0, then rows in order. */
double orc_ordered_sum(const double* v, int nr, int nc);

/* Coefficient kernels (coefficients.cpp:10-63), for the known-answer tests. c[9] in AE AW AN AS
 * AEE AWW ANN ASS AP order. */
int orc_in_boundary_band(const sgpu_params_t* p, int i, int j);
void orc_convective(const sgpu_params_t* p, double ue, double uw, double vn, double vs, int i,
                    int j, double c[9]);
void orc_diffusive(const sgpu_params_t* p, int i, int j, double c[9]);

#ifdef __cplusplus
}
#endif
#endif
