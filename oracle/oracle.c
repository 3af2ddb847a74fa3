/*
 * oracle.c — CPU restatement of simple-hpc's SIMPLE outer iteration (test infrastructure only).
 *
 * Each function follows one reference function, cited by file:line in simple-hpc. Per-cell
 * expressions keep the reference's operation order, and the build disables FMA contraction
 * (-ffp-contract=off, as the reference's CMakeLists.txt:34 does), so results are bit-identical to
 * the reference's serial path. Sums use the reference's fixed order: each row added left to right
 * from 0.0, then the row sums top to bottom (CellSums, src/decomp.cpp:176-205; det_sum,
 * src/multigrid.cpp:18-34).
 *
 * This is the checker for the GPU solver, never part of it.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NCOEF 9
enum { AE = 0, AW, AN, AS, AEE, AWW, ANN, ASS, AP };

typedef struct {
    int nx, ny, stride;
    double *AE, *AW, *AN, *AS, *AP, *b, *x, *r; /* point at interior cell (0, 0) */
    double* mem[8];                              /* owned storage (levels > 0) */
} orc_level;

struct orc_state {
    sgpu_params_t p;
    size_t n; /* nrows * ncols */
    double *u, *v, *pf;
    double *cu[NCOEF], *cv[NCOEF];
    double *AEP, *AWP, *ANP, *ASP, *APP, *b, *pc;
    double* scratch;
    double *cg_r, *cg_z, *cg_d, *cg_q;
    int cg_last_iters;
    double cg_last_rel;
    int nlev;
    orc_level lev[64];
    double* mg_r0;
    int last_coarse_sweeps;
    double* rowbuf; /* row sums, up to max(nrows, 4) * 4 values */
};

#define IX(s, i, j) ((size_t)(i) * (size_t)(s)->p.ncols + (size_t)(j))

static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* std::max(0.0, a) == (0.0 < a) ? a : 0.0, signed zeros included (coefficients.cpp:19). */
static inline double mx(double a) { return (0.0 < a) ? a : 0.0; }

/* ---- coefficients (src/coefficients.cpp) ---- */

/* in_boundary_band: coefficients.cpp:10-13 (j uses N_halo_y, i uses N_halo_x). */
int orc_in_boundary_band(const sgpu_params_t* p, int i, int j) {
    return j == p->N_halo_y + 1 || j == p->NY + p->N_halo_y || i == p->NX + p->N_halo_x - 1 ||
           i == p->N_halo_x;
}

/* convective_coefficients: coefficients.cpp:15-39. */
void orc_convective(const sgpu_params_t* p, double ue, double uw, double vn, double vs, int i,
                    int j, double c[9]) {
    const double dx = p->dx, dy = p->dy;
    if (p->convection_scheme == SGPU_UDS || orc_in_boundary_band(p, i, j)) {
        c[AE] = dy * mx(-ue);
        c[AW] = dy * mx(uw);
        c[AN] = dx * mx(-vn);
        c[AS] = dx * mx(vs);
        c[AEE] = c[AWW] = c[ANN] = c[ASS] = 0.0;
    } else {
        c[AE] = -dy * (-0.75 * mx(-ue) + 0.375 * mx(ue) - 0.125 * mx(-uw));
        c[AW] = -dy * (-0.125 * mx(ue) + 0.375 * mx(-uw) - 0.75 * mx(uw));
        c[AN] = -dx * (-0.75 * mx(-vn) + 0.375 * mx(vn) - 0.125 * mx(-vs));
        c[AS] = -dx * (-0.125 * mx(vn) + 0.375 * mx(-vn) - 0.75 * mx(vs));
        c[AEE] = -0.125 * dy * mx(-ue);
        c[AWW] = -0.125 * dy * mx(uw);
        c[ANN] = -0.125 * dx * mx(-vn);
        c[ASS] = -0.125 * dx * mx(vs);
    }
    /* AP sums S, W, N, E, then the far links (coefficients.cpp:26, 36). */
    c[AP] = c[AS] + c[AW] + c[AN] + c[AE] + c[ASS] + c[AWW] + c[ANN] + c[AEE];
}

/* diffusive_coefficients: coefficients.cpp:41-63. */
void orc_diffusive(const sgpu_params_t* p, int i, int j, double c[9]) {
    const double dx = p->dx, dy = p->dy, nu = p->nu;
    if (p->diffusion_order == 2 || orc_in_boundary_band(p, i, j)) {
        c[AE] = dy * nu / dx;
        c[AW] = dy * nu / dx;
        c[AN] = dx * nu / dy;
        c[AS] = dx * nu / dy;
        c[AEE] = c[AWW] = c[ANN] = c[ASS] = 0.0;
        c[AP] = -nu * (-2 * dx / dy - 2 * dy / dx);
    } else {
        c[AE] = 4.0 / 3 * dy * nu / dx;
        c[AW] = 4.0 / 3 * dy * nu / dx;
        c[AN] = 4.0 / 3 * dx * nu / dy;
        c[AS] = 4.0 / 3 * dx * nu / dy;
        c[AEE] = -1.0 / 12 * dy * nu / dx;
        c[AWW] = -1.0 / 12 * dy * nu / dx;
        c[ANN] = -1.0 / 12 * dx * nu / dy;
        c[ASS] = -1.0 / 12 * dx * nu / dy;
        c[AP] = -nu * (-2.5 * dx / dy - 2.5 * dy / dx);
    }
}

/* Coeffs::set(conv + diff): coefficients.cpp:5-8 and 72-82. */
static void set_coef(double* const* co, size_t q, const double* a, const double* b) {
    for (int k = 0; k < NCOEF; ++k)
        co[k][q] = a[k] + b[k];
}

/* ---- ordered sums ---- */

double orc_ordered_sum(const double* v, int nr, int nc) {
    double s = 0.0;
    for (int r = 0; r < nr; ++r) {
        double row = 0.0;
        for (int c = 0; c < nc; ++c)
            row += v[(size_t)r * nc + c];
        s += row;
    }
    return s;
}

/* ---- u-momentum (src/momentum_u.cpp) ---- */

/* assemble_u: momentum_u.cpp:8-22. */
void orc_assemble_u(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    double cc[9], cd[9];
    for (int i = p->NX + H - 1; i >= H; --i)
        for (int j = H; j <= p->NY + H; ++j) {
            double ue = (s->u[IX(s, i, j)] + s->u[IX(s, i, j + 1)]) / 2;
            double uw = (s->u[IX(s, i, j)] + s->u[IX(s, i, j - 1)]) / 2;
            double vn = (s->v[IX(s, i, j)] + s->v[IX(s, i, j + 1)]) / 2;
            double vs = (s->v[IX(s, i + 1, j)] + s->v[IX(s, i + 1, j + 1)]) / 2;
            orc_convective(p, ue, uw, vn, vs, i, j, cc);
            orc_diffusive(p, i, j, cd);
            set_coef(s->cu, IX(s, i, j), cc, cd);
        }
}

/* apply_bc_u: momentum_u.cpp:24-34. */
void orc_bc_u(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    for (int j = H + 1; j <= p->NY + H; ++j)
        s->u[IX(s, H - 1, j)] = 2 - s->u[IX(s, H, j)];
    for (int j = H + 1; j <= p->NY + H; ++j)
        s->u[IX(s, p->NX + H, j)] = -s->u[IX(s, p->NX + H - 1, j)];
}

/* nb_sum: momentum_u.cpp:36-41 (near four, then far four). */
static inline double nb_sum(double* const* c, const double* f, size_t q, size_t nc) {
    return (c[AE][q] * f[q + 1] + c[AW][q] * f[q - 1] + c[AN][q] * f[q - nc] +
            c[AS][q] * f[q + nc]) +
           (c[AEE][q] * f[q + 2] + c[AWW][q] * f[q - 2] + c[ANN][q] * f[q - 2 * nc] +
            c[ASS][q] * f[q + 2 * nc]);
}

/* near_sum: momentum_u.cpp:84-87 (2-colour case: far cells are not read). */
static inline double near_sum(double* const* c, const double* f, size_t q, size_t nc) {
    return c[AE][q] * f[q + 1] + c[AW][q] * f[q - 1] + c[AN][q] * f[q - nc] + c[AS][q] * f[q + nc];
}

/* residual_u: momentum_u.cpp:43-59, summed in CellSums order. */
double orc_residual_u(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const size_t nc = (size_t)p->ncols;
    double total = 0.0;
    for (int i = H; i <= p->NX + H - 1; ++i) {
        double res = 0.0;
        for (int j = H + 1; j <= p->NY + H - 1; ++j) {
            const size_t q = IX(s, i, j);
            double R = nb_sum(s->cu, s->u, q, nc) + (s->pf[q] - s->pf[q + 1]) * p->dy -
                       s->cu[AP][q] * s->u[q];
            res += fabs(R);
        }
        total += res;
    }
    return total;
}

/* momentum_colours / momentum_colour: momentum_u.cpp:70-72, momentum_u.hpp:15-17. */
static int momentum_colours(const sgpu_params_t* p) {
    return (p->convection_scheme == SGPU_UDS && p->diffusion_order == 2) ? 2 : 5;
}
static inline int momentum_colour(int ncol, int i, int j) {
    return ncol == 2 ? (i + j) % 2 : (i + 3 * j) % 5;
}

/* sweep_u_gs_lex: momentum_u.cpp:61-68 (rows descending, columns ascending, in place). */
static void sweep_u_gs_lex(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const double a = p->relaxation_factor_u;
    const size_t nc = (size_t)p->ncols;
    for (int i = p->NX + H - 1; i >= H; --i)
        for (int j = H + 1; j <= p->NY + H - 1; ++j) {
            const size_t q = IX(s, i, j);
            s->u[q] = a * (nb_sum(s->cu, s->u, q, nc) + (s->pf[q] - s->pf[q + 1]) * p->dy) /
                          s->cu[AP][q] +
                      (1 - a) * s->u[q];
        }
}

/* sweep_u_jacobi_batch: momentum_u.cpp:89-116 (one copy, then alternating buffers). */
static void sweep_u_jacobi_batch(orc_state* s, int nsweeps) {
    if (nsweeps <= 0)
        return;
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const double a = p->relaxation_factor_u;
    const size_t nc = (size_t)p->ncols;
    memcpy(s->scratch, s->u, s->n * sizeof(double));
    for (int k = 0; k < nsweeps; ++k) {
        const int to_u = (nsweeps - k) % 2 == 1;
        const double* src = to_u ? s->scratch : s->u;
        double* dst = to_u ? s->u : s->scratch;
        for (int i = p->NX + H - 1; i >= H; --i)
            for (int j = H + 1; j <= p->NY + H - 1; ++j) {
                const size_t q = IX(s, i, j);
                dst[q] = a * (nb_sum(s->cu, src, q, nc) + (s->pf[q] - s->pf[q + 1]) * p->dy) /
                             s->cu[AP][q] +
                         (1 - a) * src[q];
            }
    }
}

/* sweep_u_multicolour_batch: momentum_u.cpp:123-143 (colours in order, in place). */
static void sweep_u_multicolour_batch(orc_state* s, int nsweeps) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H, ncol = momentum_colours(p);
    const double a = p->relaxation_factor_u;
    const size_t nc = (size_t)p->ncols;
    for (int sw = 0; sw < nsweeps; ++sw)
        for (int c = 0; c < ncol; ++c)
            for (int i = p->NX + H - 1; i >= H; --i)
                for (int j = H + 1; j <= p->NY + H - 1; ++j) {
                    if (momentum_colour(ncol, i, j) != c)
                        continue;
                    const size_t q = IX(s, i, j);
                    const double nb =
                        ncol == 2 ? near_sum(s->cu, s->u, q, nc) : nb_sum(s->cu, s->u, q, nc);
                    s->u[q] = a * (nb + (s->pf[q] - s->pf[q + 1]) * p->dy) / s->cu[AP][q] +
                              (1 - a) * s->u[q];
                }
}

/* sweep_u_batch: momentum_u.cpp:162-171. */
void orc_sweep_u(orc_state* s, int nsweeps) {
    if (s->p.momentum_solver == SGPU_MOM_JACOBI)
        sweep_u_jacobi_batch(s, nsweeps);
    else if (s->p.momentum_solver == SGPU_MOM_GS_MULTICOLOUR)
        sweep_u_multicolour_batch(s, nsweeps);
    else
        for (int k = 0; k < nsweeps; ++k)
            sweep_u_gs_lex(s);
}

/* ---- v-momentum (src/momentum_v.cpp) ---- */

/* assemble_v: momentum_v.cpp:9-22. */
void orc_assemble_v(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    double cc[9], cd[9];
    for (int i = p->NX + H + 1; i >= H; --i)
        for (int j = H; j <= p->NY + H + 1; ++j) {
            const double ue = (s->u[IX(s, i - 1, j)] + s->u[IX(s, i, j)]) / 2;
            const double uw = (s->u[IX(s, i, j - 1)] + s->u[IX(s, i - 1, j - 1)]) / 2;
            const double vn = (s->v[IX(s, i, j)] + s->v[IX(s, i - 1, j)]) / 2;
            const double vs = (s->v[IX(s, i, j)] + s->v[IX(s, i + 1, j)]) / 2;
            orc_convective(p, ue, uw, vn, vs, i, j, cc);
            orc_diffusive(p, i, j, cd);
            set_coef(s->cv, IX(s, i, j), cc, cd);
        }
}

/* apply_bc_v: momentum_v.cpp:24-34. */
void orc_bc_v(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    for (int i = H; i <= p->NX + H - 1; ++i)
        s->v[IX(s, i, H)] = -s->v[IX(s, i, H + 1)];
    for (int i = H; i <= p->NX + H - 1; ++i)
        s->v[IX(s, i, p->NY + H + 1)] = -s->v[IX(s, i, p->NY + H)];
}

/* residual_v: momentum_v.cpp:36-55 (the neighbour sum written inline, same order as nb_sum). */
double orc_residual_v(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const size_t nc = (size_t)p->ncols;
    double total = 0.0;
    for (int i = H + 1; i <= p->NX + H - 1; ++i) {
        double res = 0.0;
        for (int j = H + 1; j <= p->NY + H; ++j) {
            const size_t q = IX(s, i, j);
            const double R = nb_sum(s->cv, s->v, q, nc) + (s->pf[q] - s->pf[q - nc]) * p->dx -
                             s->cv[AP][q] * s->v[q];
            res += fabs(R);
        }
        total += res;
    }
    return total;
}

/* sweep_v_gs_lex: momentum_v.cpp:57-70. */
static void sweep_v_gs_lex(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const double av = p->relaxation_factor_v;
    const size_t nc = (size_t)p->ncols;
    for (int i = p->NX + H - 1; i >= H + 1; --i)
        for (int j = H + 1; j <= p->NY + H; ++j) {
            const size_t q = IX(s, i, j);
            s->v[q] = av * (nb_sum(s->cv, s->v, q, nc) + (s->pf[q] - s->pf[q - nc]) * p->dx) /
                          s->cv[AP][q] +
                      (1 - av) * s->v[q];
        }
}

/* sweep_v_jacobi_batch: momentum_v.cpp:85-114. */
static void sweep_v_jacobi_batch(orc_state* s, int nsweeps) {
    if (nsweeps <= 0)
        return;
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const double av = p->relaxation_factor_v;
    const size_t nc = (size_t)p->ncols;
    memcpy(s->scratch, s->v, s->n * sizeof(double));
    for (int k = 0; k < nsweeps; ++k) {
        const int to_v = (nsweeps - k) % 2 == 1;
        const double* src = to_v ? s->scratch : s->v;
        double* dst = to_v ? s->v : s->scratch;
        for (int i = p->NX + H - 1; i >= H + 1; --i)
            for (int j = H + 1; j <= p->NY + H; ++j) {
                const size_t q = IX(s, i, j);
                dst[q] = av * (nb_sum(s->cv, src, q, nc) + (s->pf[q] - s->pf[q - nc]) * p->dx) /
                             s->cv[AP][q] +
                         (1 - av) * src[q];
            }
    }
}

/* sweep_v_multicolour_batch: momentum_v.cpp:121-145. */
static void sweep_v_multicolour_batch(orc_state* s, int nsweeps) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H, ncol = momentum_colours(p);
    const double av = p->relaxation_factor_v;
    const size_t nc = (size_t)p->ncols;
    for (int sw = 0; sw < nsweeps; ++sw)
        for (int c = 0; c < ncol; ++c)
            for (int i = p->NX + H - 1; i >= H + 1; --i)
                for (int j = H + 1; j <= p->NY + H; ++j) {
                    if (momentum_colour(ncol, i, j) != c)
                        continue;
                    const size_t q = IX(s, i, j);
                    const double nb =
                        ncol == 2 ? near_sum(s->cv, s->v, q, nc) : nb_sum(s->cv, s->v, q, nc);
                    s->v[q] = av * (nb + (s->pf[q] - s->pf[q - nc]) * p->dx) / s->cv[AP][q] +
                              (1 - av) * s->v[q];
                }
}

/* sweep_v_batch: momentum_v.cpp:164-173. */
void orc_sweep_v(orc_state* s, int nsweeps) {
    if (s->p.momentum_solver == SGPU_MOM_JACOBI)
        sweep_v_jacobi_batch(s, nsweeps);
    else if (s->p.momentum_solver == SGPU_MOM_GS_MULTICOLOUR)
        sweep_v_multicolour_batch(s, nsweeps);
    else
        for (int k = 0; k < nsweeps; ++k)
            sweep_v_gs_lex(s);
}

/* ---- pressure correction (src/pressure.cpp) ---- */

/* assemble_p: pressure.cpp:14-54. */
double orc_assemble_p(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H, NX = p->NX, NY = p->NY;
    const double dx = p->dx, dy = p->dy;
    const size_t nc = (size_t)p->ncols;
    const double* APU = s->cu[AP];
    const double* APV = s->cv[AP];
    for (int i = H; i <= NX + H - 1; ++i)
        for (int j = H + 1; j <= NY + H; ++j) {
            const size_t q = IX(s, i, j);
            s->AEP[q] = dy * dy / APU[q];
            s->AWP[q] = dy * dy / APU[q - 1];
            s->ANP[q] = dx * dx / APV[q];
            s->ASP[q] = dx * dx / APV[q + nc];
        }
    for (int i = 0; i <= p->nrows - 1; ++i) {
        s->AWP[IX(s, i, H + 1)] = 0.0;
        s->AEP[IX(s, i, NY + H)] = 0.0;
    }
    for (int j = 0; j <= p->ncols - 1; ++j)
        s->ASP[IX(s, NX + H - 1, j)] = 0.0;
    for (int j = 0; j <= p->ncols - 1; ++j)
        s->ANP[IX(s, H, j)] = 0.0;
    double total = 0.0;
    for (int i = H; i <= NX + H - 1; ++i) {
        double res = 0.0;
        for (int j = H + 1; j <= NY + H; ++j) {
            const size_t q = IX(s, i, j);
            s->APP[q] = s->AEP[q] + s->AWP[q] + s->ANP[q] + s->ASP[q];
            s->b[q] = -dx * (-s->v[q + nc] + s->v[q]) - dy * (-s->u[q - 1] + s->u[q]);
            res += fabs(s->b[q]);
        }
        total += res;
    }
    return total;
}

/* Two-statement p' update (pressure.cpp:70-75), neighbours E, W, S, N from src. */
static inline void pc_update(orc_state* s, double* dst, const double* src, size_t q, size_t nc) {
    dst[q] = s->b[q] / s->APP[q];
    dst[q] += (s->AEP[q] * src[q + 1] + s->AWP[q] * src[q - 1] + s->ASP[q] * src[q + nc] +
               s->ANP[q] * src[q - nc]) /
              s->APP[q];
}

/* solve_pc_gs_lex: pressure.cpp:56-67. */
static void solve_pc_gs_lex(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const size_t nc = (size_t)p->ncols;
    memset(s->pc, 0, s->n * sizeof(double));
    for (int k = 0; k < p->maxit_inner_p; ++k)
        for (int i = p->NX + H - 1; i >= H; --i)
            for (int j = H + 1; j <= p->NY + H; ++j)
                pc_update(s, s->pc, s->pc, IX(s, i, j), nc);
}

/* solve_pc_jacobi: pressure.cpp:77-112 (weight kPcJacobiWeight = 0.8, pressure.hpp:25). */
static void solve_pc_jacobi(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H, n = p->maxit_inner_p;
    const size_t nc = (size_t)p->ncols;
    const double w = 0.8;
    memset(s->pc, 0, s->n * sizeof(double));
    memcpy(s->scratch, s->pc, s->n * sizeof(double));
    for (int k = 0; k < n; ++k) {
        const int to_pc = (n - k) % 2 == 1;
        const double* src = to_pc ? s->scratch : s->pc;
        double* dst = to_pc ? s->pc : s->scratch;
        for (int i = p->NX + H - 1; i >= H; --i)
            for (int j = H + 1; j <= p->NY + H; ++j) {
                const size_t q = IX(s, i, j);
                pc_update(s, dst, src, q, nc);
                dst[q] = w * dst[q] + (1 - w) * src[q];
            }
    }
}

/* solve_pc_redblack: pressure.cpp:114-134; colour c = (i + j) & 1, colour 0 first. */
static void solve_pc_redblack(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const size_t nc = (size_t)p->ncols;
    memset(s->pc, 0, s->n * sizeof(double));
    for (int k = 0; k < p->maxit_inner_p; ++k)
        for (int c = 0; c < 2; ++c)
            for (int i = p->NX + H - 1; i >= H; --i)
                for (int j = H + 1 + ((i + H + 1 + c) & 1); j <= p->NY + H; j += 2)
                    pc_update(s, s->pc, s->pc, IX(s, i, j), nc);
}

/* correct: pressure.cpp:136-157. */
void orc_correct(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H, NX = p->NX, NY = p->NY;
    const double dy = p->dy, ap = p->relaxation_factor_p;
    const size_t nc = (size_t)p->ncols;
    const double* APU = s->cu[AP];
    const double* APV = s->cv[AP];
    for (int i = H; i <= NX + H - 1; ++i)
        for (int j = H + 1; j <= NY + H - 1; ++j) {
            const size_t q = IX(s, i, j);
            s->u[q] += dy * (s->pc[q] - s->pc[q + 1]) / APU[q];
        }
    for (int i = H + 1; i <= NX + H - 1; ++i)
        for (int j = H + 1; j <= NY + H; ++j) {
            const size_t q = IX(s, i, j);
            s->v[q] += p->dx * (s->pc[q] - s->pc[q - nc]) / APV[q];
        }
    for (int i = H; i <= NX + H - 1; ++i)
        for (int j = H + 1; j <= NY + H; ++j) {
            const size_t q = IX(s, i, j);
            s->pf[q] += ap * s->pc[q];
        }
}

/* ---- conjugate gradient (pressure.cpp:165-317) ---- */

/* cg_sums<K>: per-cell values f(i, j) summed in CellSums order (pressure.cpp:178-206). The callback
 * form is replaced by an explicit kind switch. */
enum { CG_SUM_B, CG_SUM_INIT, CG_SUM_DQ, CG_SUM_UPDATE, CG_SUM_X };

static void cg_pass(orc_state* s, int kind, double mb, double alpha, int K, double* out) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const size_t nc = (size_t)p->ncols;
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    double *r = s->cg_r, *z = s->cg_z, *d = s->cg_d, *q_ = s->cg_q, *x = s->pc;
    for (int i = H; i <= p->NX + H - 1; ++i) {
        double sr[4] = {0.0, 0.0, 0.0, 0.0}, v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int j = H + 1; j <= p->NY + H; ++j) {
            const size_t q = IX(s, i, j);
            if (kind == CG_SUM_B) {
                v[0] = s->b[q];
            } else if (kind == CG_SUM_INIT) {
                const double ri = s->b[q] - mb;
                r[q] = ri;
                const double zi = ri / s->APP[q];
                z[q] = zi;
                v[0] = ri * ri;
                v[1] = zi;
                v[2] = ri * zi;
                v[3] = ri;
            } else if (kind == CG_SUM_DQ) {
                const double qi = s->APP[q] * d[q] - (s->AEP[q] * d[q + 1] + s->AWP[q] * d[q - 1] +
                                                      s->ASP[q] * d[q + nc] + s->ANP[q] * d[q - nc]);
                q_[q] = qi;
                v[0] = d[q] * qi;
            } else if (kind == CG_SUM_UPDATE) {
                x[q] += alpha * d[q];
                const double ri = r[q] - alpha * q_[q];
                r[q] = ri;
                const double zi = ri / s->APP[q];
                z[q] = zi;
                v[0] = ri * ri;
                v[1] = zi;
                v[2] = ri * zi;
                v[3] = ri;
            } else {
                v[0] = x[q];
            }
            for (int m = 0; m < K; ++m)
                sr[m] += v[m];
        }
        for (int m = 0; m < K; ++m)
            tot[m] += sr[m];
    }
    for (int m = 0; m < K; ++m)
        out[m] = tot[m];
}

/* solve_pc_cg: pressure.cpp:208-317. Returns the iteration count. */
static int solve_pc_cg(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    const double n = (double)p->NX * p->NY;
    double *d = s->cg_d, *z = s->cg_z, *x = s->pc;
    s->cg_last_iters = 0;
    s->cg_last_rel = 0.0;
    memset(x, 0, s->n * sizeof(double));
    double sb = 0.0;
    cg_pass(s, CG_SUM_B, 0.0, 0.0, 1, &sb);
    const double mb = sb / n;
    double s4[4];
    cg_pass(s, CG_SUM_INIT, mb, 0.0, 4, s4);
    double rr = s4[0], sz = s4[1], rz = s4[2], sr = s4[3];
    if (rr == 0.0)
        return 0;
    const double nb = sqrt(rr);
    double mz = sz / n;
    rz -= mz * sr;
    for (int i = H; i <= p->NX + H - 1; ++i)
        for (int j = H + 1; j <= p->NY + H; ++j) {
            const size_t q = IX(s, i, j);
            d[q] = z[q] - mz;
        }
    int k = 0;
    double rel = 1.0;
    while (k < p->pressure_maxit) {
        double dq = 0.0;
        cg_pass(s, CG_SUM_DQ, 0.0, 0.0, 1, &dq);
        if (!(dq > 0.0))
            break;
        const double alpha = rz / dq;
        cg_pass(s, CG_SUM_UPDATE, 0.0, alpha, 4, s4);
        rr = s4[0];
        sz = s4[1];
        double rzn = s4[2];
        sr = s4[3];
        ++k;
        rel = sqrt(rr) / nb;
        if (rel <= p->pressure_tolerance)
            break;
        mz = sz / n;
        rzn -= mz * sr;
        const double beta = rzn / rz;
        rz = rzn;
        for (int i = H; i <= p->NX + H - 1; ++i)
            for (int j = H + 1; j <= p->NY + H; ++j) {
                const size_t q = IX(s, i, j);
                d[q] = (z[q] - mz) + beta * d[q];
            }
    }
    double sx = 0.0;
    cg_pass(s, CG_SUM_X, 0.0, 0.0, 1, &sx);
    const double mxv = sx / n;
    for (int i = H; i <= p->NX + H - 1; ++i)
        for (int j = H + 1; j <= p->NY + H; ++j)
            x[IX(s, i, j)] -= mxv;
    s->cg_last_iters = k;
    s->cg_last_rel = rel;
    return k;
}

/* ---- geometric multigrid (src/multigrid.cpp) ---- */

/* mg_level_dims: multigrid.cpp:143-151. */
int orc_mg_level_dims(int nx, int ny, int* dims) {
    int n = 0;
    dims[2 * n] = nx;
    dims[2 * n + 1] = ny;
    ++n;
    while (nx % 2 == 0 && ny % 2 == 0 && nx / 2 >= 4 && ny / 2 >= 4 && n < 64) {
        nx /= 2;
        ny /= 2;
        dims[2 * n] = nx;
        dims[2 * n + 1] = ny;
        ++n;
    }
    return n;
}

/* det_sum: multigrid.cpp:18-34 (rows left to right, then rows in order). */
static double det_sum_sq(const orc_level* L, const double* f) {
    double s = 0.0;
    for (int I = 0; I < L->nx; ++I) {
        double r = 0.0;
        for (int J = 0; J < L->ny; ++J) {
            const double a = f[I * L->stride + J];
            r += a * a;
        }
        s += r;
    }
    return s;
}
static double det_sum_val(const orc_level* L, const double* f) {
    double s = 0.0;
    for (int I = 0; I < L->nx; ++I) {
        double r = 0.0;
        for (int J = 0; J < L->ny; ++J)
            r += f[I * L->stride + J];
        s += r;
    }
    return s;
}

/* smooth: multigrid.cpp:46-70; colour (I + J) & 1 with I0 = J0 = 0, colour 0 first. */
static void mg_smooth(const orc_level* L, int sweeps) {
    const int st = L->stride;
    double* x = L->x;
    for (int sw = 0; sw < sweeps; ++sw)
        for (int c = 0; c < 2; ++c)
            for (int I = L->nx - 1; I >= 0; --I)
                for (int J = (I + c) & 1; J < L->ny; J += 2) {
                    const int q = I * st + J;
                    x[q] = L->b[q] / L->AP[q];
                    x[q] += (L->AE[q] * x[q + 1] + L->AW[q] * x[q - 1] + L->AS[q] * x[q + st] +
                             L->AN[q] * x[q - st]) /
                            L->AP[q];
                }
}

/* residual: multigrid.cpp:73-87. */
static void mg_residual(const orc_level* L) {
    const int st = L->stride;
    const double* x = L->x;
    for (int I = L->nx - 1; I >= 0; --I)
        for (int J = 0; J < L->ny; ++J) {
            const int q = I * st + J;
            L->r[q] = L->b[q] - (L->AP[q] * x[q] - (L->AE[q] * x[q + 1] + L->AW[q] * x[q - 1] +
                                                    L->AS[q] * x[q + st] + L->AN[q] * x[q - st]));
        }
}

/* restrict_residual: multigrid.cpp:90-103. */
static void mg_restrict(const orc_level* F, const orc_level* C) {
    const int fs = F->stride, cs = C->stride;
    for (int I = F->nx / 2 - 1; I >= 0; --I)
        for (int J = 0; J < F->ny / 2; ++J) {
            const int f = 2 * I * fs + 2 * J;
            C->b[I * cs + J] = F->r[f] + F->r[f + 1] + F->r[f + fs] + F->r[f + fs + 1];
            C->x[I * cs + J] = 0.0;
        }
}

/* prolong: multigrid.cpp:106-116. */
static void mg_prolong(const orc_level* C, const orc_level* F, double omega) {
    const int fs = F->stride, cs = C->stride;
    for (int i = F->nx - 1; i >= 0; --i)
        for (int j = 0; j < F->ny; ++j)
            F->x[i * fs + j] += omega * C->x[(i / 2) * cs + j / 2];
}

/* mg_remove_mean: multigrid.cpp:327-345 form used on a level (m = det_sum / (nx * ny)). */
static void mg_remove_mean(const orc_level* L, double* x) {
    const double m = det_sum_val(L, x) / ((double)L->nx * L->ny);
    for (int I = L->nx - 1; I >= 0; --I)
        for (int J = 0; J < L->ny; ++J)
            x[I * L->stride + J] -= m;
}

/* coarse_solve: multigrid.cpp:120-140 (tolerance 1e-10, at most 200 sweeps). */
static void mg_coarse_solve(orc_state* s, const orc_level* L) {
    mg_remove_mean(L, L->b);
    const double bb = det_sum_sq(L, L->b);
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        while (sweeps < 200) {
            mg_smooth(L, 1);
            ++sweeps;
            mg_residual(L);
            const double rr = det_sum_sq(L, L->r);
            if (sqrt(rr) < 1e-10 * bn)
                break;
        }
    }
    mg_remove_mean(L, L->x);
    s->last_coarse_sweeps = sweeps;
}

/* mg_build: multigrid.cpp:232-261 (Galerkin 2x2 aggregation). */
void orc_mg_build(orc_state* s) {
    for (int l = 1; l < s->nlev; ++l) {
        const orc_level* F = &s->lev[l - 1];
        const orc_level* C = &s->lev[l];
        const int fs = F->stride, cs = C->stride;
        for (int I = F->nx / 2 - 1; I >= 0; --I)
            for (int J = 0; J < F->ny / 2; ++J) {
                const int f = 2 * I * fs + 2 * J, c = I * cs + J;
                const double ae = F->AE[f + 1] + F->AE[f + fs + 1];
                const double aw = F->AW[f] + F->AW[f + fs];
                const double an = F->AN[f] + F->AN[f + 1];
                const double as = F->AS[f + fs] + F->AS[f + fs + 1];
                C->AE[c] = ae;
                C->AW[c] = aw;
                C->AN[c] = an;
                C->AS[c] = as;
                C->AP[c] = ae + aw + an + as;
            }
    }
}

/* mg_vcycle: multigrid.cpp:299-323. */
void orc_mg_vcycle(orc_state* s) {
    const sgpu_params_t* p = &s->p;
    const int nl = s->nlev;
    for (int l = 0; l + 1 < nl; ++l) {
        mg_smooth(&s->lev[l], p->mg_pre);
        mg_residual(&s->lev[l]);
        mg_restrict(&s->lev[l], &s->lev[l + 1]);
    }
    mg_coarse_solve(s, &s->lev[nl - 1]);
    for (int l = nl - 2; l >= 0; --l) {
        mg_prolong(&s->lev[l + 1], &s->lev[l], p->mg_omega);
        mg_smooth(&s->lev[l], p->mg_post);
    }
}

/* remove_mean0: multigrid.cpp:327-345 on level 0 (CellSums order over the p' interior). */
static void remove_mean0(orc_state* s, double* f) {
    const sgpu_params_t* p = &s->p;
    const int H = p->H;
    double tot = 0.0;
    for (int i = H; i <= p->NX + H - 1; ++i) {
        double r = 0.0;
        for (int j = H + 1; j <= p->NY + H; ++j)
            r += f[IX(s, i, j)];
        tot += r;
    }
    const double m = tot / ((double)p->NX * p->NY);
    for (int i = H; i <= p->NX + H - 1; ++i)
        for (int j = H + 1; j <= p->NY + H; ++j)
            f[IX(s, i, j)] -= m;
}

/* solve_pc_mg: multigrid.cpp:347-357. */
static void solve_pc_mg(orc_state* s) {
    orc_mg_build(s);
    memset(s->pc, 0, s->n * sizeof(double));
    remove_mean0(s, s->b);
    for (int c = 0; c < s->p.mg_cycles; ++c)
        orc_mg_vcycle(s);
    remove_mean0(s, s->pc);
}

/* outer_iteration's solve_p dispatch: solver.cpp:63-76. */
void orc_solve_p(orc_state* s) {
    switch (s->p.pressure_solver) {
    case SGPU_P_JACOBI: solve_pc_jacobi(s); break;
    case SGPU_P_GS_REDBLACK: solve_pc_redblack(s); break;
    case SGPU_P_CG: solve_pc_cg(s); break;
    case SGPU_P_MG: solve_pc_mg(s); break;
    default: solve_pc_gs_lex(s); break;
    }
}

/* outer_iteration: solver.cpp:27-93 (one rank: every halo exchange is a no-op). */
void orc_outer_iteration(orc_state* s, double res[3]) {
    orc_assemble_u(s);
    orc_bc_u(s);
    res[0] = orc_residual_u(s);
    orc_sweep_u(s, s->p.maxit_inner_u);
    orc_assemble_v(s);
    orc_bc_v(s);
    res[1] = orc_residual_v(s);
    orc_sweep_v(s, s->p.maxit_inner_v);
    res[2] = orc_assemble_p(s);
    orc_solve_p(s);
    orc_correct(s);
}

/* run_outer_loop: solver.cpp:106-132. max of three via std::max({...}) semantics: the first
 * element wins unless a later one compares greater. */
int orc_run(orc_state* s, int maxit, double* log, int* converged) {
    const sgpu_params_t* p = &s->p;
    double mu = 0.0, mv = 0.0, mp = 0.0;
    int iter, it_done = 0;
    *converged = 0;
    for (iter = 1; iter <= maxit; ++iter) {
        double r[3];
        orc_outer_iteration(s, r);
        if (log) {
            log[4 * (iter - 1) + 0] = (double)iter;
            log[4 * (iter - 1) + 1] = r[0];
            log[4 * (iter - 1) + 2] = r[1];
            log[4 * (iter - 1) + 3] = r[2];
        }
        it_done = iter;
        double tu = r[0], tv = r[1], tp = r[2];
        if (p->residual_normalisation == SGPU_NORM_RUNNING_MAX) {
            mu = mu < r[0] ? r[0] : mu;
            mv = mv < r[1] ? r[1] : mv;
            mp = mp < r[2] ? r[2] : mp;
            tu = mu > 0.0 ? r[0] / mu : 0.0;
            tv = mv > 0.0 ? r[1] / mv : 0.0;
            tp = mp > 0.0 ? r[2] / mp : 0.0;
        }
        double m = tu;
        if (m < tv)
            m = tv;
        if (m < tp)
            m = tp;
        if (m <= p->error_tolerance && iter > 1) {
            *converged = 1;
            break;
        }
    }
    return it_done;
}

/* ---- state ---- */

orc_state* orc_create(const sgpu_params_t* p) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s)
        return NULL;
    s->p = *p;
    s->n = (size_t)p->nrows * (size_t)p->ncols;
    s->u = zalloc(s->n);
    s->v = zalloc(s->n);
    s->pf = zalloc(s->n);
    for (int k = 0; k < NCOEF; ++k) {
        s->cu[k] = zalloc(s->n);
        s->cv[k] = zalloc(s->n);
    }
    s->AEP = zalloc(s->n);
    s->AWP = zalloc(s->n);
    s->ANP = zalloc(s->n);
    s->ASP = zalloc(s->n);
    s->APP = zalloc(s->n);
    s->b = zalloc(s->n);
    s->pc = zalloc(s->n);
    s->scratch = zalloc(s->n);
    s->cg_r = zalloc(s->n);
    s->cg_z = zalloc(s->n);
    s->cg_d = zalloc(s->n);
    s->cg_q = zalloc(s->n);
    s->mg_r0 = zalloc(s->n);
    /* MGWork: multigrid.cpp:153-185 and mg_view: multigrid.cpp:187-220. */
    int dims[128];
    s->nlev = orc_mg_level_dims(p->NX, p->NY, dims);
    for (int l = 0; l < s->nlev; ++l) {
        orc_level* L = &s->lev[l];
        L->nx = dims[2 * l];
        L->ny = dims[2 * l + 1];
        if (l == 0) {
            const size_t base = (size_t)p->H * p->ncols + p->H + 1;
            L->stride = p->ncols;
            L->AE = s->AEP + base;
            L->AW = s->AWP + base;
            L->AN = s->ANP + base;
            L->AS = s->ASP + base;
            L->AP = s->APP + base;
            L->b = s->b + base;
            L->x = s->pc + base;
            L->r = s->mg_r0 + base;
        } else {
            const size_t n = (size_t)(L->nx + 2) * (L->ny + 2);
            for (int k = 0; k < 8; ++k)
                L->mem[k] = zalloc(n);
            L->stride = L->ny + 2;
            const size_t base = (size_t)L->stride + 1;
            L->AE = L->mem[0] + base;
            L->AW = L->mem[1] + base;
            L->AN = L->mem[2] + base;
            L->AS = L->mem[3] + base;
            L->AP = L->mem[4] + base;
            L->b = L->mem[5] + base;
            L->x = L->mem[6] + base;
            L->r = L->mem[7] + base;
        }
    }
    return s;
}

void orc_destroy(orc_state* s) {
    if (!s)
        return;
    free(s->u);
    free(s->v);
    free(s->pf);
    for (int k = 0; k < NCOEF; ++k) {
        free(s->cu[k]);
        free(s->cv[k]);
    }
    free(s->AEP);
    free(s->AWP);
    free(s->ANP);
    free(s->ASP);
    free(s->APP);
    free(s->b);
    free(s->pc);
    free(s->scratch);
    free(s->cg_r);
    free(s->cg_z);
    free(s->cg_d);
    free(s->cg_q);
    free(s->mg_r0);
    for (int l = 1; l < s->nlev; ++l)
        for (int k = 0; k < 8; ++k)
            free(s->lev[l].mem[k]);
    free(s);
}

static double* field_ptr(orc_state* s, int id) {
    if (id == SGPU_F_U) return s->u;
    if (id == SGPU_F_V) return s->v;
    if (id == SGPU_F_P) return s->pf;
    if (id >= SGPU_F_CU_AE && id <= SGPU_F_CU_AP) return s->cu[id - SGPU_F_CU_AE];
    if (id >= SGPU_F_CV_AE && id <= SGPU_F_CV_AP) return s->cv[id - SGPU_F_CV_AE];
    switch (id) {
    case SGPU_F_AEP: return s->AEP;
    case SGPU_F_AWP: return s->AWP;
    case SGPU_F_ANP: return s->ANP;
    case SGPU_F_ASP: return s->ASP;
    case SGPU_F_APP: return s->APP;
    case SGPU_F_B: return s->b;
    case SGPU_F_PC: return s->pc;
    default: return NULL;
    }
}

int orc_get(orc_state* s, int id, double* out) {
    double* f = field_ptr(s, id);
    if (!f)
        return -1;
    memcpy(out, f, s->n * sizeof(double));
    return 0;
}

int orc_set(orc_state* s, int id, const double* in) {
    double* f = field_ptr(s, id);
    if (!f)
        return -1;
    memcpy(f, in, s->n * sizeof(double));
    return 0;
}

int orc_mg_nlevels(orc_state* s) { return s->nlev; }
int orc_mg_last_coarse_sweeps(orc_state* s) { return s->last_coarse_sweeps; }
int orc_cg_last_iterations(orc_state* s) { return s->cg_last_iters; }
double orc_cg_last_rel_residual(orc_state* s) { return s->cg_last_rel; }

int orc_mg_get_level(orc_state* s, int l, int k, double* out) {
    if (l < 0 || l >= s->nlev || k < 0 || k > 7)
        return -1;
    const orc_level* L = &s->lev[l];
    const double* a[8] = {L->AE, L->AW, L->AN, L->AS, L->AP, L->b, L->x, L->r};
    for (int I = 0; I < L->nx; ++I)
        for (int J = 0; J < L->ny; ++J)
            out[(size_t)I * L->ny + J] = a[k][(size_t)I * L->stride + J];
    return 0;
}
