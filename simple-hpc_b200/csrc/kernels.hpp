// kernels.hpp — host-side launchers of the FP64 kernels (one translation unit per family).
#pragma once

#include "common.hpp"

#include <cuda_runtime.h>

namespace sgpu {

// ---- ordered sums (reduce.cu) ----
//
// K planes of nr x nc values (plane m at vals + m * plane_stride, row r at + r * ld) are summed in
// the reference's fixed order: each row left to right from 0.0, then the rows top to bottom from
// 0.0 (CellSums, src/decomp.cpp:176-205; det_sum, src/multigrid.cpp:18-34). out[m] receives plane
// m's sum. rows (K * nr doubles) and counter (one unsigned int, zero between calls) are scratch. If
// skip is non-null and *skip != 0 the launch does nothing (a finished iterative solve).
struct SumScratch {
    double* rows = nullptr;
    unsigned int* counter = nullptr;
    int max_rows = 0, max_k = 0;
};
void launch_ordered_sum(const double* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                        double* out, const SumScratch& s, const int* skip, cudaStream_t st);
// One plane in the same order with a small shared-memory footprint (a 3-tile ring, 25 KB): slower
// alone, but it can run on a second stream beside a kernel whose grid fills the SMs.
void launch_ordered_sum_lean(const double* vals, int ld, int nr, int nc, double* out, const SumScratch& s,
                             cudaStream_t st);
// Two sums of one plane in one pass: out[0] = sum of |v|, out[1] = sum of v, each in the order above
// (res_p and the mean of b from the field b itself, without compact copies).
void launch_ordered_sum_abs_pair(const double* vals, int ld, int nr, int nc, double* out, const SumScratch& s,
                                 cudaStream_t st);
// The same order over FP32 values, each widened to double before it is added.
void launch_ordered_sum(const float* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                        double* out, const SumScratch& s, const int* skip, cudaStream_t st);

// Deterministic FP64 tree sums (the mixed-precision path, which is not tied to the reference's
// rounding): a fixed shuffle tree per block, the blocks' partial sums added by one CTA in a fixed
// order. The same inputs and sizes give the same bits on every run.
// out0 = the sum of part[0 .. n), and for K = 2 also out1 = the sum of part[plane .. plane + n).
void launch_sum_partials(const double* part, int n, int K, int plane, double* out0, double* out1,
                         cudaStream_t st);
// *out = the sum of an nr x nc FP32 array (row stride ld) in FP64; part holds tree_sum_partials(nr,
// nc) doubles of scratch.
int tree_sum_partials(int nr, int nc);
void launch_tree_sum(const float* vals, int ld, int nr, int nc, double* part, double* out, cudaStream_t st);

// ---- momentum and pressure phases, reference-shaped (phases.cu) ----
struct Coef9Ptr {
    double* a[9]; // AE AW AN AS AEE AWW ANN ASS AP
};
struct PressurePtr {
    double *AEP, *AWP, *ANP, *ASP, *APP, *b, *pc;
};

void launch_assemble_u(const DevParams& p, const double* u, const double* v, Coef9Ptr cu,
                       cudaStream_t st);
void launch_assemble_v(const DevParams& p, const double* u, const double* v, Coef9Ptr cv,
                       cudaStream_t st);
void launch_bc_u(const DevParams& p, double* u, cudaStream_t st);
void launch_bc_v(const DevParams& p, double* v, cudaStream_t st);
// |R| of every residual cell into cells (compact rows of the residual range).
void launch_residual_u_cells(const DevParams& p, Coef9Ptr cu, const double* u, const double* pf,
                             double* cells, cudaStream_t st);
void launch_residual_v_cells(const DevParams& p, Coef9Ptr cv, const double* v, const double* pf,
                             double* cells, cudaStream_t st);
// One colour pass of the multicolour sweep (in place).
void launch_sweep_u_colour(const DevParams& p, Coef9Ptr cu, double* u, const double* pf, int colour,
                           cudaStream_t st);
void launch_sweep_v_colour(const DevParams& p, Coef9Ptr cv, double* v, const double* pf, int colour,
                           cudaStream_t st);
// One Jacobi pass src -> dst.
void launch_sweep_u_jacobi(const DevParams& p, Coef9Ptr cu, const double* src, double* dst,
                           const double* pf, cudaStream_t st);
void launch_sweep_v_jacobi(const DevParams& p, Coef9Ptr cv, const double* src, double* dst,
                           const double* pf, cudaStream_t st);
// assemble_p: links, wall zeros, APP, b and |b| into cells[0..), b into cells + plane (if two).
void launch_assemble_p(const DevParams& p, const double* APU, const double* APV, const double* u,
                       const double* v, PressurePtr w, double* cells_absb, double* cells_b,
                       cudaStream_t st);
// The links and APP of assemble_p without b (the mixed path keeps its p' operator in FP32 and forms
// the FP64 one only when a caller downloads it).
void launch_p_links_app(const DevParams& p, const double* APU, const double* APV, PressurePtr w,
                        cudaStream_t st);
void launch_pc_redblack(const DevParams& p, PressurePtr w, int colour, cudaStream_t st);
void launch_pc_jacobi(const DevParams& p, PressurePtr w, const double* src, double* dst,
                      cudaStream_t st);
void launch_correct(const DevParams& p, PressurePtr w, const double* APU, const double* APV,
                    double* u, double* v, double* pf, cudaStream_t st);
// dst[i] = src[i] over n doubles.
void launch_copy(const double* src, double* dst, std::size_t n, cudaStream_t st);

// ---- multigrid (mg.cu) ----
// Every multigrid launcher is instantiated for double (the reference's bits) and float (the
// mixed-precision V-cycle).
template <class T> void launch_mg_build(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st);
template <class T> void launch_mg_smooth_colour(const LevelViewT<T>& L, int colour, cudaStream_t st);
template <class T> void launch_mg_residual(const LevelViewT<T>& L, cudaStream_t st);
template <class T> void launch_mg_restrict(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st);
template <class T>
void launch_mg_prolong(const LevelViewT<T>& C, const LevelViewT<T>& F, double omega, cudaStream_t st);
// (b - A x)^2 and b^2 per cell of the level into a compact nx x ny plane (FP64), for the ordered
// norms of the tolerance-driven V-cycle loop (mg_mode = tolerance).
template <class T> void launch_mg_residual_sq(const LevelViewT<T>& L, double* cells, cudaStream_t st);
template <class T> void launch_mg_b_sq(const LevelViewT<T>& L, double* cells, cudaStream_t st);
// x[I, J] -= *sum / (nx * ny) over the level interior (the mean removal after an ordered sum).
void launch_mg_sub_mean(const LevelView& L, double* x, const double* sum, cudaStream_t st);
// Coarsest-level solve in one CTA (coarse_solve, multigrid.cpp:120-140) with relative tolerance
// tol (the reference's 1e-10 in FP64); *sweeps_out gets the sweep count.
template <class T>
void launch_mg_coarse(const LevelViewT<T>& L, double* rowbuf, double tol, int* sweeps_out,
                      cudaStream_t st);
// The whole hierarchy, by value, for the single-CTA tail kernel.
template <class T> struct MgLevelsT {
    LevelViewT<T> L[24];
    int n;
};
using MgLevels = MgLevelsT<double>;
// Levels [first, n) of one V-cycle in one CTA: down-leg, coarse solve, up-leg (mg_vcycle order).
template <class T>
void launch_mg_tail(const MgLevelsT<T>& lv, int first, int pre, int post, double omega, double tol,
                    double* rowbuf, int* sweeps_out, cudaStream_t st);
// The float V-cycle's levels from `first` on one thread-block cluster of 16 CTAs (mg.cu,
// k_mg_tail_cluster): the levels of more than 1024 cells split by rows, the rest and the coarsest
// solve on one CTA. mg_cluster_tail_first: the first level from which it applies (at most 65536
// cells), or `fallback` where the device or the grid does not allow it. launch_mg_tail_cluster
// returns false (and launches nothing) where it does not apply from `first`.
int mg_cluster_tail_first(const MgLevelsT<float>& lv, int fallback);
bool launch_mg_tail_cluster(const MgLevelsT<float>& lv, int first, int pre, int post, double omega, double tol,
                            int* sweeps_out, cudaStream_t st);

// ---- streaming multigrid level kernels (mg_fast.cu), double and float ----
bool mg_fast_supported(int pre, int post);
// pre red-black sweeps on F (x from F.x, or zero), residual, restriction into C.b (C.x = 0); the
// smoothed iterate is written to xout (F.x is left unchanged when pre > 0). build: also C's links
// and AP from F's (mg_build's sums, the same bits as launch_mg_build).
template <class T>
void launch_mg_down(const LevelViewT<T>& F, const LevelViewT<T>& C, T* xout, int pre, bool x_zero,
                    int sms, int min_seg, cudaStream_t st, bool build = false);
// xout = xin + omega * P C.x, then post red-black sweeps (F's coefficients and b).
template <class T>
void launch_mg_up(const LevelViewT<T>& C, const LevelViewT<T>& F, const T* xin, T* xout,
                  double omega, int post, int sms, int min_seg, cudaStream_t st);

// ---- conjugate gradient (cg.cu) ----
struct CgScalars {
    double rz, nb, mz, alpha, beta, rel, mb;
    int k, done, maxit;
    double tol, n;
};
struct CgPtr {
    double *r, *z, *d, *q;
};
void launch_cg_init(const DevParams& p, PressurePtr w, CgPtr cg, CgScalars* sc, double* cells,
                    std::size_t plane, cudaStream_t st);
void launch_cg_scalars(int stage, CgScalars* sc, const double* sums, cudaStream_t st);
void launch_cg_dinit(const DevParams& p, CgPtr cg, const CgScalars* sc, cudaStream_t st);
void launch_cg_dq(const DevParams& p, PressurePtr w, CgPtr cg, const CgScalars* sc, double* cells,
                  cudaStream_t st);
void launch_cg_update(const DevParams& p, PressurePtr w, CgPtr cg, const CgScalars* sc,
                      double* cells, std::size_t plane, cudaStream_t st);
void launch_cg_dir(const DevParams& p, CgPtr cg, const CgScalars* sc, cudaStream_t st);

// ---- mixed precision (mixed.cu) ----
void init_mixed_kernels();
// Resident CTAs per SM of the FP32 correction sweep (its register and shared-memory footprint).
int corr_blocks_per_sm(int ncol);
// Threads per CTA of the FP32 correction sweep (its strips are this wide, halos included).
int corr_threads();
// Diagnostic: one warp's bounded wait on an mbarrier that never completes (the correction sweep's
// wait helper); it gives up after `polls` polls and sets *err.
void launch_wait_selftest(int polls, unsigned* err, cudaStream_t st);
// Per-cell FP32 momentum records of the mixed path in three arrays: the near links {AE AW AN AS},
// the far links {AEE AWW ANN ASS}, and {1/AP, R}; 40 bytes per cell. They are stored by sweep step:
// the record of cell (i, j) of colour c (c = (i + 3j) mod 5 for five colours, (i + j) mod 2 for
// two) sits at (i + 2c) * pitch + j, so the cells the streaming sweep updates at one step, one per
// column, are contiguous. The arrays have kRecExtraRows rows more than the fields, and are
// allocated with kRecFrontCols records before element 0 and kRecBackCols after the last row: the
// correction sweep copies whole step-row segments of its CTA's NT columns (NT <= 512), which reach up
// to 2 x the colour count before column 0 and up to NT past the last column.
constexpr int kRecExtraRows = 8;
constexpr int kRecFrontCols = 16, kRecBackCols = 512;
struct MomRec32 {
    float4* near_links;
    float4* far_links;
    float2* diag;
};
// FP64 prep over the update range: AP (FP64), the cell's FP32 record, and one partial sum of |R|
// per block into part; returns the number of partial sums (for launch_sum_partials).
int launch_mom_prep_mixed(const DevParams& p, bool v_component, const double* x, const double* oth,
                          const double* pf, double* AP, double* part, MomRec32 rec, cudaStream_t st);
// One FP32 multicolour correction sweep e_in -> e_out (e_zero: e_in is zero and not read).
// xfinal != null: the last sweep of a component adds e to the FP64 field x over the update range
// (x += e in FP64) instead of writing eout. *err (a device word) gets a nonzero bit if one of the
// kernel's bounded waits for its record copies gave up.
void launch_corr_sweep(const DevParams& p, bool v_component, const float* ein, float* eout,
                       MomRec32 rec, bool e_zero, int seg_rows, unsigned* err, cudaStream_t st,
                       double* xfinal = nullptr);
// All nsweeps correction sweeps of a component on one 16-CTA thread-block cluster, e from zero and
// x += e at the end, where the component's records and e fit the cluster's shared memory (small
// grids); returns false, and launches nothing, where they do not (or the device runs no such
// cluster, or SGPU_CORR_CLUSTER=0).
bool launch_corr_cluster(const DevParams& p, bool v_component, MomRec32 rec, int nsweeps, double* x,
                         cudaStream_t st);
// assemble_p with the FP32 level-0 operator; per block one partial sum of |b| into part[k] and one
// of b into part[n + k] (n = the returned number of blocks).
int launch_assemble_p_mixed(const DevParams& p, const double* APU, const double* APV, const double* u,
                            const double* v, double* bfield, const LevelView32& L0, double* part,
                            cudaStream_t st);
// Doubles of partial-sum scratch the two launchers above need at most.
int mixed_partials(const DevParams& p);
// FP64 defect correction of the mixed-precision p' solve (mg_mode = tolerance); see mixed.cu.
// Each returns the number of blocks whose partial sums it wrote (k_sum_partials adds them):
// launch_dc_rhs0 one plane (sum of (b - mean b)^2), launch_dc_update two (sum of r^2, sum of p').
int launch_dc_rhs0(const DevParams& p, const double* bfield, const double* sum_b, const LevelView32& L0,
                   double* part, cudaStream_t st);
int launch_dc_update(const DevParams& p, const double* APU, const double* APV, const double* bfield,
                     const double* sum_b, const LevelView32& L0, const double* pold, double* pnew, bool first,
                     double* part, cudaStream_t st);
void launch_correct_dc(const DevParams& p, const double* pc64, const double* sum_pc, const double* APU,
                       const double* APV, double* u, double* v, double* pf, cudaStream_t st);
void launch_pc_from64(const DevParams& p, const double* src, const double* sum_pc, double* dst, cudaStream_t st);
void launch_b_to_f32(const DevParams& p, const double* bfield, const double* sum_b,
                     const LevelView32& L0, cudaStream_t st);
// pc64 = FP32 p' minus its FP64 mean over the p' cells (the field correct_mixed applied).
void launch_pc_from32(const DevParams& p, const LevelView32& L0, const double* sum_pc, double* pc64,
                      cudaStream_t st);
// correct with the FP32 level-0 p' minus its FP64 mean (the mixed iteration's last phase).
void launch_correct_mixed(const DevParams& p, const LevelView32& L0, const double* sum_pc,
                          const double* APU, const double* APV, double* u, double* v, double* pf,
                          cudaStream_t st);

// ---- fused fast path (fused.cu) ----
// Rows per CTA segment of the streaming sweeps: one wave of blocks_per_sm resident CTAs per SM, at
// least min_seg rows (min_seg <= 0: 8 x the colour count).
int stream_seg_rows(const DevParams& p, int sms, int blocks_per_sm = 2, int min_seg = 0, int nt = 256);
// Momentum prep: |R| into cells, AP over the update range, frozen copy xF of x.
void launch_mom_prep(const DevParams& p, bool v_component, const double* x, const double* oth,
                     const double* pf, double* xF, double* AP, double* cells, cudaStream_t st);
// One whole multicolour sweep xin -> xout (every cell of xout written).
void launch_mom_sweep(const DevParams& p, bool v_component, const double* xin, double* xout,
                      const double* xF, const double* oth, const double* pf, int seg_rows,
                      cudaStream_t st);
void launch_assemble_p_fused(const DevParams& p, const double* APU, const double* APV,
                             const double* u, const double* v, PressurePtr w, double* cabs,
                             double* cb, cudaStream_t st);

} // namespace sgpu
