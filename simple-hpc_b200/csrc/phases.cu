// phases.cu — the reference-shaped FP64 kernels behind the per-phase C ABI (sgpu_assemble_u, ...).
//
// One thread per cell, coefficients materialised in 9 + 9 arrays, one launch per colour: the same
// work split as the reference GPU backend (src/hip/solver_hip.hip:168-304), so every array the
// reference's State holds can be downloaded and compared after every phase. The fused fast path in
// fused.cu produces the same bits without materialising the coefficients.
#include "kernels.hpp"
#include "stencil.cuh"

namespace sgpu {

namespace {

constexpr int BX = 32, BY = 8;

__device__ __forceinline__ bool cell_of(const Range& r, int& i, int& j) {
    j = r.j0 + static_cast<int>(blockIdx.x * BX + threadIdx.x);
    i = r.i0 + static_cast<int>(blockIdx.y * BY + threadIdx.y);
    return i <= r.i1 && j <= r.j1;
}

dim3 grid_of(const Range& r) { return dim3((r.cols() + BX - 1) / BX, (r.rows() + BY - 1) / BY); }

__device__ __forceinline__ std::size_t ix(const DevParams& p, int i, int j) {
    return static_cast<std::size_t>(i) * p.pitch + j;
}

__device__ __forceinline__ void store_coef(const Coef9Ptr& c, std::size_t q, const Coef9& k) {
    c.a[0][q] = k.AE;
    c.a[1][q] = k.AW;
    c.a[2][q] = k.AN;
    c.a[3][q] = k.AS;
    c.a[4][q] = k.AEE;
    c.a[5][q] = k.AWW;
    c.a[6][q] = k.ANN;
    c.a[7][q] = k.ASS;
    c.a[8][q] = k.AP;
}

// nb_sum (momentum_u.cpp:36-41): near four, then far four, E W N S order.
__device__ __forceinline__ double nb_sum(const Coef9Ptr& c, const double* f, std::size_t q,
                                         std::size_t ld) {
    return (c.a[0][q] * f[q + 1] + c.a[1][q] * f[q - 1] + c.a[2][q] * f[q - ld] +
            c.a[3][q] * f[q + ld]) +
           (c.a[4][q] * f[q + 2] + c.a[5][q] * f[q - 2] + c.a[6][q] * f[q - 2 * ld] +
            c.a[7][q] * f[q + 2 * ld]);
}

// near_sum (momentum_u.cpp:84-87): the 2-colour case reads no far cell.
__device__ __forceinline__ double near_sum(const Coef9Ptr& c, const double* f, std::size_t q,
                                           std::size_t ld) {
    return c.a[0][q] * f[q + 1] + c.a[1][q] * f[q - 1] + c.a[2][q] * f[q - ld] +
           c.a[3][q] * f[q + ld];
}

// assemble_u (momentum_u.cpp:8-22): face velocities, then Coeffs::set(conv + diff).
__global__ void k_assemble_u(DevParams p, const double* __restrict__ u, const double* __restrict__ v,
                             Coef9Ptr cu, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double ue = (u[q] + u[q + 1]) / 2;
    const double uw = (u[q] + u[q - 1]) / 2;
    const double vn = (v[q] + v[q + 1]) / 2;
    const double vs = (v[q + ld] + v[q + ld + 1]) / 2;
    store_coef(cu, q, momentum_coef(p, ue, uw, vn, vs, i, j));
}

// assemble_v (momentum_v.cpp:9-22).
__global__ void k_assemble_v(DevParams p, const double* __restrict__ u, const double* __restrict__ v,
                             Coef9Ptr cv, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double ue = (u[q - ld] + u[q]) / 2;
    const double uw = (u[q - 1] + u[q - ld - 1]) / 2;
    const double vn = (v[q] + v[q - ld]) / 2;
    const double vs = (v[q] + v[q + ld]) / 2;
    store_coef(cv, q, momentum_coef(p, ue, uw, vn, vs, i, j));
}

// apply_bc_u (momentum_u.cpp:24-34): lid ghost row and south ghost row.
__global__ void k_bc_u(DevParams p, double* u) {
    const int H = p.H, j = H + 1 + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (j > p.NY + H) return;
    u[ix(p, H - 1, j)] = 2 - u[ix(p, H, j)];
    u[ix(p, p.NX + H, j)] = -u[ix(p, p.NX + H - 1, j)];
}

// apply_bc_v (momentum_v.cpp:24-34): west and east ghost columns.
__global__ void k_bc_v(DevParams p, double* v) {
    const int H = p.H, i = H + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i > p.NX + H - 1) return;
    v[ix(p, i, H)] = -v[ix(p, i, H + 1)];
    v[ix(p, i, p.NY + H + 1)] = -v[ix(p, i, p.NY + H)];
}

// residual_u (momentum_u.cpp:43-59): |R| per cell; the ordered sum runs after.
__global__ void k_residual_u(DevParams p, Coef9Ptr cu, const double* __restrict__ u,
                             const double* __restrict__ pf, double* __restrict__ cells, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double R = nb_sum(cu, u, q, ld) + (pf[q] - pf[q + 1]) * p.dy - cu.a[8][q] * u[q];
    cells[static_cast<std::size_t>(i - r.i0) * r.cols() + (j - r.j0)] = fabs(R);
}

// residual_v (momentum_v.cpp:36-55).
__global__ void k_residual_v(DevParams p, Coef9Ptr cv, const double* __restrict__ v,
                             const double* __restrict__ pf, double* __restrict__ cells, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double R = nb_sum(cv, v, q, ld) + (pf[q] - pf[q - ld]) * p.dx - cv.a[8][q] * v[q];
    cells[static_cast<std::size_t>(i - r.i0) * r.cols() + (j - r.j0)] = fabs(R);
}

// One colour of sweep_u_multicolour_batch (momentum_u.cpp:123-143), in place.
__global__ void k_sweep_u(DevParams p, Coef9Ptr cu, double* u, const double* __restrict__ pf,
                          Range r, int colour) {
    int i, j;
    if (!cell_of(r, i, j) || momentum_colour(p.ncol, i, j) != colour) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double a = p.au;
    const double nb = p.ncol == 2 ? near_sum(cu, u, q, ld) : nb_sum(cu, u, q, ld);
    u[q] = a * (nb + (pf[q] - pf[q + 1]) * p.dy) / cu.a[8][q] + (1 - a) * u[q];
}

// One colour of sweep_v_multicolour_batch (momentum_v.cpp:121-145).
__global__ void k_sweep_v(DevParams p, Coef9Ptr cv, double* v, const double* __restrict__ pf,
                          Range r, int colour) {
    int i, j;
    if (!cell_of(r, i, j) || momentum_colour(p.ncol, i, j) != colour) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double av = p.av;
    const double nb = p.ncol == 2 ? near_sum(cv, v, q, ld) : nb_sum(cv, v, q, ld);
    v[q] = av * (nb + (pf[q] - pf[q - ld]) * p.dx) / cv.a[8][q] + (1 - av) * v[q];
}

// One pass of sweep_u_jacobi_batch (momentum_u.cpp:89-116): src -> dst.
__global__ void k_jacobi_u(DevParams p, Coef9Ptr cu, const double* __restrict__ src,
                           double* __restrict__ dst, const double* __restrict__ pf, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double a = p.au;
    dst[q] = a * (nb_sum(cu, src, q, ld) + (pf[q] - pf[q + 1]) * p.dy) / cu.a[8][q] +
             (1 - a) * src[q];
}

// One pass of sweep_v_jacobi_batch (momentum_v.cpp:85-114).
__global__ void k_jacobi_v(DevParams p, Coef9Ptr cv, const double* __restrict__ src,
                           double* __restrict__ dst, const double* __restrict__ pf, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double av = p.av;
    dst[q] = av * (nb_sum(cv, src, q, ld) + (pf[q] - pf[q - ld]) * p.dx) / cv.a[8][q] +
             (1 - av) * src[q];
}

// assemble_p links (pressure.cpp:19-26). The wall links are zeroed by k_p_zero afterwards.
__global__ void k_p_links(DevParams p, const double* __restrict__ APU, const double* __restrict__ APV,
                          PressurePtr w, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double dx = p.dx, dy = p.dy;
    w.AEP[q] = dy * dy / APU[q];
    w.AWP[q] = dy * dy / APU[q - 1];
    w.ANP[q] = dx * dx / APV[q];
    w.ASP[q] = dx * dx / APV[q + ld];
}

// assemble_p wall links (pressure.cpp:27-38): whole rows / columns of the stored grid.
__global__ void k_p_zero(DevParams p, PressurePtr w) {
    const int k = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x), H = p.H;
    if (k < p.nrows) {
        w.AWP[ix(p, k, H + 1)] = 0.0;
        w.AEP[ix(p, k, p.NY + H)] = 0.0;
    }
    if (k < p.ncols) {
        w.ASP[ix(p, p.NX + H - 1, k)] = 0.0;
        w.ANP[ix(p, H, k)] = 0.0;
    }
}

// assemble_p APP and b (pressure.cpp:39-53); |b| (and b) per cell for the ordered sums.
__global__ void k_p_rhs(DevParams p, const double* __restrict__ u, const double* __restrict__ v,
                        PressurePtr w, double* __restrict__ cells_abs, double* __restrict__ cells_b,
                        Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double dx = p.dx, dy = p.dy;
    w.APP[q] = w.AEP[q] + w.AWP[q] + w.ANP[q] + w.ASP[q];
    const double b = -dx * (-v[q + ld] + v[q]) - dy * (-u[q - 1] + u[q]);
    w.b[q] = b;
    const std::size_t c = static_cast<std::size_t>(i - r.i0) * r.cols() + (j - r.j0);
    cells_abs[c] = fabs(b);
    if (cells_b) cells_b[c] = b;
}

// Two-statement p' update (pressure.cpp:70-75): E, W, S, N.
__global__ void k_pc_redblack(DevParams p, PressurePtr w, Range r, int colour) {
    int i, j;
    if (!cell_of(r, i, j) || ((i + j) & 1) != colour) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    double t = w.b[q] / w.APP[q];
    t += (w.AEP[q] * w.pc[q + 1] + w.AWP[q] * w.pc[q - 1] + w.ASP[q] * w.pc[q + ld] +
          w.ANP[q] * w.pc[q - ld]) /
         w.APP[q];
    w.pc[q] = t;
}

// One damped Jacobi pass of solve_pc_jacobi (pressure.cpp:77-112), weight 0.8.
__global__ void k_pc_jacobi(DevParams p, PressurePtr w, const double* __restrict__ src,
                            double* __restrict__ dst, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    double t = w.b[q] / w.APP[q];
    t += (w.AEP[q] * src[q + 1] + w.AWP[q] * src[q - 1] + w.ASP[q] * src[q + ld] +
          w.ANP[q] * src[q - ld]) /
         w.APP[q];
    const double wgt = 0.8;
    dst[q] = wgt * t + (1 - wgt) * src[q];
}

// correct (pressure.cpp:136-157): the three loops write different arrays and read only pc. Each
// thread corrects the two cells (j, j + 1) of a column pair (j even; the pitch is even), reading and
// writing every array as 16-byte pairs; an element of a pair outside the range keeps its value (the
// thread writes back what it read). The per-cell expressions are the reference's.
__device__ __forceinline__ double2 ld2(const double* q) { return *reinterpret_cast<const double2*>(q); }
__device__ __forceinline__ void st2(double* q, double2 v) { *reinterpret_cast<double2*>(q) = v; }
__global__ void k_correct(DevParams p, PressurePtr w, const double* __restrict__ APU,
                          const double* __restrict__ APV, double* __restrict__ u, double* __restrict__ v,
                          double* __restrict__ pf, Range r) {
    const int j = (r.j0 & ~1) + 2 * static_cast<int>(blockIdx.x * BX + threadIdx.x);
    const int i = r.i0 + static_cast<int>(blockIdx.y * BY + threadIdx.y);
    if (i > r.i1 || j > r.j1) return;
    const int H = p.H;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const bool vrow = i >= H + 1;
    const double2 pc = ld2(w.pc + q), apu = ld2(APU + q), pp = ld2(pf + q);
    const double pce = w.pc[q + 2];
    double2 uu = ld2(u + q), vv = make_double2(0.0, 0.0), pcn = vv, apv = make_double2(1.0, 1.0);
    if (vrow) {
        vv = ld2(v + q);
        pcn = ld2(w.pc + q - ld);
        apv = ld2(APV + q);
    }
    const double pcq[2] = {pc.x, pc.y}, pceq[2] = {pc.y, pce}, pcnq[2] = {pcn.x, pcn.y};
    const double apuq[2] = {apu.x, apu.y}, apvq[2] = {apv.x, apv.y};
    double uq[2] = {uu.x, uu.y}, vq[2] = {vv.x, vv.y}, pq[2] = {pp.x, pp.y};
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int jj = j + e;
        if (jj < r.j0 || jj > r.j1) continue;
        if (jj <= p.NY + H - 1) uq[e] += p.dy * (pcq[e] - pceq[e]) / apuq[e];
        if (vrow) vq[e] += p.dx * (pcq[e] - pcnq[e]) / apvq[e];
        pq[e] += p.ap * pcq[e];
    }
    st2(u + q, make_double2(uq[0], uq[1]));
    if (vrow) st2(v + q, make_double2(vq[0], vq[1]));
    st2(pf + q, make_double2(pq[0], pq[1]));
}

// APP alone (pressure.cpp:42): the links' sum, without touching b.
__global__ void k_p_app(DevParams p, PressurePtr w, Range r) {
    int i, j;
    if (!cell_of(r, i, j)) return;
    const std::size_t q = ix(p, i, j);
    w.APP[q] = w.AEP[q] + w.AWP[q] + w.ANP[q] + w.ASP[q];
}

__global__ void k_copy(const double* __restrict__ src, double* __restrict__ dst, std::size_t n) {
    for (std::size_t k = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<std::size_t>(gridDim.x) * blockDim.x)
        dst[k] = src[k];
}

// Kernel ranges (the loop bounds of the CPU kernels).
Range r_assemble_u(const DevParams& p) { return {p.H, p.NX + p.H - 1, p.H, p.NY + p.H}; }
Range r_assemble_v(const DevParams& p) { return {p.H, p.NX + p.H + 1, p.H, p.NY + p.H + 1}; }
Range r_u(const DevParams& p) { return {p.H, p.NX + p.H - 1, p.H + 1, p.NY + p.H - 1}; }
Range r_v(const DevParams& p) { return {p.H + 1, p.NX + p.H - 1, p.H + 1, p.NY + p.H}; }
Range r_p(const DevParams& p) { return {p.H, p.NX + p.H - 1, p.H + 1, p.NY + p.H}; }

} // namespace

void launch_assemble_u(const DevParams& p, const double* u, const double* v, Coef9Ptr cu,
                       cudaStream_t st) {
    const Range r = r_assemble_u(p);
    k_assemble_u<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, u, v, cu, r);
    SGPU_LAUNCH();
}
void launch_assemble_v(const DevParams& p, const double* u, const double* v, Coef9Ptr cv,
                       cudaStream_t st) {
    const Range r = r_assemble_v(p);
    k_assemble_v<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, u, v, cv, r);
    SGPU_LAUNCH();
}
void launch_bc_u(const DevParams& p, double* u, cudaStream_t st) {
    k_bc_u<<<(p.NY + 255) / 256, 256, 0, st>>>(p, u);
    SGPU_LAUNCH();
}
void launch_bc_v(const DevParams& p, double* v, cudaStream_t st) {
    k_bc_v<<<(p.NX + 255) / 256, 256, 0, st>>>(p, v);
    SGPU_LAUNCH();
}
void launch_residual_u_cells(const DevParams& p, Coef9Ptr cu, const double* u, const double* pf,
                             double* cells, cudaStream_t st) {
    const Range r = r_u(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_residual_u<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cu, u, pf, cells, r);
    SGPU_LAUNCH();
}
void launch_residual_v_cells(const DevParams& p, Coef9Ptr cv, const double* v, const double* pf,
                             double* cells, cudaStream_t st) {
    const Range r = r_v(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_residual_v<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cv, v, pf, cells, r);
    SGPU_LAUNCH();
}
void launch_sweep_u_colour(const DevParams& p, Coef9Ptr cu, double* u, const double* pf, int colour,
                           cudaStream_t st) {
    const Range r = r_u(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_sweep_u<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cu, u, pf, r, colour);
    SGPU_LAUNCH();
}
void launch_sweep_v_colour(const DevParams& p, Coef9Ptr cv, double* v, const double* pf, int colour,
                           cudaStream_t st) {
    const Range r = r_v(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_sweep_v<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cv, v, pf, r, colour);
    SGPU_LAUNCH();
}
void launch_sweep_u_jacobi(const DevParams& p, Coef9Ptr cu, const double* src, double* dst,
                           const double* pf, cudaStream_t st) {
    const Range r = r_u(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_jacobi_u<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cu, src, dst, pf, r);
    SGPU_LAUNCH();
}
void launch_sweep_v_jacobi(const DevParams& p, Coef9Ptr cv, const double* src, double* dst,
                           const double* pf, cudaStream_t st) {
    const Range r = r_v(p);
    if (r.rows() <= 0 || r.cols() <= 0) return;
    k_jacobi_v<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, cv, src, dst, pf, r);
    SGPU_LAUNCH();
}
void launch_assemble_p(const DevParams& p, const double* APU, const double* APV, const double* u,
                       const double* v, PressurePtr w, double* cells_absb, double* cells_b,
                       cudaStream_t st) {
    const Range r = r_p(p);
    k_p_links<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, APU, APV, w, r);
    SGPU_LAUNCH();
    const int n = p.nrows > p.ncols ? p.nrows : p.ncols;
    k_p_zero<<<(n + 255) / 256, 256, 0, st>>>(p, w);
    SGPU_LAUNCH();
    k_p_rhs<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, u, v, w, cells_absb, cells_b, r);
    SGPU_LAUNCH();
}
void launch_p_links_app(const DevParams& p, const double* APU, const double* APV, PressurePtr w,
                        cudaStream_t st) {
    const Range r = r_p(p);
    k_p_links<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, APU, APV, w, r);
    SGPU_LAUNCH();
    const int n = p.nrows > p.ncols ? p.nrows : p.ncols;
    k_p_zero<<<(n + 255) / 256, 256, 0, st>>>(p, w);
    SGPU_LAUNCH();
    k_p_app<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, w, r);
    SGPU_LAUNCH();
}
void launch_pc_redblack(const DevParams& p, PressurePtr w, int colour, cudaStream_t st) {
    const Range r = r_p(p);
    k_pc_redblack<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, w, r, colour);
    SGPU_LAUNCH();
}
void launch_pc_jacobi(const DevParams& p, PressurePtr w, const double* src, double* dst,
                      cudaStream_t st) {
    const Range r = r_p(p);
    k_pc_jacobi<<<grid_of(r), dim3(BX, BY), 0, st>>>(p, w, src, dst, r);
    SGPU_LAUNCH();
}
void launch_correct(const DevParams& p, PressurePtr w, const double* APU, const double* APV,
                    double* u, double* v, double* pf, cudaStream_t st) {
    const Range r = r_p(p);
    const int pairs = (r.j1 - (r.j0 & ~1)) / 2 + 1;
    k_correct<<<dim3((pairs + BX - 1) / BX, (r.rows() + BY - 1) / BY), dim3(BX, BY), 0, st>>>(p, w, APU, APV, u,
                                                                                              v, pf, r);
    SGPU_LAUNCH();
}
void launch_copy(const double* src, double* dst, std::size_t n, cudaStream_t st) {
    if (n == 0) return;
    const std::size_t blocks = (n + 255) / 256;
    k_copy<<<static_cast<unsigned>(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(src, dst, n);
    SGPU_LAUNCH();
}

} // namespace sgpu
