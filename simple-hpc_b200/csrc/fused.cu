// fused.cu — the fast FP64 outer iteration: same bits as the reference, a fraction of the traffic.
//
// Momentum phase (assemble + bc + residual + maxit_inner multicolour sweeps, momentum_u.cpp /
// momentum_v.cpp) without the 9 coefficient arrays:
//  * k_mom_prep computes each cell's coefficients from the velocity at assembly time, writes the
//    residual |R| (ordered sum afterwards), the AP coefficient (the only one assemble_p and correct
//    read) and a frozen copy xF of the velocity, from which every later sweep recomputes the
//    coefficients (convective_coefficients + diffusive_coefficients, coefficients.cpp:15-63).
//  * k_mom_stream runs one whole multicolour sweep (all colours) in one pass over memory. A CTA
//    owns a strip of columns plus a halo and walks it top to bottom; cell (r, j) of colour c is
//    updated at step t = r + 2c. Every stencil neighbour of a cell is updated at least two steps
//    before it (if its colour comes first) or two steps after it (if later), so the update order
//    of each cell relative to its neighbours is exactly the reference's colour order and one
//    barrier per step suffices. Rows stream through a shared-memory ring filled by cp.async; halo
//    cells are updated redundantly and only the owned block is written, to a second buffer.
// Pressure assembly (assemble_p, pressure.cpp:14-54) is one kernel with the wall zeros folded in.
#include "kernels.hpp"
#include "stencil.cuh"

#include <climits>

namespace sgpu {

namespace {

__device__ __forceinline__ std::size_t ix(const DevParams& p, int i, int j) {
    return static_cast<std::size_t>(i) * p.pitch + j;
}

// Coefficients of a u cell (assemble_u, momentum_u.cpp:12-19) from the frozen u and from v.
__device__ __forceinline__ Coef9 coef_u(const DevParams& p, const double* __restrict__ uF,
                                        const double* __restrict__ v, int i, int j) {
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double ue = (uF[q] + uF[q + 1]) / 2;
    const double uw = (uF[q] + uF[q - 1]) / 2;
    const double vn = (v[q] + v[q + 1]) / 2;
    const double vs = (v[q + ld] + v[q + ld + 1]) / 2;
    return momentum_coef(p, ue, uw, vn, vs, i, j);
}

// Coefficients of a v cell (assemble_v, momentum_v.cpp:13-19) from u and the frozen v.
__device__ __forceinline__ Coef9 coef_v(const DevParams& p, const double* __restrict__ u,
                                        const double* __restrict__ vF, int i, int j) {
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double ue = (u[q - ld] + u[q]) / 2;
    const double uw = (u[q - 1] + u[q - ld - 1]) / 2;
    const double vn = (vF[q] + vF[q - ld]) / 2;
    const double vs = (vF[q] + vF[q + ld]) / 2;
    return momentum_coef(p, ue, uw, vn, vs, i, j);
}

// Residual / copy pass. Grid over the copy range cr (the update range ur widened by the cells the
// coefficient recomputation reads); cells of ur also get |R| and AP.
template <bool V>
__global__ void k_mom_prep(DevParams p, const double* __restrict__ x, const double* __restrict__ oth,
                           const double* __restrict__ pf, double* __restrict__ xF,
                           double* __restrict__ AP, double* __restrict__ cells, Range ur, Range cr) {
    const int j = cr.j0 + static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int i = cr.i0 + static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (i > cr.i1 || j > cr.j1) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    xF[q] = x[q];
    if (i < ur.i0 || i > ur.i1 || j < ur.j0 || j > ur.j1) return;
    const Coef9 c = V ? coef_v(p, oth, x, i, j) : coef_u(p, x, oth, i, j);
    // nb_sum (momentum_u.cpp:36-41); residual_u / residual_v (momentum_u.cpp:51, momentum_v.cpp:43-47).
    const double nb = (c.AE * x[q + 1] + c.AW * x[q - 1] + c.AN * x[q - ld] + c.AS * x[q + ld]) +
                      (c.AEE * x[q + 2] + c.AWW * x[q - 2] + c.ANN * x[q - 2 * ld] +
                       c.ASS * x[q + 2 * ld]);
    const double pt = V ? (pf[q] - pf[q - ld]) * p.dx : (pf[q] - pf[q + 1]) * p.dy;
    const double R = nb + pt - c.AP * x[q];
    cells[static_cast<std::size_t>(i - ur.i0) * ur.cols() + (j - ur.j0)] = fabs(R);
    AP[q] = c.AP;
}

constexpr int kRing = 32; // rows held in the shared-memory ring (power of two)
constexpr int kPrefetch = 8;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One multicolour sweep of u (V = false) or v (V = true) from xin to xout. NT threads per CTA, one
// column each; the CTA owns W = NT - 4 * NCOL columns starting at blockIdx.x * W and rows
// [blockIdx.y * seg_rows, + seg_rows).
template <int NCOL, bool V, int NT>
__global__ void __launch_bounds__(NT, 2)
    k_mom_stream(DevParams p, const double* __restrict__ xin, double* __restrict__ xout,
                 const double* __restrict__ xF, const double* __restrict__ oth,
                 const double* __restrict__ pf, int seg_rows) {
    static_assert(kPrefetch <= kRing - 2 * NCOL - 4, "ring too small for the prefetch distance");
    extern __shared__ double ring_mem[];
    double(*ring)[NT] = reinterpret_cast<double(*)[NT]>(ring_mem); // kRing rows of NT columns
    constexpr int HC = 2 * NCOL; // halo: a sweep's dependency reach (2 cells per colour)
    constexpr int W = NT - 2 * HC;
    const int tid = threadIdx.x;
    const int j0 = blockIdx.x * W;
    const int C0 = j0 - HC, C1 = j0 + W + HC; // loaded columns [C0, C1)
    const int col = C0 + tid;
    const int R0 = blockIdx.y * seg_rows;
    const int R1 = min(R0 + seg_rows, p.nrows);
    const int L0 = max(R0 - HC, 0), L1 = min(R1 + HC, p.nrows); // loaded rows [L0, L1)
    const bool col_in = col >= 0 && col < p.ncols;
    const bool col_out = col_in && col >= j0 && col < j0 + W;
    const int H = p.H;
    const int iu0 = V ? H + 1 : H, iu1 = p.NX + H - 1;
    const int ju0 = H + 1, ju1 = V ? p.NY + H : p.NY + H - 1;
    const bool cut_top = L0 > 0, cut_bot = L1 < p.nrows, cut_left = C0 > 0, cut_right = C1 < p.ncols;
    const std::size_t ld = p.pitch;
    const double relax = V ? p.av : p.au;

    int next = L0;
    auto issue = [&]() {
        if (next < L1 && col_in) cp_async8(&ring[next & (kRing - 1)][tid], xin + ix(p, next, col));
        cp_async_commit();
        ++next;
    };
    for (int k = 0; k < kPrefetch + 3; ++k) issue(); // rows L0 .. L0 + 2 + kPrefetch

    const int t_last = R1 + 2 * NCOL - 2; // the step that writes back row R1 - 1
    for (int t = L0; t <= t_last; ++t) {
        cp_async_wait<kPrefetch>(); // row t + 2 has landed (this thread's copies)
        __syncthreads();            // ... everyone's, and step t - 1's updates are visible
        issue();                    // row t + 3 + kPrefetch into the slot of a row no longer read

        // The one cell of this column updated at step t: colour c at row t - 2c.
        const int c = NCOL == 5 ? (2 * t + col + 1000) % 5 : (t + col + 1000) & 1;
        const int r = t - 2 * c;
        bool ok = r >= iu0 && r <= iu1 && col >= ju0 && col <= ju1;
        ok = ok && (!cut_top || r >= L0 + 2 + 2 * c) && (!cut_bot || r <= L1 - 3 - 2 * c);
        ok = ok && (!cut_left || col >= C0 + 2 + 2 * c) && (!cut_right || col <= C1 - 3 - 2 * c);
        if (ok) {
            const Coef9 k = V ? coef_v(p, oth, xF, r, col) : coef_u(p, xF, oth, r, col);
            const double* rc = ring[r & (kRing - 1)];
            const double xe = rc[tid + 1], xw = rc[tid - 1];
            const double xn = ring[(r - 1) & (kRing - 1)][tid], xs = ring[(r + 1) & (kRing - 1)][tid];
            // near_sum for two colours (momentum_u.cpp:84-87), nb_sum for five (:36-41).
            double nb = k.AE * xe + k.AW * xw + k.AN * xn + k.AS * xs;
            if (NCOL == 5) {
                const double xee = rc[tid + 2], xww = rc[tid - 2];
                const double xnn = ring[(r - 2) & (kRing - 1)][tid];
                const double xss = ring[(r + 2) & (kRing - 1)][tid];
                nb = nb + (k.AEE * xee + k.AWW * xww + k.ANN * xnn + k.ASS * xss);
            }
            const std::size_t q = ix(p, r, col);
            const double pt = V ? (pf[q] - pf[q - ld]) * p.dx : (pf[q] - pf[q + 1]) * p.dy;
            const double xo = rc[tid];
            ring[r & (kRing - 1)][tid] = relax * (nb + pt) / k.AP + (1 - relax) * xo;
        }
        // Row t - (2 NCOL - 1) had its last update at step t - 1: write the owned part back.
        const int rw = t - (2 * NCOL - 1);
        if (rw >= R0 && rw < R1 && col_out) xout[ix(p, rw, col)] = ring[rw & (kRing - 1)][tid];
    }
    cp_async_wait<0>();
}

// assemble_p (pressure.cpp:14-54) in one pass: links with the wall zeros, APP, b, |b| and b.
__global__ void k_assemble_p(DevParams p, const double* __restrict__ APU,
                             const double* __restrict__ APV, const double* __restrict__ u,
                             const double* __restrict__ v, PressurePtr w, double* __restrict__ cabs,
                             double* __restrict__ cb) {
    const int H = p.H;
    const int j = H + 1 + static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int i = H + static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (i > p.NX + H - 1 || j > p.NY + H) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double dx = p.dx, dy = p.dy;
    const double aep = (j == p.NY + H) ? 0.0 : dy * dy / APU[q];
    const double awp = (j == H + 1) ? 0.0 : dy * dy / APU[q - 1];
    const double anp = (i == H) ? 0.0 : dx * dx / APV[q];
    const double asp = (i == p.NX + H - 1) ? 0.0 : dx * dx / APV[q + ld];
    w.AEP[q] = aep;
    w.AWP[q] = awp;
    w.ANP[q] = anp;
    w.ASP[q] = asp;
    w.APP[q] = aep + awp + anp + asp;
    const double b = -dx * (-v[q + ld] + v[q]) - dy * (-u[q - 1] + u[q]);
    w.b[q] = b;
    const std::size_t c = static_cast<std::size_t>(i - H) * p.NY + (j - H - 1);
    cabs[c] = fabs(b);
    if (cb) cb[c] = b;
}

template <bool V>
void prep_ranges(const DevParams& p, Range& ur, Range& cr) {
    const int H = p.H;
    if (!V) {
        ur = {H, p.NX + H - 1, H + 1, p.NY + H - 1};
        cr = {ur.i0, ur.i1, ur.j0 - 1, ur.j1 + 1}; // coef_u reads uF at j - 1 .. j + 1
    } else {
        ur = {H + 1, p.NX + H - 1, H + 1, p.NY + H};
        cr = {ur.i0 - 1, ur.i1 + 1, ur.j0, ur.j1}; // coef_v reads vF at i - 1 .. i + 1
    }
}

template <int NCOL, bool V, int NT>
void launch_stream(const DevParams& p, const double* xin, double* xout, const double* xF,
                   const double* oth, const double* pf, int seg_rows, cudaStream_t st) {
    constexpr int W = NT - 4 * NCOL;
    const dim3 grid((p.ncols + W - 1) / W, (p.nrows + seg_rows - 1) / seg_rows);
    constexpr int smem = kRing * NT * static_cast<int>(sizeof(double));
    static bool attr_set = false; // per process; the attribute applies to every device
    if (!attr_set) {
        SGPU_CUDA(cudaFuncSetAttribute(k_mom_stream<NCOL, V, NT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_set = true;
    }
    k_mom_stream<NCOL, V, NT><<<grid, NT, smem, st>>>(p, xin, xout, xF, oth, pf, seg_rows);
    SGPU_LAUNCH();
}

} // namespace

// Rows per CTA segment of the streaming sweep: enough segments to fill the GPU (2 CTAs per SM),
// but never so short that the 2 * NCOL-row halo dominates.
int stream_seg_rows(const DevParams& p, int sms) {
    const int W = 256 - 4 * p.ncol;
    const int strips = (p.ncols + W - 1) / W;
    const int want = (2 * sms + strips - 1) / strips;
    int seg = (p.nrows + want - 1) / want;
    const int min_seg = 8 * p.ncol;
    if (seg < min_seg) seg = min_seg;
    return seg;
}

void launch_mom_prep(const DevParams& p, bool v_component, const double* x, const double* oth,
                     const double* pf, double* xF, double* AP, double* cells, cudaStream_t st) {
    Range ur, cr;
    if (v_component) prep_ranges<true>(p, ur, cr);
    else prep_ranges<false>(p, ur, cr);
    if (cr.rows() <= 0 || cr.cols() <= 0) return;
    const dim3 grid((cr.cols() + 31) / 32, (cr.rows() + 7) / 8);
    if (v_component) k_mom_prep<true><<<grid, dim3(32, 8), 0, st>>>(p, x, oth, pf, xF, AP, cells, ur, cr);
    else k_mom_prep<false><<<grid, dim3(32, 8), 0, st>>>(p, x, oth, pf, xF, AP, cells, ur, cr);
    SGPU_LAUNCH();
}

void launch_mom_sweep(const DevParams& p, bool v_component, const double* xin, double* xout,
                      const double* xF, const double* oth, const double* pf, int seg_rows,
                      cudaStream_t st) {
    if (p.ncol == 5) {
        if (v_component) launch_stream<5, true, 256>(p, xin, xout, xF, oth, pf, seg_rows, st);
        else launch_stream<5, false, 256>(p, xin, xout, xF, oth, pf, seg_rows, st);
    } else {
        if (v_component) launch_stream<2, true, 256>(p, xin, xout, xF, oth, pf, seg_rows, st);
        else launch_stream<2, false, 256>(p, xin, xout, xF, oth, pf, seg_rows, st);
    }
}

void launch_assemble_p_fused(const DevParams& p, const double* APU, const double* APV,
                             const double* u, const double* v, PressurePtr w, double* cabs,
                             double* cb, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + 7) / 8);
    k_assemble_p<<<grid, dim3(32, 8), 0, st>>>(p, APU, APV, u, v, w, cabs, cb);
    SGPU_LAUNCH();
}

} // namespace sgpu
