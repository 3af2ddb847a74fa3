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
//    of each cell relative to its neighbours is exactly the reference's colour order. Rows stream
//    through a shared-memory ring filled by cp.async; halo cells are updated redundantly and only
//    the owned block is written, to a second buffer.
// Pressure assembly (assemble_p, pressure.cpp:14-54) is one kernel with the wall zeros folded in.
#include "kernels.hpp"
#include "stencil.cuh"

#include <algorithm>
#include <cstdlib>
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

constexpr int kRing = 32;    // rows held in the shared-memory ring (power of two)
constexpr int kPrefetch = 8; // rows the cp.async ring runs ahead of the rows being read
#ifndef SGPU_STREAM_PF
#define SGPU_STREAM_PF 0
#endif
constexpr int kStreamPF = SGPU_STREAM_PF; // input staging of k_mom_stream (see the kernel)

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The 9 global inputs of one cell's coefficient recomputation and pressure term, read through
// per-thread column pointers (xF, oth, pf already offset by the thread's column) at row offset o.
//   u cell: uF(r, j-1), uF(r, j), uF(r, j+1), v(r, j), v(r, j+1), v(r+1, j), v(r+1, j+1),
//           p(r, j), p(r, j+1)
//   v cell: u(r-1, j), u(r, j), u(r, j-1), u(r-1, j-1), vF(r, j), vF(r-1, j), vF(r+1, j),
//           p(r, j), p(r-1, j)
template <bool V>
__device__ __forceinline__ void load_inputs(const double* __restrict__ xF,
                                            const double* __restrict__ oth,
                                            const double* __restrict__ pf, int o, int ld,
                                            double a[9]) {
    if (!V) {
        const double* f = xF + o;
        const double* g = oth + o;
        const double* h = pf + o;
        a[0] = __ldg(f - 1); a[1] = __ldg(f); a[2] = __ldg(f + 1);
        a[3] = __ldg(g); a[4] = __ldg(g + 1); a[5] = __ldg(g + ld); a[6] = __ldg(g + ld + 1);
        a[7] = __ldg(h); a[8] = __ldg(h + 1);
    } else {
        const double* f = xF + o;
        const double* g = oth + o;
        const double* h = pf + o;
        a[0] = __ldg(g - ld); a[1] = __ldg(g); a[2] = __ldg(g - 1); a[3] = __ldg(g - ld - 1);
        a[4] = __ldg(f); a[5] = __ldg(f - ld); a[6] = __ldg(f + ld);
        a[7] = __ldg(h); a[8] = __ldg(h - ld);
    }
}

// max(0, a) for the coefficient recomputation. The reference's std::max(0.0, a) returns +0.0 for
// a = -0.0, where fmax may return either zero; the sign of that zero never reaches a coefficient,
// because every coefficient adds its diffusive part, which is non-zero or +0.0, to the convective
// part last (coefficients.cpp:5-8), and x + d == x' + d for the two zeros x, x'. NaN gives 0.0 in
// both forms.
__device__ __forceinline__ double mxf(double a) { return fmax(a, 0.0); }

// The 9 coefficients of a momentum cell from its face velocities: convective_coefficients
// (coefficients.cpp:15-39) plus the precomputed diffusive ones (:41-63), specialised on the scheme
// and the diffusion order. Band cells (rare: two rows and two columns) take the UDS / 2nd-order
// branch like the reference; warp_has_band (the same for the whole warp) keeps every other warp
// off that path.
template <bool QUICK, int ORDER>
__device__ __forceinline__ Coef9 coef_spec(const DevParams& p, double ue, double uw, double vn,
                                           double vs, bool band, bool warp_has_band) {
    const double dx = p.dx, dy = p.dy;
    Coef9 c;
    if (QUICK) {
        c.AE = -dy * (-0.75 * mxf(-ue) + 0.375 * mxf(ue) - 0.125 * mxf(-uw));
        c.AW = -dy * (-0.125 * mxf(ue) + 0.375 * mxf(-uw) - 0.75 * mxf(uw));
        c.AN = -dx * (-0.75 * mxf(-vn) + 0.375 * mxf(vn) - 0.125 * mxf(-vs));
        c.AS = -dx * (-0.125 * mxf(vn) + 0.375 * mxf(-vn) - 0.75 * mxf(vs));
        c.AEE = -0.125 * dy * mxf(-ue);
        c.AWW = -0.125 * dy * mxf(uw);
        c.ANN = -0.125 * dx * mxf(-vn);
        c.ASS = -0.125 * dx * mxf(vs);
    } else {
        c.AE = dy * mxf(-ue);
        c.AW = dy * mxf(uw);
        c.AN = dx * mxf(-vn);
        c.AS = dx * mxf(vs);
        c.AEE = c.AWW = c.ANN = c.ASS = 0.0;
    }
    // Diffusive part: the 2nd-order (band) values for ORDER 2, else the 4th-order ones. Indexed
    // directly so the parameter arrays stay in constant space.
#define SGPU_D(k) (ORDER == 2 ? p.dband[k] : p.dint[k])
    c.AP = c.AS + c.AW + c.AN + c.AE + c.ASS + c.AWW + c.ANN + c.AEE;
    c.AE += SGPU_D(0);
    c.AW += SGPU_D(1);
    c.AN += SGPU_D(2);
    c.AS += SGPU_D(3);
    c.AEE += SGPU_D(4);
    c.AWW += SGPU_D(5);
    c.ANN += SGPU_D(6);
    c.ASS += SGPU_D(7);
    c.AP += SGPU_D(8);
#undef SGPU_D
    if (QUICK || ORDER == 4) {
        if (warp_has_band && band) {
            // in_boundary_band: UDS convection and 2nd-order diffusion (coefficients.cpp:20-27, 45-51).
            c.AE = dy * mxf(-ue);
            c.AW = dy * mxf(uw);
            c.AN = dx * mxf(-vn);
            c.AS = dx * mxf(vs);
            c.AP = c.AS + c.AW + c.AN + c.AE + 0.0 + 0.0 + 0.0 + 0.0;
            c.AE += p.dband[0];
            c.AW += p.dband[1];
            c.AN += p.dband[2];
            c.AS += p.dband[3];
            c.AEE = 0.0 + p.dband[4];
            c.AWW = 0.0 + p.dband[5];
            c.ANN = 0.0 + p.dband[6];
            c.ASS = 0.0 + p.dband[7];
            c.AP += p.dband[8];
        }
    }
    return c;
}

__device__ __forceinline__ void prefetch_l1(const double* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// One multicolour sweep of u (V = false) or v (V = true) from xin to xout. NT threads per CTA, one
// column each; the CTA owns W = NT - 4 * NCOL columns starting at blockIdx.x * W and rows
// [blockIdx.y * seg_rows, + seg_rows). For five colours every dependency between two updates is at
// least two steps apart, so two steps run between barriers (SPB = 2). PF selects how the cells'
// global inputs are brought in: 0 = loaded into registers one super-step ahead, 1 = loaded when
// used (more CTAs per SM hide the latency), 2 = their cache lines prefetched into L1 one
// super-step ahead and loaded when used.
template <int NCOL, bool V, int NT, bool QUICK, int ORDER, int PF>
__global__ void __launch_bounds__(NT, PF == 0 ? 2 : 3)
    k_mom_stream(DevParams p, const double* __restrict__ xin, double* __restrict__ xout,
                 const double* __restrict__ xF, const double* __restrict__ oth,
                 const double* __restrict__ pf, int seg_rows) {
    constexpr int SPB = NCOL == 5 ? 2 : 1;       // steps per barrier
    constexpr int HC = 2 * NCOL;                 // halo: a sweep's dependency reach
    constexpr int W = NT - 2 * HC;
    constexpr int A = kPrefetch + SPB + 2;       // rows issued ahead of the first super-step
    static_assert(kPrefetch + 2 * SPB + 1 < kRing - 2 * NCOL, "ring too small for the prefetch");
    extern __shared__ double ring_mem[];
    __shared__ int s_rmin[NCOL], s_rmax[NCOL];
    const int tid = threadIdx.x;
    const int j0 = blockIdx.x * W;
    const int C0 = j0 - HC, C1 = j0 + W + HC; // loaded columns [C0, C1)
    const int col = C0 + tid;
    const int R0 = blockIdx.y * seg_rows;
    const int R1 = min(R0 + seg_rows, p.nrows);
    const int L0 = max(R0 - HC, 0), L1 = min(R1 + HC, p.nrows); // loaded rows [L0, L1)
    const int ld = p.pitch;
    const bool col_in = col >= 0 && col < p.ncols;
    const bool col_out = col_in && col >= j0 && col < j0 + W;
    const int H = p.H;
    // Per colour: the rows a cell of that colour may be updated at (the update range clipped to
    // the window's dependency cone; only cut sides constrain).
    if (tid < NCOL) {
        const int c = tid;
        int lo = V ? H + 1 : H, hi = p.NX + H - 1;
        if (L0 > 0) lo = max(lo, L0 + 2 + 2 * c);
        if (L1 < p.nrows) hi = min(hi, L1 - 3 - 2 * c);
        s_rmin[c] = lo;
        s_rmax[c] = hi;
    }
    // Colours for which this column is updatable (update range and cut columns).
    unsigned colmask = 0;
    {
        const int ju0 = H + 1, ju1 = V ? p.NY + H : p.NY + H - 1;
#pragma unroll
        for (int c = 0; c < NCOL; ++c) {
            bool ok = col >= ju0 && col <= ju1;
            if (C0 > 0) ok = ok && col >= C0 + 2 + 2 * c;
            if (C1 < p.ncols) ok = ok && col <= C1 - 3 - 2 * c;
            colmask |= (ok ? 1u : 0u) << c;
        }
    }
    // Band tests need global indices: in_boundary_band (coefficients.cpp:10-13).
    const bool col_band = col == p.Hy + 1 || col == p.NY + p.Hy;
    const int band_r0 = p.Hx, band_r1 = p.NX + p.Hx - 1;
    const double relax = V ? p.av : p.au;
    const double omr = 1 - relax;
    const double* xFc = xF + col;
    const double* othc = oth + col;
    const double* pfc = pf + col;
    double* ringc = ring_mem + tid; // column tid of ring row k at ringc[k * NT]
    const double* xinc = xin + col;

    int next = L0;
    auto issue = [&]() {
        if (next < L1 && col_in) cp_async8(ringc + (next & (kRing - 1)) * NT, xinc + next * ld);
        cp_async_commit();
        ++next;
    };
    auto step_cell = [&](int c, int t, int& r) -> bool {
        r = t - 2 * c;
        return ((colmask >> c) & 1u) && r >= s_rmin[c] && r <= s_rmax[c];
    };
    auto prefetch_cell = [&](int r) {
        const int o = r * ld;
        if (!V) {
            prefetch_l1(xFc + o);
            prefetch_l1(othc + o);
            prefetch_l1(othc + o + ld);
            prefetch_l1(pfc + o);
        } else {
            prefetch_l1(othc + o - ld);
            prefetch_l1(othc + o);
            prefetch_l1(xFc + o - ld);
            prefetch_l1(xFc + o);
            prefetch_l1(xFc + o + ld);
            prefetch_l1(pfc + o - ld);
            prefetch_l1(pfc + o);
        }
    };
    auto is_band = [&](bool ok, int r) { return ok && (col_band || r == band_r1 || r == band_r0); };
    auto update = [&](int r, const double a[9], bool warp_has_band) {
        double ue, uw, vn, vs, pt;
        if (!V) {
            ue = (a[1] + a[2]) / 2;
            uw = (a[1] + a[0]) / 2;
            vn = (a[3] + a[4]) / 2;
            vs = (a[5] + a[6]) / 2;
            pt = (a[7] - a[8]) * p.dy;
        } else {
            ue = (a[0] + a[1]) / 2;
            uw = (a[2] + a[3]) / 2;
            vn = (a[4] + a[5]) / 2;
            vs = (a[4] + a[6]) / 2;
            pt = (a[7] - a[8]) * p.dx;
        }
        const bool band = col_band || r == band_r1 || r == band_r0;
        const Coef9 k = coef_spec<QUICK, ORDER>(p, ue, uw, vn, vs, band, warp_has_band);
        double* rc = ringc + (r & (kRing - 1)) * NT;
        const double xe = rc[1], xw = rc[-1];
        const double xn = ringc[((r - 1) & (kRing - 1)) * NT];
        const double xs = ringc[((r + 1) & (kRing - 1)) * NT];
        // near_sum for two colours (momentum_u.cpp:84-87), nb_sum for five (:36-41).
        double nb = k.AE * xe + k.AW * xw + k.AN * xn + k.AS * xs;
        if (NCOL == 5) {
            const double xee = rc[2], xww = rc[-2];
            const double xnn = ringc[((r - 2) & (kRing - 1)) * NT];
            const double xss = ringc[((r + 2) & (kRing - 1)) * NT];
            nb = nb + (k.AEE * xee + k.AWW * xww + k.ANN * xnn + k.ASS * xss);
        }
        const double xo = rc[0];
        rc[0] = relax * (nb + pt) / k.AP + omr * xo;
    };

    for (int k = 0; k < A; ++k) issue(); // rows L0 .. L0 + A - 1
    __syncthreads();                     // s_rmin / s_rmax

    const int c_start = NCOL == 5 ? (2 * L0 + col + 1000) % 5 : (L0 + col + 1000) & 1;
    auto next_colour = [&](int c, int steps) {
        return NCOL == 5 ? (c + 2 * steps) % 5 : (c + steps) & 1;
    };
    // Row R1 - 1 is written back by the super-step starting at R1 + 2 NCOL - 2 or one later.
    const int t_last = R1 + 2 * NCOL - 2 + (SPB - 1);

    auto write_back = [&](int t) {
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            const int rw = t - 2 * NCOL + 1 - (SPB - 1) + s;
            if (rw >= R0 && rw < R1 && col_out) xout[col + rw * ld] = ringc[(rw & (kRing - 1)) * NT];
        }
    };

    if (PF == 0) {
        // Register prefetch: two register sets, alternating between consecutive super-steps.
        double bufA[SPB][9], bufB[SPB][9];
        int rA[SPB], rB[SPB];
        bool okA[SPB], okB[SPB];
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            okA[s] = step_cell(next_colour(c_start, s), L0 + s, rA[s]);
            if (okA[s]) load_inputs<V>(xFc, othc, pfc, rA[s] * ld, ld, bufA[s]);
        }
        auto super_step = [&](int t, int c0, double (&cur)[SPB][9], const int (&rcur)[SPB],
                              const bool (&okcur)[SPB], double (&nxt)[SPB][9], int (&rnxt)[SPB],
                              bool (&oknxt)[SPB]) {
            cp_async_wait<kPrefetch>(); // rows <= t + SPB + 1 have landed (this thread's copies)
            __syncthreads();            // ... everyone's, and the previous super-step's updates
#pragma unroll
            for (int s = 0; s < SPB; ++s) issue();
            const int cn = next_colour(c0, SPB);
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                oknxt[s] = step_cell(next_colour(cn, s), t + SPB + s, rnxt[s]);
                if (oknxt[s]) load_inputs<V>(xFc, othc, pfc, rnxt[s] * ld, ld, nxt[s]);
            }
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                const bool wb = __any_sync(0xffffffffu, is_band(okcur[s], rcur[s]));
                if (okcur[s]) update(rcur[s], cur[s], wb);
            }
            write_back(t);
            return cn;
        };
        int c0 = c_start;
        for (int t = L0; t <= t_last; t += 2 * SPB) {
            c0 = super_step(t, c0, bufA, rA, okA, bufB, rB, okB);
            if (t + SPB <= t_last) c0 = super_step(t + SPB, c0, bufB, rB, okB, bufA, rA, okA);
        }
    } else {
        int c0 = c_start;
        if (PF == 2) {
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                int r;
                if (step_cell(next_colour(c0, s), L0 + s, r)) prefetch_cell(r);
            }
        }
        for (int t = L0; t <= t_last; t += SPB) {
            cp_async_wait<kPrefetch>();
            __syncthreads();
#pragma unroll
            for (int s = 0; s < SPB; ++s) issue();
            const int cn = next_colour(c0, SPB);
            if (PF == 2) {
#pragma unroll
                for (int s = 0; s < SPB; ++s) {
                    int r;
                    if (step_cell(next_colour(cn, s), t + SPB + s, r)) prefetch_cell(r);
                }
            }
            int r[SPB];
            bool ok[SPB];
            double a[SPB][9];
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                ok[s] = step_cell(next_colour(c0, s), t + s, r[s]);
                if (ok[s]) load_inputs<V>(xFc, othc, pfc, r[s] * ld, ld, a[s]);
            }
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                const bool wb = __any_sync(0xffffffffu, is_band(ok[s], r[s]));
                if (ok[s]) update(r[s], a[s], wb);
            }
            write_back(t);
            c0 = cn;
        }
    }
    cp_async_wait<0>();
}

// assemble_p (pressure.cpp:14-54) in one pass: links with the wall zeros, APP, b, |b| and b. Each
// thread assembles the two cells (j, j + 1) of a column pair (j even; the pitch is even): the FP64
// inputs and outputs move as 16-byte pairs (a single store where only one of the two is a cell).
// The per-cell expressions are the reference's.
__device__ __forceinline__ double2 ld2(const double* q) { return *reinterpret_cast<const double2*>(q); }
__global__ void k_assemble_p(DevParams p, const double* __restrict__ APU,
                             const double* __restrict__ APV, const double* __restrict__ u,
                             const double* __restrict__ v, PressurePtr w, double* __restrict__ cabs,
                             double* __restrict__ cb) {
    const int H = p.H;
    const int j = ((H + 1) & ~1) + 2 * static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int i = H + static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (i > p.NX + H - 1 || j > p.NY + H) return;
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    const double dx = p.dx, dy = p.dy;
    const double2 apu = ld2(APU + q), apv = ld2(APV + q), apvs = ld2(APV + q + ld);
    const double2 uu = ld2(u + q), vv = ld2(v + q), vs = ld2(v + q + ld);
    const double apuw = APU[q - 1], uw = u[q - 1];
    const double apu_e[2] = {apu.x, apu.y}, apu_w[2] = {apuw, apu.x};
    const double apv_n[2] = {apv.x, apv.y}, apv_s[2] = {apvs.x, apvs.y};
    const double u_e[2] = {uu.x, uu.y}, u_w[2] = {uw, uu.x};
    const double v_n[2] = {vv.x, vv.y}, v_s[2] = {vs.x, vs.y};
    double ae[2], aw[2], an[2], as[2], ap[2], bb[2];
    bool cell[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int jj = j + e;
        cell[e] = jj >= H + 1 && jj <= p.NY + H;
        if (!cell[e]) continue;
        ae[e] = (jj == p.NY + H) ? 0.0 : dy * dy / apu_e[e];
        aw[e] = (jj == H + 1) ? 0.0 : dy * dy / apu_w[e];
        an[e] = (i == H) ? 0.0 : dx * dx / apv_n[e];
        as[e] = (i == p.NX + H - 1) ? 0.0 : dx * dx / apv_s[e];
        ap[e] = ae[e] + aw[e] + an[e] + as[e];
        bb[e] = -dx * (-v_s[e] + v_n[e]) - dy * (-u_w[e] + u_e[e]);
        const std::size_t c = static_cast<std::size_t>(i - H) * p.NY + (jj - H - 1);
        if (cabs) cabs[c] = fabs(bb[e]);
        if (cb) cb[c] = bb[e];
    }
    auto put = [&](double* dst, const double* val) {
        if (cell[0] && cell[1]) *reinterpret_cast<double2*>(dst + q) = make_double2(val[0], val[1]);
        else if (cell[0]) dst[q] = val[0];
        else if (cell[1]) dst[q + 1] = val[1];
    };
    put(w.AEP, ae);
    put(w.AWP, aw);
    put(w.ANP, an);
    put(w.ASP, as);
    put(w.APP, ap);
    put(w.b, bb);
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

template <int NCOL, bool V, int NT, bool QUICK, int ORDER, int PF>
void launch_stream(const DevParams& p, const double* xin, double* xout, const double* xF,
                   const double* oth, const double* pf, int seg_rows, cudaStream_t st) {
    constexpr int W = NT - 4 * NCOL;
    const dim3 grid((p.ncols + W - 1) / W, (p.nrows + seg_rows - 1) / seg_rows);
    constexpr int smem = kRing * NT * static_cast<int>(sizeof(double));
    static PerDeviceOnce attr; // the attribute lives in each device's context
    attr.get([] {
        SGPU_CUDA(cudaFuncSetAttribute(k_mom_stream<NCOL, V, NT, QUICK, ORDER, PF>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return 0;
    });
    k_mom_stream<NCOL, V, NT, QUICK, ORDER, PF><<<grid, NT, smem, st>>>(p, xin, xout, xF, oth, pf, seg_rows);
    SGPU_LAUNCH();
}

template <bool V, int PF>
void launch_stream_v(const DevParams& p, const double* xin, double* xout, const double* xF,
                     const double* oth, const double* pf, int seg_rows, cudaStream_t st) {
    if (p.uds && p.order == 2) launch_stream<2, V, 256, false, 2, PF>(p, xin, xout, xF, oth, pf, seg_rows, st);
    else if (p.uds) launch_stream<5, V, 256, false, 4, PF>(p, xin, xout, xF, oth, pf, seg_rows, st);
    else if (p.order == 2) launch_stream<5, V, 256, true, 2, PF>(p, xin, xout, xF, oth, pf, seg_rows, st);
    else launch_stream<5, V, 256, true, 4, PF>(p, xin, xout, xF, oth, pf, seg_rows, st);
}

} // namespace

// Rows per CTA segment of the streaming sweep: enough segments to fill the GPU with one wave of
// 2 CTAs per SM, but never so short that the 2 * NCOL-row halo dominates.
int stream_seg_rows(const DevParams& p, int sms, int blocks_per_sm, int min_seg, int nt) {
    const int W = nt - 4 * p.ncol;
    const int strips = (p.ncols + W - 1) / W;
    const int want = std::max(1, (blocks_per_sm * sms) / strips); // one wave of resident CTAs
    int seg = (p.nrows + want - 1) / want;
    const int lo = min_seg > 0 ? min_seg : 8 * p.ncol;
    if (seg < lo) seg = lo;
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
    if (v_component) launch_stream_v<true, kStreamPF>(p, xin, xout, xF, oth, pf, seg_rows, st);
    else launch_stream_v<false, kStreamPF>(p, xin, xout, xF, oth, pf, seg_rows, st);
}

void launch_assemble_p_fused(const DevParams& p, const double* APU, const double* APV,
                             const double* u, const double* v, PressurePtr w, double* cabs,
                             double* cb, cudaStream_t st) {
    const int pairs = (p.NY + p.H - ((p.H + 1) & ~1)) / 2 + 1; // column pairs over j = H + 1 .. NY + H
    const dim3 grid((pairs + 31) / 32, (p.NX + 7) / 8);
    k_assemble_p<<<grid, dim3(32, 8), 0, st>>>(p, APU, APV, u, v, w, cabs, cb);
    SGPU_LAUNCH();
}

} // namespace sgpu
