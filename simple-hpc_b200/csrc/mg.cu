// mg.cu — geometric multigrid for p' on the device, bit-identical to the reference in FP64.
//
// The reference runs multigrid on the CPU only (src/multigrid.cpp). These kernels restate each of
// its loops with the same per-cell expression order: the Galerkin 2x2 build (mg_build, :232-261),
// the red-black two-statement smoother (smooth, :46-70), residual (:73-87), restriction (:90-103),
// prolongation with over-correction (:106-116), and the coarsest-level solve with its fixed-order
// norms (coarse_solve, :120-140), which runs inside one CTA so its data-dependent sweep count
// needs no host round trip. Every kernel is a template on the element type: double gives the
// reference's bits; float is the mixed-precision mode's V-cycle (sums and norms still in double).
#include "kernels.hpp"
#include "blocksum.cuh"

namespace sgpu {

namespace {

constexpr int BX = 32, BY = 8;

dim3 grid2(int nx, int ny) { return dim3((ny + BX - 1) / BX, (nx + BY - 1) / BY); }

// mg_build: coarse links are the sums of the two fine links crossing each coarse face.
template <class T> __global__ void k_mg_build(LevelViewT<T> F, LevelViewT<T> C) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= C.nx || J >= C.ny) return;
    const int fs = F.stride;
    const int f = 2 * I * fs + 2 * J, c = I * C.stride + J;
    const Links<T> k00 = links(F, f), k01 = links(F, f + 1), k10 = links(F, f + fs), k11 = links(F, f + fs + 1);
    const T ae = k01.e + k11.e;
    const T aw = k00.w + k10.w;
    const T an = k00.n + k01.n;
    const T as = k10.s + k11.s;
    set_links(C, c, ae, aw, an, as);
    C.AP[c] = ae + aw + an + as;
}

// One colour of smooth: colour (I + J) & 1, update x = b/AP; x += (E W S N)/AP.
template <class T> __global__ void k_mg_smooth(LevelViewT<T> L, int colour) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny || ((I + J) & 1) != colour) return;
    const int s = L.stride, q = I * s + J;
    T* x = L.x;
    const Links<T> k = links(L, q);
    x[q] = rb_value(L.b[q], k.e * x[q + 1] + k.w * x[q - 1] + k.s * x[q + s] + k.n * x[q - s], L.AP[q]);
}

template <class T> __global__ void k_mg_residual(LevelViewT<T> L) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const int s = L.stride, q = I * s + J;
    const T* x = L.x;
    const Links<T> k = links(L, q);
    L.r[q] = L.b[q] - (L.AP[q] * x[q] - (k.e * x[q + 1] + k.w * x[q - 1] + k.s * x[q + s] + k.n * x[q - s]));
}

template <class T> __global__ void k_mg_restrict(LevelViewT<T> F, LevelViewT<T> C) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= F.nx / 2 || J >= F.ny / 2) return;
    const int fs = F.stride, f = 2 * I * fs + 2 * J, c = I * C.stride + J;
    C.b[c] = F.r[f] + F.r[f + 1] + F.r[f + fs] + F.r[f + fs + 1];
    C.x[c] = T(0);
}

template <class T> __global__ void k_mg_prolong(LevelViewT<T> C, LevelViewT<T> F, double omega) {
    const int j = blockIdx.x * BX + threadIdx.x, i = blockIdx.y * BY + threadIdx.y;
    if (i >= F.nx || j >= F.ny) return;
    F.x[i * F.stride + j] += static_cast<T>(omega) * C.x[(i / 2) * C.stride + j / 2];
}

// Squares of the level residual r = b - A x (multigrid.cpp:84-85 form), in FP64, one per cell of a
// compact nx x ny plane, for the ordered norm of the tolerance-driven V-cycle loop.
template <class T> __global__ void k_mg_residual_sq(LevelViewT<T> L, double* cells) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const int s = L.stride, q = I * s + J;
    const T* x = L.x;
    const Links<T> k = links(L, q);
    const double r = static_cast<double>(L.b[q]) -
                     (static_cast<double>(L.AP[q]) * x[q] -
                      (static_cast<double>(k.e) * x[q + 1] + static_cast<double>(k.w) * x[q - 1] +
                       static_cast<double>(k.s) * x[q + s] + static_cast<double>(k.n) * x[q - s]));
    cells[static_cast<std::size_t>(I) * L.ny + J] = r * r;
}

// Squares of b, for ||b|| of the same loop.
template <class T> __global__ void k_mg_b_sq(LevelViewT<T> L, double* cells) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const double b = L.b[I * L.stride + J];
    cells[static_cast<std::size_t>(I) * L.ny + J] = b * b;
}

__global__ void k_mg_sub_mean(LevelView L, double* x, const double* sum) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const double m = *sum / (static_cast<double>(L.nx) * L.ny);
    x[I * L.stride + J] -= m;
}

// ---- levels inside one CTA ----

constexpr int kCoarseThreads = 512;

// det_sum (multigrid.cpp:18-34) of f(q) in one CTA: one thread per row chain, then row order.
// Accumulates in double for both element types.
template <class T, class F>
__device__ double cta_det_sum(const LevelViewT<T>& L, double* rowbuf, F f) {
    for (int I = threadIdx.x; I < L.nx; I += blockDim.x) {
        double s = 0.0;
        for (int J = 0; J < L.ny; ++J) s += f(I * L.stride + J);
        rowbuf[I] = s;
    }
    __syncthreads();
    __shared__ double total;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int I = 0; I < L.nx; ++I) s += rowbuf[I];
        total = s;
    }
    __syncthreads();
    const double t = total;
    __syncthreads();
    return t;
}

template <class T> __device__ void cta_remove_mean(const LevelViewT<T>& L, double* rowbuf, T* x) {
    const double m = cta_det_sum(L, rowbuf, [x](int q) { return static_cast<double>(x[q]); }) /
                     (static_cast<double>(L.nx) * L.ny);
    const int n = L.nx * L.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny;
        x[I * L.stride + J] = static_cast<T>(x[I * L.stride + J] - m);
    }
    __syncthreads();
}

template <class T> __device__ void cta_smooth_colour(const LevelViewT<T>& L, int colour) {
    const int n = L.nx * L.ny, s = L.stride;
    T* x = L.x;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny;
        if (((I + J) & 1) != colour) continue;
        const int q = I * s + J;
        const Links<T> k4 = links(L, q);
        x[q] = rb_value(L.b[q], k4.e * x[q + 1] + k4.w * x[q - 1] + k4.s * x[q + s] + k4.n * x[q - s], L.AP[q]);
    }
    __syncthreads();
}

template <class T> __device__ void cta_residual(const LevelViewT<T>& L) {
    const int n = L.nx * L.ny, s = L.stride;
    const T* x = L.x;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny, q = I * s + J;
        const Links<T> k4 = links(L, q);
        L.r[q] = L.b[q] - (L.AP[q] * x[q] - (k4.e * x[q + 1] + k4.w * x[q - 1] + k4.s * x[q + s] + k4.n * x[q - s]));
    }
    __syncthreads();
}

// restrict_residual (multigrid.cpp:90-103) inside one CTA.
template <class T> __device__ void cta_restrict(const LevelViewT<T>& F, const LevelViewT<T>& C) {
    const int n = C.nx * C.ny, fs = F.stride;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / C.ny, J = k % C.ny;
        const int f = 2 * I * fs + 2 * J, c = I * C.stride + J;
        C.b[c] = F.r[f] + F.r[f + 1] + F.r[f + fs] + F.r[f + fs + 1];
        C.x[c] = T(0);
    }
    __syncthreads();
}

// prolong (multigrid.cpp:106-116) inside one CTA.
template <class T>
__device__ void cta_prolong(const LevelViewT<T>& C, const LevelViewT<T>& F, double omega) {
    const int n = F.nx * F.ny;
    const T om = static_cast<T>(omega);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int i = k / F.ny, j = k % F.ny;
        F.x[i * F.stride + j] += om * C.x[(i / 2) * C.stride + j / 2];
    }
    __syncthreads();
}

// coarse_solve (multigrid.cpp:120-140): remove the mean of b; red-black sweeps until
// ||b - A x|| < tol ||b|| (tol = 1e-10 in the reference) or 200 sweeps; remove the mean of x.
template <class T>
__device__ void cta_coarse_solve(const LevelViewT<T>& L, double* rowbuf, double tol, int* sweeps_out) {
    cta_remove_mean(L, rowbuf, L.b);
    const T* b = L.b;
    const double bb = cta_det_sum(L, rowbuf, [b](int q) {
        const double v = b[q];
        return v * v;
    });
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        const T* r = L.r;
        while (sweeps < 200) {
            cta_smooth_colour(L, 0);
            cta_smooth_colour(L, 1);
            ++sweeps;
            cta_residual(L);
            const double rr = cta_det_sum(L, rowbuf, [r](int q) {
                const double v = r[q];
                return v * v;
            });
            if (sqrt(rr) < tol * bn) break;
        }
    }
    cta_remove_mean(L, rowbuf, L.x);
    if (threadIdx.x == 0 && sweeps_out) *sweeps_out = sweeps;
}

// The float V-cycle's coarse_solve in one warp, with the level (x, b, AP and links, zero ring
// included) copied to shared memory: the same red-black sweeps, stopping test (||b - A x|| <
// tol ||b|| or 200 sweeps) and mean removals as cta_coarse_solve, but no block barrier per pass,
// which on a level of a few cells is most of a pass's cost. Its sums are FP64: each lane adds its
// cells in order and a fixed xor-shuffle tree combines the lanes (not the reference's row chain,
// which only the FP64 V-cycle needs). Levels of up to kWarpCoarseCells cells with their ring.
constexpr int kWarpCoarseCells = 1024;

__device__ void warp_coarse_solve(const LevelViewT<float>& L, double tol, int* sweeps_out) {
    __shared__ float sx[kWarpCoarseCells], sb[kWarpCoarseCells], sap[kWarpCoarseCells];
    __shared__ float4 sl[kWarpCoarseCells];
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int S = L.ny + 2, n2 = (L.nx + 2) * S, n = L.nx * L.ny;
    for (int k = lane; k < n2; k += 32) { // (I, J) in [-1, nx] x [-1, ny]
        const int I = k / S - 1, J = k % S - 1;
        const int q = I * L.stride + J;
        sx[k] = L.x[q];
        const bool in = I >= 0 && I < L.nx && J >= 0 && J < L.ny;
        sb[k] = in ? L.b[q] : 0.0f;
        sap[k] = in ? L.AP[q] : 0.0f;
        if (in) {
            const Links<float> a = links(L, q);
            sl[k] = make_float4(a.e, a.w, a.n, a.s);
        }
    }
    __syncwarp();
    // cell k of the interior (row-major) at smem index (I + 1) * S + J + 1
    auto at = [&](int k) {
        const int I = k / L.ny;
        return (I + 1) * S + (k - I * L.ny) + 1;
    };
    auto sum = [&](auto f) {
        double a = 0.0;
        for (int k = lane; k < n; k += 32) a += f(at(k));
        return warp_sum(a);
    };
    auto smooth = [&](int colour) {
        for (int k = lane; k < n; k += 32) {
            const int I = k / L.ny, J = k - I * L.ny;
            if (((I + J) & 1) != colour) continue;
            const int q = (I + 1) * S + J + 1;
            const float4 a = sl[q];
            sx[q] = rb_value(sb[q], a.x * sx[q + 1] + a.y * sx[q - 1] + a.w * sx[q + S] + a.z * sx[q - S], sap[q]);
        }
        __syncwarp();
    };
    const double dn = static_cast<double>(L.nx) * L.ny;
    const double mb = sum([&](int q) { return static_cast<double>(sb[q]); }) / dn;
    for (int k = lane; k < n; k += 32) {
        const int q = at(k);
        sb[q] = static_cast<float>(sb[q] - mb);
    }
    __syncwarp();
    const double bb = sum([&](int q) {
        const double v = sb[q];
        return v * v;
    });
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        while (sweeps < 200) {
            smooth(0);
            smooth(1);
            ++sweeps;
            const double rr = sum([&](int q) {
                const float4 a = sl[q];
                const double r = sb[q] - (sap[q] * sx[q] - (a.x * sx[q + 1] + a.y * sx[q - 1] + a.w * sx[q + S] +
                                                            a.z * sx[q - S]));
                return r * r;
            });
            if (sqrt(rr) < tol * bn) break;
        }
    }
    const double mx = sum([&](int q) { return static_cast<double>(sx[q]); }) / dn;
    for (int k = lane; k < n; k += 32) {
        const int I = k / L.ny, J = k - I * L.ny, q = (I + 1) * S + J + 1;
        L.x[I * L.stride + J] = static_cast<float>(sx[q] - mx);
        L.b[I * L.stride + J] = sb[q];
    }
    if (lane == 0 && sweeps_out) *sweeps_out = sweeps;
}

template <class T>
__global__ void __launch_bounds__(kCoarseThreads) k_mg_coarse(LevelViewT<T> L, double* rowbuf,
                                                              double tol, int* sweeps_out) {
    cta_coarse_solve(L, rowbuf, tol, sweeps_out);
}

// Levels [first, nl) of one V-cycle (mg_vcycle, multigrid.cpp:299-323) in one CTA: the small
// levels are latency-bound, so they run back to back with a block barrier between passes.
template <class T>
__global__ void __launch_bounds__(kCoarseThreads)
    k_mg_tail(MgLevelsT<T> lv, int first, int pre, int post, double omega, double tol,
              double* rowbuf, int* sweeps_out) {
    const int nl = lv.n;
    for (int l = first; l + 1 < nl; ++l) {
        for (int s = 0; s < pre; ++s) {
            cta_smooth_colour(lv.L[l], 0);
            cta_smooth_colour(lv.L[l], 1);
        }
        cta_residual(lv.L[l]);
        cta_restrict(lv.L[l], lv.L[l + 1]);
    }
    bool warp_solve = false;
    if constexpr (sizeof(T) == 4)
        warp_solve = (lv.L[nl - 1].nx + 2) * (lv.L[nl - 1].ny + 2) <= kWarpCoarseCells;
    if (warp_solve) {
        if constexpr (sizeof(T) == 4)
            if (threadIdx.x < 32) warp_coarse_solve(lv.L[nl - 1], tol, sweeps_out);
        __syncthreads();
    } else {
        cta_coarse_solve(lv.L[nl - 1], rowbuf, tol, sweeps_out);
    }
    for (int l = nl - 2; l >= first; --l) {
        cta_prolong(lv.L[l + 1], lv.L[l], omega);
        for (int s = 0; s < post; ++s) {
            cta_smooth_colour(lv.L[l], 0);
            cta_smooth_colour(lv.L[l], 1);
        }
    }
}

} // namespace

template <class T>
void launch_mg_tail(const MgLevelsT<T>& lv, int first, int pre, int post, double omega, double tol,
                    double* rowbuf, int* sweeps_out, cudaStream_t st) {
    k_mg_tail<T><<<1, kCoarseThreads, 0, st>>>(lv, first, pre, post, omega, tol, rowbuf, sweeps_out);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_build(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st) {
    k_mg_build<T><<<grid2(C.nx, C.ny), dim3(BX, BY), 0, st>>>(F, C);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_smooth_colour(const LevelViewT<T>& L, int colour, cudaStream_t st) {
    k_mg_smooth<T><<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, colour);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_residual(const LevelViewT<T>& L, cudaStream_t st) {
    k_mg_residual<T><<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_restrict(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st) {
    k_mg_restrict<T><<<grid2(F.nx / 2, F.ny / 2), dim3(BX, BY), 0, st>>>(F, C);
    SGPU_LAUNCH();
}
template <class T>
void launch_mg_prolong(const LevelViewT<T>& C, const LevelViewT<T>& F, double omega, cudaStream_t st) {
    k_mg_prolong<T><<<grid2(F.nx, F.ny), dim3(BX, BY), 0, st>>>(C, F, omega);
    SGPU_LAUNCH();
}
template <class T>
void launch_mg_coarse(const LevelViewT<T>& L, double* rowbuf, double tol, int* sweeps_out, cudaStream_t st) {
    k_mg_coarse<T><<<1, kCoarseThreads, 0, st>>>(L, rowbuf, tol, sweeps_out);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_residual_sq(const LevelViewT<T>& L, double* cells, cudaStream_t st) {
    k_mg_residual_sq<T><<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, cells);
    SGPU_LAUNCH();
}
template <class T> void launch_mg_b_sq(const LevelViewT<T>& L, double* cells, cudaStream_t st) {
    k_mg_b_sq<T><<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, cells);
    SGPU_LAUNCH();
}
#ifndef SGPU_FLOAT_UNIT
void launch_mg_sub_mean(const LevelView& L, double* x, const double* sum, cudaStream_t st) {
    k_mg_sub_mean<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, x, sum);
    SGPU_LAUNCH();
}
#endif

#define SGPU_MG_INST(T)                                                                            \
    template void launch_mg_tail<T>(const MgLevelsT<T>&, int, int, int, double, double, double*,   \
                                    int*, cudaStream_t);                                           \
    template void launch_mg_build<T>(const LevelViewT<T>&, const LevelViewT<T>&, cudaStream_t);    \
    template void launch_mg_smooth_colour<T>(const LevelViewT<T>&, int, cudaStream_t);             \
    template void launch_mg_residual<T>(const LevelViewT<T>&, cudaStream_t);                       \
    template void launch_mg_restrict<T>(const LevelViewT<T>&, const LevelViewT<T>&, cudaStream_t); \
    template void launch_mg_prolong<T>(const LevelViewT<T>&, const LevelViewT<T>&, double,         \
                                       cudaStream_t);                                              \
    template void launch_mg_coarse<T>(const LevelViewT<T>&, double*, double, int*, cudaStream_t);  \
    template void launch_mg_residual_sq<T>(const LevelViewT<T>&, double*, cudaStream_t);           \
    template void launch_mg_b_sq<T>(const LevelViewT<T>&, double*, cudaStream_t);
// This file alone instantiates the double kernels (built without contraction: the reference's
// bits); mg32.cu includes it with SGPU_FLOAT_UNIT for the float ones (contraction allowed).
#ifndef SGPU_FLOAT_UNIT
SGPU_MG_INST(double)
#else
SGPU_MG_INST(float)
#endif
#undef SGPU_MG_INST

} // namespace sgpu
