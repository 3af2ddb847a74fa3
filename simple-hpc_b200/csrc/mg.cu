// mg.cu — geometric multigrid for p' on the device, FP64, bit-identical to the reference.
//
// The reference runs multigrid on the CPU only (src/multigrid.cpp). These kernels restate each of
// its loops with the same per-cell expression order: the Galerkin 2x2 build (mg_build, :232-261),
// the red-black two-statement smoother (smooth, :46-70), residual (:73-87), restriction (:90-103),
// prolongation with over-correction (:106-116), and the coarsest-level solve with its fixed-order
// norms (coarse_solve, :120-140), which runs inside one CTA so its data-dependent sweep count
// needs no host round trip.
#include "kernels.hpp"

namespace sgpu {

namespace {

constexpr int BX = 32, BY = 8;

dim3 grid2(int nx, int ny) { return dim3((ny + BX - 1) / BX, (nx + BY - 1) / BY); }

// mg_build: coarse links are the sums of the two fine links crossing each coarse face.
__global__ void k_mg_build(LevelView F, LevelView C) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= C.nx || J >= C.ny) return;
    const int fs = F.stride;
    const int f = 2 * I * fs + 2 * J, c = I * C.stride + J;
    const double ae = F.AE[f + 1] + F.AE[f + fs + 1];
    const double aw = F.AW[f] + F.AW[f + fs];
    const double an = F.AN[f] + F.AN[f + 1];
    const double as = F.AS[f + fs] + F.AS[f + fs + 1];
    C.AE[c] = ae;
    C.AW[c] = aw;
    C.AN[c] = an;
    C.AS[c] = as;
    C.AP[c] = ae + aw + an + as;
}

// One colour of smooth: colour (I + J) & 1, update x = b/AP; x += (E W S N)/AP.
__global__ void k_mg_smooth(LevelView L, int colour) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny || ((I + J) & 1) != colour) return;
    const int s = L.stride, q = I * s + J;
    double* x = L.x;
    double t = L.b[q] / L.AP[q];
    t += (L.AE[q] * x[q + 1] + L.AW[q] * x[q - 1] + L.AS[q] * x[q + s] + L.AN[q] * x[q - s]) / L.AP[q];
    x[q] = t;
}

__global__ void k_mg_residual(LevelView L) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const int s = L.stride, q = I * s + J;
    const double* x = L.x;
    L.r[q] = L.b[q] - (L.AP[q] * x[q] -
                       (L.AE[q] * x[q + 1] + L.AW[q] * x[q - 1] + L.AS[q] * x[q + s] +
                        L.AN[q] * x[q - s]));
}

__global__ void k_mg_restrict(LevelView F, LevelView C) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= F.nx / 2 || J >= F.ny / 2) return;
    const int fs = F.stride, f = 2 * I * fs + 2 * J, c = I * C.stride + J;
    C.b[c] = F.r[f] + F.r[f + 1] + F.r[f + fs] + F.r[f + fs + 1];
    C.x[c] = 0.0;
}

__global__ void k_mg_prolong(LevelView C, LevelView F, double omega) {
    const int j = blockIdx.x * BX + threadIdx.x, i = blockIdx.y * BY + threadIdx.y;
    if (i >= F.nx || j >= F.ny) return;
    F.x[i * F.stride + j] += omega * C.x[(i / 2) * C.stride + j / 2];
}

__global__ void k_mg_sub_mean(LevelView L, double* x, const double* sum) {
    const int J = blockIdx.x * BX + threadIdx.x, I = blockIdx.y * BY + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const double m = *sum / (static_cast<double>(L.nx) * L.ny);
    x[I * L.stride + J] -= m;
}

// ---- coarsest level in one CTA ----

constexpr int kCoarseThreads = 512;

// det_sum (multigrid.cpp:18-34) of f(q) in one CTA: one thread per row chain, then row order.
template <class F>
__device__ double cta_det_sum(const LevelView& L, double* rowbuf, F f) {
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

__device__ void cta_remove_mean(const LevelView& L, double* rowbuf, double* x) {
    const double m =
        cta_det_sum(L, rowbuf, [x](int q) { return x[q]; }) / (static_cast<double>(L.nx) * L.ny);
    const int n = L.nx * L.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny;
        x[I * L.stride + J] -= m;
    }
    __syncthreads();
}

__device__ void cta_smooth_colour(const LevelView& L, int colour) {
    const int n = L.nx * L.ny, s = L.stride;
    double* x = L.x;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny;
        if (((I + J) & 1) != colour) continue;
        const int q = I * s + J;
        double t = L.b[q] / L.AP[q];
        t += (L.AE[q] * x[q + 1] + L.AW[q] * x[q - 1] + L.AS[q] * x[q + s] + L.AN[q] * x[q - s]) /
             L.AP[q];
        x[q] = t;
    }
    __syncthreads();
}

__device__ void cta_residual(const LevelView& L) {
    const int n = L.nx * L.ny, s = L.stride;
    const double* x = L.x;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k % L.ny, q = I * s + J;
        L.r[q] = L.b[q] - (L.AP[q] * x[q] - (L.AE[q] * x[q + 1] + L.AW[q] * x[q - 1] +
                                             L.AS[q] * x[q + s] + L.AN[q] * x[q - s]));
    }
    __syncthreads();
}

// coarse_solve (multigrid.cpp:120-140): remove the mean of b; red-black sweeps until
// ||b - A x|| < 1e-10 ||b|| or 200 sweeps; remove the mean of x.
__global__ void __launch_bounds__(kCoarseThreads) k_mg_coarse(LevelView L, double* rowbuf,
                                                              int* sweeps_out) {
    cta_remove_mean(L, rowbuf, L.b);
    const double* b = L.b;
    const double bb = cta_det_sum(L, rowbuf, [b](int q) { return b[q] * b[q]; });
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        const double* r = L.r;
        while (sweeps < 200) {
            cta_smooth_colour(L, 0);
            cta_smooth_colour(L, 1);
            ++sweeps;
            cta_residual(L);
            const double rr = cta_det_sum(L, rowbuf, [r](int q) { return r[q] * r[q]; });
            if (sqrt(rr) < 1e-10 * bn) break;
        }
    }
    cta_remove_mean(L, rowbuf, L.x);
    if (threadIdx.x == 0 && sweeps_out) *sweeps_out = sweeps;
}

// restrict_residual (multigrid.cpp:90-103) inside one CTA.
__device__ void cta_restrict(const LevelView& F, const LevelView& C) {
    const int n = C.nx * C.ny, fs = F.stride;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / C.ny, J = k % C.ny;
        const int f = 2 * I * fs + 2 * J, c = I * C.stride + J;
        C.b[c] = F.r[f] + F.r[f + 1] + F.r[f + fs] + F.r[f + fs + 1];
        C.x[c] = 0.0;
    }
    __syncthreads();
}

// prolong (multigrid.cpp:106-116) inside one CTA.
__device__ void cta_prolong(const LevelView& C, const LevelView& F, double omega) {
    const int n = F.nx * F.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int i = k / F.ny, j = k % F.ny;
        F.x[i * F.stride + j] += omega * C.x[(i / 2) * C.stride + j / 2];
    }
    __syncthreads();
}

// Levels [first, nl) of one V-cycle (mg_vcycle, multigrid.cpp:299-323) in one CTA: the small
// levels are latency-bound, so they run back to back with a block barrier between passes.
__global__ void __launch_bounds__(kCoarseThreads)
    k_mg_tail(MgLevels lv, int first, int pre, int post, double omega, double* rowbuf,
              int* sweeps_out) {
    const int nl = lv.n;
    for (int l = first; l + 1 < nl; ++l) {
        for (int s = 0; s < pre; ++s) {
            cta_smooth_colour(lv.L[l], 0);
            cta_smooth_colour(lv.L[l], 1);
        }
        cta_residual(lv.L[l]);
        cta_restrict(lv.L[l], lv.L[l + 1]);
    }
    // coarse_solve (multigrid.cpp:120-140)
    const LevelView& L = lv.L[nl - 1];
    cta_remove_mean(L, rowbuf, L.b);
    const double* b = L.b;
    const double bb = cta_det_sum(L, rowbuf, [b](int q) { return b[q] * b[q]; });
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        const double* r = L.r;
        while (sweeps < 200) {
            cta_smooth_colour(L, 0);
            cta_smooth_colour(L, 1);
            ++sweeps;
            cta_residual(L);
            const double rr = cta_det_sum(L, rowbuf, [r](int q) { return r[q] * r[q]; });
            if (sqrt(rr) < 1e-10 * bn) break;
        }
    }
    cta_remove_mean(L, rowbuf, L.x);
    if (threadIdx.x == 0 && sweeps_out) *sweeps_out = sweeps;
    for (int l = nl - 2; l >= first; --l) {
        cta_prolong(lv.L[l + 1], lv.L[l], omega);
        for (int s = 0; s < post; ++s) {
            cta_smooth_colour(lv.L[l], 0);
            cta_smooth_colour(lv.L[l], 1);
        }
    }
}

} // namespace

void launch_mg_tail(const MgLevels& lv, int first, int pre, int post, double omega, double* rowbuf,
                    int* sweeps_out, cudaStream_t st) {
    k_mg_tail<<<1, kCoarseThreads, 0, st>>>(lv, first, pre, post, omega, rowbuf, sweeps_out);
    SGPU_LAUNCH();
}

void launch_mg_build(const LevelView& F, const LevelView& C, cudaStream_t st) {
    k_mg_build<<<grid2(C.nx, C.ny), dim3(BX, BY), 0, st>>>(F, C);
    SGPU_LAUNCH();
}
void launch_mg_smooth_colour(const LevelView& L, int colour, cudaStream_t st) {
    k_mg_smooth<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, colour);
    SGPU_LAUNCH();
}
void launch_mg_residual(const LevelView& L, cudaStream_t st) {
    k_mg_residual<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L);
    SGPU_LAUNCH();
}
void launch_mg_restrict(const LevelView& F, const LevelView& C, cudaStream_t st) {
    k_mg_restrict<<<grid2(F.nx / 2, F.ny / 2), dim3(BX, BY), 0, st>>>(F, C);
    SGPU_LAUNCH();
}
void launch_mg_prolong(const LevelView& C, const LevelView& F, double omega, cudaStream_t st) {
    k_mg_prolong<<<grid2(F.nx, F.ny), dim3(BX, BY), 0, st>>>(C, F, omega);
    SGPU_LAUNCH();
}
void launch_mg_sub_mean(const LevelView& L, double* x, const double* sum, cudaStream_t st) {
    k_mg_sub_mean<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, st>>>(L, x, sum);
    SGPU_LAUNCH();
}
void launch_mg_coarse(const LevelView& L, double* rowbuf, int* sweeps_out, cudaStream_t st) {
    k_mg_coarse<<<1, kCoarseThreads, 0, st>>>(L, rowbuf, sweeps_out);
    SGPU_LAUNCH();
}

} // namespace sgpu
