// mg.cu — geometric multigrid for p' on the device, bit-identical to the reference in FP64.
//
// The reference runs multigrid on the CPU only (src/multigrid.cpp). These kernels restate each of
// its loops with the same per-cell expression order: the Galerkin 2x2 build (mg_build, :232-261),
// the red-black two-statement smoother (smooth, :46-70), residual (:73-87), restriction (:90-103),
// prolongation with over-correction (:106-116), and the coarsest-level solve with its fixed-order
// norms (coarse_solve, :120-140), which runs inside one CTA so its data-dependent sweep count
// needs no host round trip. Every kernel is a template on the element type: double gives the
// reference's bits; float is the mixed-precision mode's V-cycle (sums and norms still in double).
// The float V-cycle also has its own tail: the small levels held in shared memory
// (k_mg_tail_smem), the coarsest solve in one warp with FP64 tree sums (warp_coarse_core).
#include "kernels.hpp"
#include "blocksum.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>

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

// A float level held in shared memory: (nx + 2) x (ny + 2) cells with the zero ring, row stride S,
// interior cell (I, J) at index (I + 1) * S + J + 1; links {e, w, n, s}, AP, b and x per cell.
struct SLevel {
    int nx, ny, S;
    float4* l4;
    float *x, *b, *ap;
    __device__ int at(int I, int J) const { return (I + 1) * S + J + 1; }
};
// Bytes of one SLevel block (links first, 16-byte aligned).
[[maybe_unused]] __host__ __device__ inline int slevel_bytes(int nx, int ny) {
    const int n2 = (nx + 2) * (ny + 2);
    return ((n2 * 28) + 15) / 16 * 16;
}
__device__ inline SLevel slevel_at(unsigned char* base, int nx, int ny) {
    const int n2 = (nx + 2) * (ny + 2);
    SLevel v;
    v.nx = nx;
    v.ny = ny;
    v.S = ny + 2;
    v.l4 = reinterpret_cast<float4*>(base);
    v.x = reinterpret_cast<float*>(base + 16 * n2);
    v.b = v.x + n2;
    v.ap = v.b + n2;
    return v;
}

// The float V-cycle's coarse_solve in one warp on a shared-memory level: the same red-black
// sweeps, stopping test (||b - A x|| < tol ||b|| or 200 sweeps) and mean removals as
// cta_coarse_solve, but no block barrier per pass, which on a level of a few cells is most of a
// pass's cost. Its sums are FP64: each lane adds its cells in order and a fixed xor-shuffle tree
// combines the lanes (not the reference's row chain, which only the FP64 V-cycle needs).
__device__ void warp_coarse_core(const SLevel& L, double tol, int* sweeps_out) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int n = L.nx * L.ny, S = L.S;
    auto at = [&](int k) {
        const int I = k / L.ny;
        return L.at(I, k - I * L.ny);
    };
    auto sum = [&](auto f) {
        double a = 0.0;
        for (int k = lane; k < n; k += 32) a += f(at(k));
        return warp_sum(a);
    };
    float *sx = L.x, *sb = L.b, *sap = L.ap;
    const float4* sl = L.l4;
    auto smooth = [&](int colour) {
        for (int k = lane; k < n; k += 32) {
            const int I = k / L.ny, J = k - I * L.ny;
            if (((I + J) & 1) != colour) continue;
            const int q = L.at(I, J);
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
        const int q = at(k);
        sx[q] = static_cast<float>(sx[q] - mx);
    }
    __syncwarp();
    if (lane == 0 && sweeps_out) *sweeps_out = sweeps;
}

// Global level L into the shared level s (links, AP; b and x when `values`; zero elsewhere,
// the ring included), by all threads of the block.
__device__ void slevel_load(const LevelViewT<float>& L, const SLevel& s, bool values) {
    const int n2 = (L.nx + 2) * s.S;
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        const int I = k / s.S - 1, J = k % s.S - 1;
        const bool in = I >= 0 && I < L.nx && J >= 0 && J < L.ny;
        const int q = I * L.stride + J;
        float4 l = make_float4(0.f, 0.f, 0.f, 0.f);
        if (in) {
            const Links<float> a = links(L, q);
            l = make_float4(a.e, a.w, a.n, a.s);
        }
        s.l4[k] = l;
        s.ap[k] = in ? L.AP[q] : 0.0f;
        s.b[k] = (in && values) ? L.b[q] : 0.0f;
        s.x[k] = (in && values) ? L.x[q] : 0.0f;
    }
}
// The interior x and b of the shared level back to L.
__device__ void slevel_store(const LevelViewT<float>& L, const SLevel& s) {
    const int n = L.nx * L.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int I = k / L.ny, J = k - I * L.ny;
        L.x[I * L.stride + J] = s.x[s.at(I, J)];
        L.b[I * L.stride + J] = s.b[s.at(I, J)];
    }
}

// The coarsest level of the float V-cycle in a global-memory tail: copied to shared memory, solved
// by one warp, copied back. Levels of up to kWarpCoarseCells cells with their ring.
constexpr int kWarpCoarseCells = 1024;

[[maybe_unused]] __device__ void warp_coarse_solve(const LevelViewT<float>& L, double tol, int* sweeps_out) {
    __shared__ __align__(16) unsigned char sm[kWarpCoarseCells * 28];
    const SLevel s = slevel_at(sm, L.nx, L.ny);
    if (threadIdx.x < 32) {
        const int S = s.S, n2 = (L.nx + 2) * S;
        for (int k = threadIdx.x; k < n2; k += 32) {
            const int I = k / S - 1, J = k % S - 1;
            const bool in = I >= 0 && I < L.nx && J >= 0 && J < L.ny;
            const int q = I * L.stride + J;
            float4 l = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in) {
                const Links<float> a = links(L, q);
                l = make_float4(a.e, a.w, a.n, a.s);
            }
            s.l4[k] = l;
            s.ap[k] = in ? L.AP[q] : 0.0f;
            s.b[k] = in ? L.b[q] : 0.0f;
            s.x[k] = in ? L.x[q] : 0.0f;
        }
        __syncwarp();
        warp_coarse_core(s, tol, sweeps_out);
        const int n = L.nx * L.ny;
        for (int k = threadIdx.x; k < n; k += 32) {
            const int I = k / L.ny, J = k - I * L.ny;
            L.x[I * L.stride + J] = s.x[s.at(I, J)];
            L.b[I * L.stride + J] = s.b[s.at(I, J)];
        }
    }
}

// ---- the float tail with every level in shared memory ----

// Byte offset of each tail level's SLevel block in dynamic shared memory, and the total.
struct TailSmem {
    int off[24];
    int bytes;
};

// One colour of smooth on a shared level: warps take rows, lanes the colour's cells of a row.
__device__ void s_smooth(const SLevel& L, int colour) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5, S = L.S;
    for (int I = w; I < L.nx; I += nw)
        for (int J = ((I + colour) & 1) + 2 * lane; J < L.ny; J += 64) {
            const int q = L.at(I, J);
            const float4 a = L.l4[q];
            L.x[q] = rb_value(L.b[q], a.x * L.x[q + 1] + a.y * L.x[q - 1] + a.w * L.x[q + S] + a.z * L.x[q - S],
                              L.ap[q]);
        }
    __syncthreads();
}
// Residual of F (multigrid.cpp:84-85 form) restricted 2x2 into C.b (multigrid.cpp:90-103), C.x = 0.
__device__ void s_residual_restrict(const SLevel& F, const SLevel& C) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5, S = F.S;
    auto r = [&](int q) {
        const float4 a = F.l4[q];
        return F.b[q] - (F.ap[q] * F.x[q] - (a.x * F.x[q + 1] + a.y * F.x[q - 1] + a.w * F.x[q + S] + a.z * F.x[q - S]));
    };
    for (int I = w; I < C.nx; I += nw)
        for (int J = lane; J < C.ny; J += 32) {
            const int f = F.at(2 * I, 2 * J), c = C.at(I, J);
            C.b[c] = r(f) + r(f + 1) + r(f + S) + r(f + S + 1);
            C.x[c] = 0.0f;
        }
    __syncthreads();
}
// prolong (multigrid.cpp:106-116): F.x += omega * C.x of the parent cell.
__device__ void s_prolong(const SLevel& C, const SLevel& F, float om) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5;
    for (int i = w; i < F.nx; i += nw)
        for (int j = lane; j < F.ny; j += 32) F.x[F.at(i, j)] += om * C.x[C.at(i >> 1, j >> 1)];
    __syncthreads();
}

// Levels [first, nl) of one float V-cycle (mg_vcycle, multigrid.cpp:299-323) in one CTA with every
// level in shared memory: the links, AP, b and x of the first tail level are read once, the passes
// run against shared memory with a block barrier between them, and x and b of every tail level are
// written back at the end. Same passes and per-cell expressions as k_mg_tail.
__global__ void __launch_bounds__(kCoarseThreads)
    k_mg_tail_smem(MgLevelsT<float> lv, int first, int pre, int post, double omega, double tol, TailSmem ts,
                   int* sweeps_out) {
    extern __shared__ __align__(16) unsigned char tail_sm[];
    const int nl = lv.n;
    auto sl = [&](int l) { return slevel_at(tail_sm + ts.off[l], lv.L[l].nx, lv.L[l].ny); };
    for (int l = first; l < nl; ++l) slevel_load(lv.L[l], sl(l), l == first);
    __syncthreads();
    for (int l = first; l + 1 < nl; ++l) {
        const SLevel L = sl(l);
        for (int s = 0; s < pre; ++s) {
            s_smooth(L, 0);
            s_smooth(L, 1);
        }
        s_residual_restrict(L, sl(l + 1));
    }
    if (threadIdx.x < 32) warp_coarse_core(sl(nl - 1), tol, sweeps_out);
    __syncthreads();
    const float om = static_cast<float>(omega);
    for (int l = nl - 2; l >= first; --l) {
        const SLevel L = sl(l);
        s_prolong(sl(l + 1), L, om);
        for (int s = 0; s < post; ++s) {
            s_smooth(L, 0);
            s_smooth(L, 1);
        }
    }
    for (int l = first; l < nl; ++l) slevel_store(lv.L[l], sl(l));
}

#ifdef SGPU_FLOAT_UNIT
// ---- the float tail on a thread-block cluster ----
//
// Levels [first, lg) of the float V-cycle are split by rows over the kClusterTail CTAs of one
// cluster, each CTA's band of a level held in its shared memory as an SLevel whose ring rows are
// ghost copies of the neighbouring bands' edge rows; levels [lg, nl) (at most kGatherCells cells
// each) and the coarsest solve run on CTA 0 as in k_mg_tail_smem. The passes and per-cell
// expressions are k_mg_tail_smem's, with a cluster barrier between passes instead of a block
// barrier. Levels halve exactly (mg_level_dims halves only even sizes), and the bands of the
// coarsest split level start at even rows, so every band of every split level starts at an even
// row: a 2 x 2 restriction block and a prolongation parent lie in the CTA's own bands, and the
// red-black colour of a cell is the parity of its local row plus column. A pass that updates a
// band's first or last row also stores the value into the ghost row of the neighbouring band
// (distributed shared memory). In a colour pass the neighbours read only the other colour's ghost
// cells, and a prolongation reads no ghost cell, so the stores race with no read, and one cluster
// barrier per pass publishes them.
constexpr int kClusterTail = 16;        // CTAs per cluster (a non-portable size)
constexpr int kGatherCells = 1024;      // levels of at most this many cells run on CTA 0
constexpr int kClusterTailCells = 65536; // the cluster tail takes levels of at most this many cells

struct ClusterTailPlan {
    int first, lg, nl;             // split levels [first, lg), gathered levels [lg, nl)
    int band[kClusterTail + 1];    // band starts of level lg - 1 for ranks 0 .. R (band[R] = its nx)
    int off[24];                   // byte offset of each level's block in every CTA's shared memory
    int rows[24];                  // rows allocated per split level (its largest band)
    int bytes;                     // dynamic shared memory per CTA
};

namespace cg = cooperative_groups;

// One colour of smooth on a band; xup / xdn: the x arrays of the bands above / below (null at the
// cluster's ends), mup: the rows of the band above (its bottom ghost row mirrors our row 0).
__device__ void c_smooth(const SLevel& L, float* xup, int mup, float* xdn, int colour) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5, S = L.S;
    for (int I = w; I < L.nx; I += nw)
        for (int J = ((I + colour) & 1) + 2 * lane; J < L.ny; J += 64) {
            const int q = L.at(I, J);
            const float4 a = L.l4[q];
            const float v = rb_value(L.b[q], a.x * L.x[q + 1] + a.y * L.x[q - 1] + a.w * L.x[q + S] +
                                                 a.z * L.x[q - S],
                                     L.ap[q]);
            L.x[q] = v;
            if (I == 0 && xup) xup[(mup + 1) * S + J + 1] = v;
            if (I == L.nx - 1 && xdn) xdn[J + 1] = v;
        }
    cg::this_cluster().sync();
}
// The residual of the band F restricted 2 x 2 into rows c0 + I of the coarse level C (a band of
// this CTA, c0 = 0, or the gathered level on CTA 0), C.x = 0 there.
__device__ void c_restrict(const SLevel& F, const SLevel& C, int c0) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5, S = F.S;
    auto r = [&](int q) {
        const float4 a = F.l4[q];
        return F.b[q] - (F.ap[q] * F.x[q] - (a.x * F.x[q + 1] + a.y * F.x[q - 1] + a.w * F.x[q + S] + a.z * F.x[q - S]));
    };
    for (int I = w; I < F.nx / 2; I += nw)
        for (int J = lane; J < C.ny; J += 32) {
            const int f = F.at(2 * I, 2 * J), cq = C.at(c0 + I, J);
            C.b[cq] = r(f) + r(f + 1) + r(f + S) + r(f + S + 1);
            C.x[cq] = 0.0f;
        }
    cg::this_cluster().sync();
}
// prolong into the band F from rows c0 + I / 2 of the coarse level C (this CTA's band, c0 = 0, or
// the gathered level on CTA 0), with the ghost stores of c_smooth.
__device__ void c_prolong(const SLevel& C, int c0, const SLevel& F, float* xup, int mup, float* xdn, float om) {
    const int w = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int nw = static_cast<int>(blockDim.x) >> 5, S = F.S;
    for (int I = w; I < F.nx; I += nw)
        for (int J = lane; J < F.ny; J += 32) {
            const int q = F.at(I, J);
            const float v = F.x[q] + om * C.x[C.at(c0 + (I >> 1), J >> 1)];
            F.x[q] = v;
            if (I == 0 && xup) xup[(mup + 1) * S + J + 1] = v;
            if (I == F.nx - 1 && xdn) xdn[J + 1] = v;
        }
    cg::this_cluster().sync();
}

__global__ void __launch_bounds__(kCoarseThreads)
    k_mg_tail_cluster(MgLevelsT<float> lv, ClusterTailPlan pl, int pre, int post, double omega, double tol,
                      int* sweeps_out) {
    extern __shared__ __align__(16) unsigned char tail_sm[];
    cg::cluster_group cl = cg::this_cluster();
    const int R = static_cast<int>(cl.num_blocks()), rank = static_cast<int>(cl.block_rank());
    const int first = pl.first, lg = pl.lg, nl = pl.nl, Lc = lg - 1;
    auto start = [&](int l, int rr) { return pl.band[rr] << (Lc - l); }; // band start of rank rr
    // this CTA's band of split level l (laid out for the level's largest band: the same offsets in
    // every CTA, so a neighbour's arrays are this CTA's mapped to its rank)
    auto band = [&](int l) {
        SLevel s = slevel_at(tail_sm + pl.off[l], pl.rows[l], lv.L[l].ny);
        s.nx = start(l, rank + 1) - start(l, rank);
        return s;
    };
    auto xup = [&](const SLevel& s) { return rank > 0 ? cl.map_shared_rank(s.x, rank - 1) : nullptr; };
    auto xdn = [&](const SLevel& s) { return rank < R - 1 ? cl.map_shared_rank(s.x, rank + 1) : nullptr; };
    auto mup = [&](int l) { return rank > 0 ? start(l, rank) - start(l, rank - 1) : 0; };
    auto gathered = [&](int l) { return slevel_at(tail_sm + pl.off[l], lv.L[l].nx, lv.L[l].ny); };
    auto gathered0 = [&](int l) { // the gathered level l in CTA 0's shared memory
        SLevel s = gathered(l);
        s.l4 = cl.map_shared_rank(s.l4, 0);
        s.x = cl.map_shared_rank(s.x, 0);
        s.b = cl.map_shared_rank(s.b, 0);
        s.ap = cl.map_shared_rank(s.ap, 0);
        return s;
    };
    cl.sync(); // every CTA of the cluster runs before any touches another's shared memory
    for (int l = first; l < lg; ++l) { // the bands, with their ghost rows of x
        const LevelViewT<float>& L = lv.L[l];
        const SLevel s = band(l);
        const int g0 = start(l, rank), n2 = (s.nx + 2) * s.S;
        for (int k = threadIdx.x; k < n2; k += blockDim.x) {
            const int I = k / s.S - 1, J = k % s.S - 1, g = g0 + I;
            const bool cin = J >= 0 && J < L.ny, own = cin && I >= 0 && I < s.nx;
            const int q = g * L.stride + J;
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
            if (own) {
                const Links<float> k4 = links(L, q);
                a = make_float4(k4.e, k4.w, k4.n, k4.s);
            }
            s.l4[k] = a;
            s.ap[k] = own ? L.AP[q] : 0.0f;
            s.b[k] = (own && l == first) ? L.b[q] : 0.0f;
            s.x[k] = (l == first && cin && g >= 0 && g < L.nx) ? L.x[q] : 0.0f;
        }
    }
    if (rank == 0)
        for (int l = lg; l < nl; ++l) slevel_load(lv.L[l], gathered(l), false);
    cl.sync();
    const float om = static_cast<float>(omega);
    for (int l = first; l < lg; ++l) {
        const SLevel s = band(l);
        for (int k = 0; k < pre; ++k) {
            c_smooth(s, xup(s), mup(l), xdn(s), 0);
            c_smooth(s, xup(s), mup(l), xdn(s), 1);
        }
        if (l + 1 < lg) c_restrict(s, band(l + 1), 0);
        else c_restrict(s, gathered0(lg), start(l, rank) / 2);
    }
    if (rank == 0) { // the gathered levels and the coarsest solve, as k_mg_tail_smem
        for (int l = lg; l + 1 < nl; ++l) {
            const SLevel L = gathered(l);
            for (int k = 0; k < pre; ++k) {
                s_smooth(L, 0);
                s_smooth(L, 1);
            }
            s_residual_restrict(L, gathered(l + 1));
        }
        if (threadIdx.x < 32) warp_coarse_core(gathered(nl - 1), tol, sweeps_out);
        __syncthreads();
        for (int l = nl - 2; l >= lg; --l) {
            const SLevel L = gathered(l);
            s_prolong(gathered(l + 1), L, om);
            for (int k = 0; k < post; ++k) {
                s_smooth(L, 0);
                s_smooth(L, 1);
            }
        }
    }
    cl.sync();
    for (int l = lg - 1; l >= first; --l) {
        const SLevel s = band(l);
        if (l + 1 < lg) c_prolong(band(l + 1), 0, s, xup(s), mup(l), xdn(s), om);
        else c_prolong(gathered0(lg), start(l, rank) / 2, s, xup(s), mup(l), xdn(s), om);
        for (int k = 0; k < post; ++k) {
            c_smooth(s, xup(s), mup(l), xdn(s), 0);
            c_smooth(s, xup(s), mup(l), xdn(s), 1);
        }
    }
    for (int l = first; l < lg; ++l) { // the bands' x and b back
        const LevelViewT<float>& L = lv.L[l];
        const SLevel s = band(l);
        const int g0 = start(l, rank), n = s.nx * L.ny;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int I = k / L.ny, J = k - I * L.ny;
            L.x[(g0 + I) * L.stride + J] = s.x[s.at(I, J)];
            L.b[(g0 + I) * L.stride + J] = s.b[s.at(I, J)];
        }
    }
    if (rank == 0)
        for (int l = lg; l < nl; ++l) slevel_store(lv.L[l], gathered(l));
}
#endif

// coarse_solve (multigrid.cpp:120-140) of an FP64 level in one warp on a shared-memory copy, bit for
// bit the passes of cta_coarse_solve: the same per-cell expressions, and det_sum's order (each row
// added left to right by one lane, then the row sums in order by lane 0, multigrid.cpp:18-34), so
// the sweep count and every value equal the reference's; but no block barrier per pass, which on a
// coarsest level of a few cells is most of a pass's cost. sm: coarse64_bytes(nx, ny) bytes.
__host__ __device__ inline int coarse64_bytes(int nx, int ny) { return (8 * (nx + 2) * (ny + 2) + nx) * 8; }

__device__ void warp_coarse_solve64(const LevelViewT<double>& L, double tol, int* sweeps_out, double* sm) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int nx = L.nx, ny = L.ny, S = ny + 2, n2 = (nx + 2) * S, n = nx * ny;
    double *le = sm, *lw = le + n2, *ln = lw + n2, *ls = ln + n2, *ap = ls + n2, *b = ap + n2, *x = b + n2,
           *r = x + n2, *rows = r + n2;
    for (int k = lane; k < n2; k += 32) { // the level with its zero ring
        const int I = k / S - 1, J = k % S - 1;
        const bool in = I >= 0 && I < nx && J >= 0 && J < ny;
        const int q = I * L.stride + J;
        le[k] = in ? L.AE[q] : 0.0;
        lw[k] = in ? L.AW[q] : 0.0;
        ln[k] = in ? L.AN[q] : 0.0;
        ls[k] = in ? L.AS[q] : 0.0;
        ap[k] = in ? L.AP[q] : 0.0;
        b[k] = in ? L.b[q] : 0.0;
        x[k] = in ? L.x[q] : 0.0;
        r[k] = 0.0;
    }
    __syncwarp();
    auto at = [&](int I, int J) { return (I + 1) * S + J + 1; };
    auto det_sum = [&](auto f) {
        for (int I = lane; I < nx; I += 32) {
            double a = 0.0;
            for (int J = 0; J < ny; ++J) a += f(at(I, J));
            rows[I] = a;
        }
        __syncwarp();
        double t = 0.0;
        if (lane == 0)
            for (int I = 0; I < nx; ++I) t += rows[I];
        t = __shfl_sync(0xffffffffu, t, 0);
        __syncwarp();
        return t;
    };
    auto remove_mean = [&](double* f) {
        const double m = det_sum([&](int q) { return f[q]; }) / (static_cast<double>(nx) * ny);
        for (int k = lane; k < n; k += 32) {
            const int q = at(k / ny, k % ny);
            f[q] = f[q] - m;
        }
        __syncwarp();
    };
    auto smooth = [&](int colour) {
        for (int k = lane; k < n; k += 32) {
            const int I = k / ny, J = k % ny;
            if (((I + J) & 1) != colour) continue;
            const int q = at(I, J);
            x[q] = rb_value(b[q], le[q] * x[q + 1] + lw[q] * x[q - 1] + ls[q] * x[q + S] + ln[q] * x[q - S], ap[q]);
        }
        __syncwarp();
    };
    remove_mean(b);
    const double bb = det_sum([&](int q) {
        const double v = b[q];
        return v * v;
    });
    int sweeps = 0;
    if (bb > 0.0) {
        const double bn = sqrt(bb);
        while (sweeps < 200) {
            smooth(0);
            smooth(1);
            ++sweeps;
            const double rr = det_sum([&](int q) { // the residual (cta_residual's expression), squared
                const double v = b[q] - (ap[q] * x[q] - (le[q] * x[q + 1] + lw[q] * x[q - 1] + ls[q] * x[q + S] +
                                                         ln[q] * x[q - S]));
                r[q] = v;
                return v * v;
            });
            if (sqrt(rr) < tol * bn) break;
        }
    }
    remove_mean(x);
    for (int k = lane; k < n; k += 32) {
        const int I = k / ny, J = k % ny, q = I * L.stride + J, c = at(I, J);
        L.x[q] = x[c];
        L.b[q] = b[c];
        L.r[q] = r[c];
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
              double* rowbuf, int* sweeps_out, int warp64) {
    extern __shared__ __align__(16) unsigned char tail_dyn[];
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
    } else if (warp64) {
        __threadfence_block(); // the other warps' restriction writes, made visible to warp 0
        __syncthreads();
        if constexpr (sizeof(T) == 8)
            if (threadIdx.x < 32)
                warp_coarse_solve64(lv.L[nl - 1], tol, sweeps_out, reinterpret_cast<double*>(tail_dyn));
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

// The float tail runs with every level in shared memory when they fit (the 64^2-and-below levels
// of a square grid take about 170 KB); otherwise, and for double, through global memory.
constexpr int kTailSmemMax = 200 * 1024;
// Shared memory for the FP64 warp coarse solve (about 1400 cells with their ring).
constexpr int kCoarse64Max = 96 * 1024;

template <class T>
void launch_mg_tail(const MgLevelsT<T>& lv, int first, int pre, int post, double omega, double tol,
                    double* rowbuf, int* sweeps_out, cudaStream_t st) {
    if constexpr (sizeof(T) == 4) {
        TailSmem ts{};
        int bytes = 0;
        for (int l = first; l < lv.n && l < 24; ++l) {
            ts.off[l] = bytes;
            bytes += slevel_bytes(lv.L[l].nx, lv.L[l].ny);
        }
        ts.bytes = bytes;
        const int nc = lv.L[lv.n - 1].nx * lv.L[lv.n - 1].ny;
        if (lv.n <= 24 && bytes <= kTailSmemMax && nc <= kWarpCoarseCells) {
            static PerDeviceOnce attr; // the attribute lives in each device's context
            attr.get([] {
                SGPU_CUDA(cudaFuncSetAttribute(k_mg_tail_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               kTailSmemMax));
                return 0;
            });
            k_mg_tail_smem<<<1, kCoarseThreads, bytes, st>>>(lv, first, pre, post, omega, tol, ts, sweeps_out);
            SGPU_LAUNCH();
            return;
        }
    }
    // FP64: the coarsest solve in one warp on a shared-memory copy when the level fits
    int dyn = 0;
    if constexpr (sizeof(T) == 8) {
        const int b = coarse64_bytes(lv.L[lv.n - 1].nx, lv.L[lv.n - 1].ny);
        if (b <= kCoarse64Max) dyn = b;
        static PerDeviceOnce attr;
        attr.get([] {
            SGPU_CUDA(cudaFuncSetAttribute(k_mg_tail<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kCoarse64Max));
            return 0;
        });
    }
    k_mg_tail<T><<<1, kCoarseThreads, dyn, st>>>(lv, first, pre, post, omega, tol, rowbuf, sweeps_out, dyn > 0 ? 1 : 0);
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

#ifdef SGPU_FLOAT_UNIT
namespace {
// Dynamic shared memory per CTA of the cluster tail (the 227 KB a CTA may have).
constexpr int kClusterSmemMax = 227 * 1024;

// The cluster tail's plan from level `first`; false where it does not apply: fewer than one split
// level, a split level that does not halve exactly into the next, a coarsest split level of fewer
// than 2 rows per CTA, or more shared memory per CTA than kClusterSmemMax.
bool cluster_tail_plan(const MgLevelsT<float>& lv, int first, ClusterTailPlan& pl) {
    const int nl = lv.n;
    if (nl > 24 || first < 0 || first >= nl - 1) return false;
    int lg = first;
    while (lg < nl - 1 && lv.L[lg].nx * lv.L[lg].ny > kGatherCells) ++lg;
    if (lg == first || lv.L[lg].nx * lv.L[lg].ny > kGatherCells) return false;
    for (int l = first; l < lg; ++l)
        if (lv.L[l].nx != 2 * lv.L[l + 1].nx || lv.L[l].ny != 2 * lv.L[l + 1].ny) return false;
    const int Lc = lg - 1, nxc = lv.L[Lc].nx;
    if (nxc < 2 * kClusterTail) return false;
    pl.first = first;
    pl.lg = lg;
    pl.nl = nl;
    for (int r = 0; r < kClusterTail; ++r) pl.band[r] = 2 * ((r * (nxc / 2)) / kClusterTail);
    pl.band[kClusterTail] = nxc;
    int bytes = 0;
    for (int l = first; l < lg; ++l) {
        int rows = 0;
        for (int r = 0; r < kClusterTail; ++r) rows = std::max(rows, (pl.band[r + 1] - pl.band[r]) << (Lc - l));
        pl.rows[l] = rows;
        pl.off[l] = bytes;
        bytes += slevel_bytes(rows, lv.L[l].ny);
    }
    for (int l = lg; l < nl; ++l) {
        pl.off[l] = bytes;
        bytes += slevel_bytes(lv.L[l].nx, lv.L[l].ny);
    }
    pl.bytes = bytes;
    return bytes <= kClusterSmemMax;
}

// Whether this device runs the cluster tail: its function attributes set (the dynamic shared memory
// and the non-portable cluster size, once per device) and at least one such cluster resident.
// SGPU_MG_CLUSTER=0 turns it off for the solvers created while it is set (their float tail then
// runs as streamed levels and the single-CTA tail, as without a cluster).
bool cluster_tail_available() {
    if (const char* e = std::getenv("SGPU_MG_CLUSTER"))
        if (std::atoi(e) == 0) return false;
    static PerDeviceOnce once;
    return once.get([] {
        // a device that refuses either attribute runs the kernels without a cluster
        if (cudaFuncSetAttribute(k_mg_tail_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_mg_tail_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            (void)cudaGetLastError();
            return 0;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterTail);
        cfg.blockDim = dim3(kCoarseThreads);
        cfg.dynamicSmemBytes = kClusterSmemMax;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kClusterTail;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_mg_tail_cluster, &cfg) != cudaSuccess) {
            (void)cudaGetLastError(); // not supported here: the clear-up of the failed query
            return 0;
        }
        return n > 0 ? 1 : 0;
    }) != 0;
}
} // namespace

int mg_cluster_tail_first(const MgLevelsT<float>& lv, int fallback) {
    if (!cluster_tail_available()) return fallback;
    int t = 0;
    while (t < lv.n - 1 && lv.L[t].nx * lv.L[t].ny > kClusterTailCells) ++t;
    ClusterTailPlan pl{};
    for (; t < fallback; ++t)
        if (cluster_tail_plan(lv, t, pl)) return t;
    return fallback;
}

bool launch_mg_tail_cluster(const MgLevelsT<float>& lv, int first, int pre, int post, double omega, double tol,
                            int* sweeps_out, cudaStream_t st) {
    ClusterTailPlan pl{};
    if (!cluster_tail_plan(lv, first, pl)) return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterTail);
    cfg.blockDim = dim3(kCoarseThreads);
    cfg.dynamicSmemBytes = static_cast<std::size_t>(pl.bytes);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kClusterTail;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    SGPU_CUDA(cudaLaunchKernelEx(&cfg, k_mg_tail_cluster, lv, pl, pre, post, omega, tol, sweeps_out));
    SGPU_LAUNCH();
    return true;
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
