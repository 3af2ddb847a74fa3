// mg_fast.cu — the multigrid V-cycle of multigrid.cpp with fused, streaming level kernels
// (bit-identical to the reference in FP64; the float instantiation is the mixed-precision mode's).
//
// Per fine level two passes over memory instead of one per colour:
//  * k_mg_down: `pre` red-black sweeps (smooth, multigrid.cpp:46-70), the residual (:73-87) and the
//    2x2 restriction (:90-103) in one streaming pass; with `build`, also the coarse level's Galerkin
//    links and AP (mg_build, :232-261) from the fine links the residual has just loaded, with
//    mg_build's additions in its order (the same bits as k_mg_build). A CTA owns a strip of columns plus a halo and
//    walks it top to bottom; in sweep s the cell (I, J) of colour c = (I + J) & 1 is updated at step
//    t = I + 4s + 2c, so each cell sees its neighbours in exactly the reference's colour order; the
//    residual of row I is formed at step I + 4 pre, when its neighbours are final, and pairs of
//    residual rows are summed 2x2 (lanes exchange the odd column by shuffle) into the coarse
//    right-hand side. The residual array itself is never stored.
//  * k_mg_up: prolongation with over-correction (:106-116) applied to each row as it arrives,
//    followed by `post` red-black sweeps, in the same streaming order.
// The smoothed iterate goes to a second buffer (CTAs read their neighbours' rows as halo). Levels
// below a size threshold and the coarsest solve run in one CTA (k_mg_tail in mg.cu).
#include "kernels.hpp"

#include <algorithm>
#include <cstdlib>

namespace sgpu {

namespace {

constexpr int kRing = 32;
constexpr int kPD = 8; // prefetch distance in rows

template <class T> __device__ __forceinline__ void cp_async(T* smem, const T* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Window geometry shared by both kernels. Level indices: interior 0 <= I < nx, 0 <= J < ny; the
// arrays hold a zero ring at I = -1, nx and J = -1, ny.
struct Win {
    int R0, R1;      // owned rows
    int L0, L1;      // loaded rows [L0, L1)
    int J0, C0;      // first owned column; first loaded column (even)
    int W;           // owned columns per CTA
    bool cut_top, cut_bot, cut_left, cut_right;
};

template <int NT>
__device__ __forceinline__ Win make_win(int nx, int ny, int seg_rows, int HC) {
    Win w;
    w.W = NT - 2 * HC;
    w.R0 = blockIdx.y * seg_rows;
    w.R1 = min(w.R0 + seg_rows, nx);
    w.L0 = max(w.R0 - HC, -1);
    w.L1 = min(w.R1 + HC, nx + 1);
    w.J0 = blockIdx.x * w.W;
    w.C0 = w.J0 - HC;
    w.cut_top = w.L0 > -1;
    w.cut_bot = w.L1 < nx + 1;
    w.cut_left = w.C0 > -1;
    w.cut_right = w.C0 + NT < ny + 1;
    return w;
}

// Is pass k's update (or, with k = 2 * sweeps, the residual) of an interior cell (I, Jc) computable
// from the window: (!cut_top || I >= L0 + 1 + k) && (!cut_bot || I <= L1 - 2 - k) && (!cut_left ||
// Jc >= C0 + 1 + k) && (!cut_right || Jc <= C0 + NT - 2 - k). A thread's column is fixed, so its
// column tests (and whether the column is interior) become one bit per k, and the row tests with
// 0 <= I < nx two bounds linear in k: lo + k dt <= I <= hi - k db.
struct Cone {
    int lo, hi, dt, db;
    unsigned cols;
    __device__ __forceinline__ bool ok(int I, int k) const {
        return ((cols >> k) & 1u) && I >= lo + k * dt && I <= hi - k * db;
    }
};
__device__ __forceinline__ Cone make_cone(const Win& w, int Jc, bool cint, int nx, int NT, int kmax) {
    Cone c;
    c.dt = w.cut_top ? 1 : 0;
    c.db = w.cut_bot ? 1 : 0;
    c.lo = w.cut_top ? w.L0 + 1 : 0; // L0 >= 0 when cut, so the bound is inside [0, nx)
    c.hi = w.cut_bot ? w.L1 - 2 : nx - 1;
    c.cols = 0u;
    for (int k = 0; k <= kmax; ++k) {
        const bool ok = cint && (!w.cut_left || Jc >= w.C0 + 1 + k) && (!w.cut_right || Jc <= w.C0 + NT - 2 - k);
        c.cols |= (ok ? 1u : 0u) << k;
    }
    return c;
}

// The 6 per-cell inputs of a red-black update or a residual: AE, AW, AN, AS, AP, b.
template <class T> __device__ __forceinline__ void load6(const LevelViewT<T>& L, int q, T a[6]) {
    const Links<T> k = links(L, q);
    a[0] = k.e;
    a[1] = k.w;
    a[2] = k.n;
    a[3] = k.s;
    a[4] = __ldg(L.AP + q);
    a[5] = __ldg(L.b + q);
}

// Red-black two-statement update of one cell (multigrid.cpp:61-63) on the ring.
template <int NT, class T>
__device__ __forceinline__ void rb_update(T (*ring)[NT], int I, int tid, const T a[6]) {
    T* row = ring[I & (kRing - 1)];
    row[tid] = rb_value(a[5],
                        a[0] * row[tid + 1] + a[1] * row[tid - 1] + a[3] * ring[(I + 1) & (kRing - 1)][tid] +
                            a[2] * ring[(I - 1) & (kRing - 1)][tid],
                        a[4]);
}

// The coefficient loads of a step are issued PD steps before the step runs, into one of PD
// register sets used in rotation (the step loop is unrolled by PD so every set index is a
// compile-time constant): a step then waits on loads issued PD steps earlier, not on a memory round
// trip of its own.
template <int NC, class T> struct StepRegs {
    int I[NC];
    bool ok[NC];
    T a[NC][6];
};

// PRE red-black sweeps, residual and restriction in one streaming pass (see the file comment).
template <int NT, int PRE, int PD, int MINB, class T>
__global__ void __launch_bounds__(NT, MINB)
    k_mg_down(LevelViewT<T> L, LevelViewT<T> C, T* __restrict__ xout, int x_zero, int seg_rows,
              int HC, int build) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*ring)[NT] = reinterpret_cast<T(*)[NT]>(smem_raw);
    const Win w = make_win<NT>(L.nx, L.ny, seg_rows, HC);
    const int tid = threadIdx.x;
    const int Jc = w.C0 + tid;
    const bool cload = Jc >= -1 && Jc <= L.ny;
    const bool cint = Jc >= 0 && Jc < L.ny;
    const bool cown = cint && Jc >= w.J0 && Jc < w.J0 + w.W;
    const int s = L.stride;
    const Cone cone = make_cone(w, Jc, cint, L.nx, NT, 2 * PRE);

    int next = w.L0;
    auto issue = [&]() {
        if (next < w.L1 && cload) {
            T* dst = &ring[next & (kRing - 1)][tid];
            if (x_zero) *dst = T(0);
            else cp_async(dst, L.x + next * s + Jc);
        }
        cp_async_commit();
        ++next;
    };
    // Cells of step t: PRE updates (rows t - 2c - 4 sw) and the residual (row t - 4 PRE), with
    // their six inputs loaded.
    constexpr int NC = PRE + 1;
    auto prepare = [&](int t, StepRegs<NC, T>& r) {
        const int cpar = (t + Jc + 4) & 1;
#pragma unroll
        for (int sw = 0; sw < PRE; ++sw) {
            r.I[sw] = t - 2 * cpar - 4 * sw;
            r.ok[sw] = cone.ok(r.I[sw], 2 * sw + cpar);
        }
        r.I[PRE] = t - 4 * PRE;
        r.ok[PRE] = cone.ok(r.I[PRE], 2 * PRE);
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (r.ok[c]) load6(L, r.I[c] * s + Jc, r.a[c]);
    };
    for (int k = 0; k < kPD + 2; ++k) issue(); // rows L0 .. L0 + 1 + kPD

    StepRegs<NC, T> S[PD];
#pragma unroll
    for (int d = 0; d < PD; ++d) prepare(w.L0 + d, S[d]);

    const int t_last = w.R1 - 1 + 4 * PRE;
    T r_prev = T(0);
    T lp[4] = {T(0), T(0), T(0), T(0)}; // links e, w, n, s of the previous residual row's cell
    auto step = [&](int t, StepRegs<NC, T>& R) {
        cp_async_wait<kPD>(); // rows <= t + 1 have landed
        __syncthreads();
        issue();
#pragma unroll
        for (int sw = 0; sw < PRE; ++sw)
            if (R.ok[sw]) rb_update<NT>(ring, R.I[sw], tid, R.a[sw]);
        // Residual of row Ir = t - 4 PRE (multigrid.cpp:84-85): its neighbours are final.
        const int Ir = R.I[PRE];
        T r = T(0);
        if (R.ok[PRE]) {
            const T* row = ring[Ir & (kRing - 1)];
            const T* aa = R.a[PRE];
            r = aa[5] - (aa[4] * row[tid] -
                         (aa[0] * row[tid + 1] + aa[1] * row[tid - 1] +
                          aa[3] * ring[(Ir + 1) & (kRing - 1)][tid] +
                          aa[2] * ring[(Ir - 1) & (kRing - 1)][tid]));
        }
        // Restriction of the row pair (Ir - 1, Ir): C.b = r[f] + r[f+1] + r[f+fs] + r[f+fs+1].
        // With build, the coarse cell's links from the fine cells f (row Ir - 1, this column), f + 1
        // (the odd column, from lane + 1), f + fs and f + fs + 1 (row Ir), as mg_build adds them.
        const T* la = R.a[PRE];
        if ((Ir & 1) && Ir >= 1) { // uniform over the CTA
            const T rp_odd = __shfl_down_sync(0xffffffffu, r_prev, 1);
            const T r_odd = __shfl_down_sync(0xffffffffu, r, 1);
            T ep_odd = T(0), e_odd = T(0), np_odd = T(0), s_odd = T(0);
            if (build) { // uniform
                ep_odd = __shfl_down_sync(0xffffffffu, lp[0], 1);
                e_odd = __shfl_down_sync(0xffffffffu, la[0], 1);
                np_odd = __shfl_down_sync(0xffffffffu, lp[2], 1);
                s_odd = __shfl_down_sync(0xffffffffu, la[3], 1);
            }
            const int Rc = Ir >> 1;
            if (cown && !(Jc & 1) && Ir - 1 >= w.R0 && Ir < w.R1 && Rc < C.nx) {
                const int cq = Rc * C.stride + (Jc >> 1);
                C.b[cq] = r_prev + rp_odd + r + r_odd;
                C.x[cq] = T(0);
                if (build) {
                    const T ae = ep_odd + e_odd;    // k01.e + k11.e
                    const T aw = lp[1] + la[1];     // k00.w + k10.w
                    const T an = lp[2] + np_odd;    // k00.n + k01.n
                    const T as = la[3] + s_odd;     // k10.s + k11.s
                    set_links(C, cq, ae, aw, an, as);
                    C.AP[cq] = ae + aw + an + as;
                }
            }
        }
        r_prev = r;
#pragma unroll
        for (int k = 0; k < 4; ++k) lp[k] = la[k];
        // The smoothed iterate: row t - 4 PRE + 1 had its last update at step t - 1.
        const int rw = t - 4 * PRE + 1;
        if (cown && rw >= w.R0 && rw < w.R1) xout[rw * s + Jc] = ring[rw & (kRing - 1)][tid];
        prepare(t + PD, R); // this set's next use is PD steps on
    };
    for (int t = w.L0; t <= t_last; t += PD) {
#pragma unroll
        for (int d = 0; d < PD; ++d)
            if (t + d <= t_last) step(t + d, S[d]);
    }
    cp_async_wait<0>();
}

// Prolongation and POST red-black sweeps in one streaming pass (see the file comment).
template <int NT, int POST, int PD, int MINB, class T>
__global__ void __launch_bounds__(NT, MINB)
    k_mg_up(LevelViewT<T> C, LevelViewT<T> L, const T* __restrict__ xin, T* __restrict__ xout,
            double omega, int seg_rows, int HC) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*ring)[NT] = reinterpret_cast<T(*)[NT]>(smem_raw);
    const Win w = make_win<NT>(L.nx, L.ny, seg_rows, HC);
    const int tid = threadIdx.x;
    const int Jc = w.C0 + tid;
    const bool cload = Jc >= -1 && Jc <= L.ny;
    const bool cint = Jc >= 0 && Jc < L.ny;
    const bool cown = cint && Jc >= w.J0 && Jc < w.J0 + w.W;
    const int s = L.stride;
    const T om = static_cast<T>(omega);
    const Cone cone = make_cone(w, Jc, cint, L.nx, NT, 2 * POST);

    int next = w.L0;
    auto issue = [&]() {
        if (next < w.L1 && cload) cp_async(&ring[next & (kRing - 1)][tid], xin + next * s + Jc);
        cp_async_commit();
        ++next;
    };
    constexpr int NC = POST > 0 ? POST : 1;
    auto prepare = [&](int t, StepRegs<NC, T>& r) {
        const int cpar = (t + Jc + 4) & 1;
#pragma unroll
        for (int sw = 0; sw < POST; ++sw) {
            r.I[sw] = t - 2 * cpar - 4 * sw;
            r.ok[sw] = cone.ok(r.I[sw], 2 * sw + cpar);
            if (r.ok[sw]) load6(L, r.I[sw] * s + Jc, r.a[sw]);
        }
    };
    auto coarse_at = [&](int Ip) {
        return (cint && Ip >= 0 && Ip < L.nx && Ip < w.L1)
                   ? __ldg(C.x + (Ip >> 1) * C.stride + (Jc >> 1))
                   : T(0);
    };
    for (int k = 0; k < kPD + 3; ++k) issue(); // rows L0 .. L0 + 2 + kPD

    const int t0 = w.L0 - 2;
    StepRegs<NC, T> S[PD];
    T cxs[PD]; // coarse correction of row t + 2 for each set's step
#pragma unroll
    for (int d = 0; d < PD; ++d) {
        prepare(t0 + d, S[d]);
        cxs[d] = coarse_at(t0 + d + 2);
    }

    const int t_last = w.R1 - 1 + 4 * POST;
    auto step = [&](int t, StepRegs<NC, T>& R, T& cx) {
        if (t >= w.L0) cp_async_wait<kPD>(); // rows <= t + 2 have landed
        else cp_async_wait<kPD + 1>();
        __syncthreads();
        if (t >= w.L0) issue();
        // Prolongation of row t + 2 (read first at step t + 1): x += omega * coarse x.
        const int Ip = t + 2;
        if (cint && Ip >= 0 && Ip < L.nx && Ip < w.L1) {
            T* cell = &ring[Ip & (kRing - 1)][tid];
            *cell += om * cx;
        }
#pragma unroll
        for (int sw = 0; sw < POST; ++sw)
            if (R.ok[sw]) rb_update<NT>(ring, R.I[sw], tid, R.a[sw]);
        const int rw = t - 4 * POST + 1;
        if (cown && rw >= w.R0 && rw < w.R1) xout[rw * s + Jc] = ring[rw & (kRing - 1)][tid];
        prepare(t + PD, R);
        cx = coarse_at(t + PD + 2);
    };
    for (int t = t0; t <= t_last; t += PD) {
#pragma unroll
        for (int d = 0; d < PD; ++d)
            if (t + d <= t_last) step(t + d, S[d], cxs[d]);
    }
    cp_async_wait<0>();
}

constexpr int kNT = 256;

// Rows per CTA segment: one wave of the kernel's resident CTAs (blocks_per_sm per SM), at least
// min_seg rows (min_seg <= 0: 2 HC + 8, which bounds the halo and skew rows a CTA walks besides its
// own to about half of them). A lone small level is bound by the per-step latency of each CTA's
// walk, so a single solve takes short segments and more CTAs; a batch of cavities fills the GPU
// and keeps the bound.
int seg_for(int nx, int ny, int HC, int sms, int blocks_per_sm, int min_seg) {
    const int W = kNT - 2 * HC;
    const int strips = (ny + W - 1) / W;
    const int want = (blocks_per_sm * sms) / strips > 0 ? (blocks_per_sm * sms) / strips : 1;
    int seg = (nx + want - 1) / want;
    seg = (seg + 1) & ~1; // even: restriction pairs stay inside one CTA
    const int lo = min_seg > 0 ? std::max(2, min_seg & ~1) : 2 * HC + 8;
    if (seg < lo) seg = lo;
    return seg;
}

// Sets the kernel's shared-memory attribute on the current device (once per device) and returns its
// resident CTAs per SM there.
template <class K> int prepare_kernel(K kernel, int smem, PerDeviceOnce& once) {
    return once.get([&] {
        SGPU_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int blocks = 0;
        SGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kNT, smem));
        return blocks < 1 ? 1 : blocks;
    });
}

// Register budget of the level kernels: PD register sets in the coefficient pipeline against
// MINB resident CTAs per SM. The kernels are latency-bound, so resident warps count for more than
// prefetch depth. Measured at 4096^2: float (1, 4) beats (2, 3) and (3, 2). SGPU_MG_VARIANT and
// SGPU_MG_VARIANT64 select other budgets for the float and double kernels (tuning switches: the
// arithmetic is the same).
int env_variant(const char* name, int dflt) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : dflt;
}
int mg_variant() {
    static const int v = env_variant("SGPU_MG_VARIANT", 2);
    return v;
}
int mg_variant64() {
    static const int v = env_variant("SGPU_MG_VARIANT64", 0);
    return v;
}

template <int PRE, int PD, int MINB, class T>
void down_v(const LevelViewT<T>& F, const LevelViewT<T>& C, T* xout, bool x_zero, bool build, int sms,
            int min_seg, cudaStream_t st) {
    const int HC = 2 * PRE + 2;
    constexpr int smem = kRing * kNT * static_cast<int>(sizeof(T));
    static PerDeviceOnce once;
    auto kernel = k_mg_down<kNT, PRE, PD, MINB, T>;
    const int seg = seg_for(F.nx, F.ny, HC, sms, prepare_kernel(kernel, smem, once), min_seg);
    const int W = kNT - 2 * HC;
    const dim3 grid((F.ny + W - 1) / W, (F.nx + seg - 1) / seg);
    kernel<<<grid, kNT, smem, st>>>(F, C, xout, x_zero ? 1 : 0, seg, HC, build ? 1 : 0);
    SGPU_LAUNCH();
}

template <int POST, int PD, int MINB, class T>
void up_v(const LevelViewT<T>& C, const LevelViewT<T>& F, const T* xin, T* xout, double omega,
          int sms, int min_seg, cudaStream_t st) {
    const int HC = 2 * POST + 2;
    constexpr int smem = kRing * kNT * static_cast<int>(sizeof(T));
    static PerDeviceOnce once;
    auto kernel = k_mg_up<kNT, POST, PD, MINB, T>;
    const int seg = seg_for(F.nx, F.ny, HC, sms, prepare_kernel(kernel, smem, once), min_seg);
    const int W = kNT - 2 * HC;
    const dim3 grid((F.ny + W - 1) / W, (F.nx + seg - 1) / seg);
    kernel<<<grid, kNT, smem, st>>>(C, F, xin, xout, omega, seg, HC);
    SGPU_LAUNCH();
}

template <int PRE, class T>
void down_t(const LevelViewT<T>& F, const LevelViewT<T>& C, T* xout, bool x_zero, bool build, int sms,
            int min_seg, cudaStream_t st) {
    if constexpr (sizeof(T) == 8) {
        switch (mg_variant64()) {
        case 1: down_v<PRE, 1, 3>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        case 2: down_v<PRE, 1, 4>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        default: down_v<PRE, 2, 2>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        }
    } else {
        switch (mg_variant()) {
        case 0: down_v<PRE, 3, 2>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        case 1: down_v<PRE, 2, 3>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        case 3: down_v<PRE, 1, 5>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        case 4: down_v<PRE, 1, 6>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        default: down_v<PRE, 1, 4>(F, C, xout, x_zero, build, sms, min_seg, st); break;
        }
    }
}

template <int POST, class T>
void up_t(const LevelViewT<T>& C, const LevelViewT<T>& F, const T* xin, T* xout, double omega,
          int sms, int min_seg, cudaStream_t st) {
    if constexpr (sizeof(T) == 8) {
        switch (mg_variant64()) {
        case 1: up_v<POST, 1, 3>(C, F, xin, xout, omega, sms, min_seg, st); break;
        case 2: up_v<POST, 1, 4>(C, F, xin, xout, omega, sms, min_seg, st); break;
        default: up_v<POST, 2, 2>(C, F, xin, xout, omega, sms, min_seg, st); break;
        }
    } else {
        switch (mg_variant()) {
        case 0: up_v<POST, 3, 2>(C, F, xin, xout, omega, sms, min_seg, st); break;
        case 1: up_v<POST, 2, 3>(C, F, xin, xout, omega, sms, min_seg, st); break;
        case 3: up_v<POST, 1, 5>(C, F, xin, xout, omega, sms, min_seg, st); break;
        case 4: up_v<POST, 1, 6>(C, F, xin, xout, omega, sms, min_seg, st); break;
        default: up_v<POST, 1, 4>(C, F, xin, xout, omega, sms, min_seg, st); break;
        }
    }
}

} // namespace

#ifndef SGPU_FLOAT_UNIT
bool mg_fast_supported(int pre, int post) { return pre >= 1 && pre <= 4 && post >= 0 && post <= 4; }
#endif

template <class T>
void launch_mg_down(const LevelViewT<T>& F, const LevelViewT<T>& C, T* xout, int pre, bool x_zero,
                    int sms, int min_seg, cudaStream_t st, bool build) {
    switch (pre) {
    case 1: down_t<1>(F, C, xout, x_zero, build, sms, min_seg, st); break;
    case 2: down_t<2>(F, C, xout, x_zero, build, sms, min_seg, st); break;
    case 3: down_t<3>(F, C, xout, x_zero, build, sms, min_seg, st); break;
    case 4: down_t<4>(F, C, xout, x_zero, build, sms, min_seg, st); break;
    default: throw Error(SGPU_E_INVALID, "streaming multigrid supports mg_pre 1..4");
    }
}

template <class T>
void launch_mg_up(const LevelViewT<T>& C, const LevelViewT<T>& F, const T* xin, T* xout,
                  double omega, int post, int sms, int min_seg, cudaStream_t st) {
    switch (post) {
    case 0: up_t<0>(C, F, xin, xout, omega, sms, min_seg, st); break;
    case 1: up_t<1>(C, F, xin, xout, omega, sms, min_seg, st); break;
    case 2: up_t<2>(C, F, xin, xout, omega, sms, min_seg, st); break;
    case 3: up_t<3>(C, F, xin, xout, omega, sms, min_seg, st); break;
    case 4: up_t<4>(C, F, xin, xout, omega, sms, min_seg, st); break;
    default: throw Error(SGPU_E_INVALID, "streaming multigrid supports mg_post 0..4");
    }
}

// This file alone instantiates the double kernels (built without contraction: the reference's
// bits); mg_fast32.cu includes it with SGPU_FLOAT_UNIT for the float ones (contraction allowed).
#ifndef SGPU_FLOAT_UNIT
template void launch_mg_down<double>(const LevelViewT<double>&, const LevelViewT<double>&, double*,
                                     int, bool, int, int, cudaStream_t, bool);
template void launch_mg_up<double>(const LevelViewT<double>&, const LevelViewT<double>&,
                                   const double*, double*, double, int, int, int, cudaStream_t);
#else
template void launch_mg_down<float>(const LevelViewT<float>&, const LevelViewT<float>&, float*, int,
                                    bool, int, int, cudaStream_t, bool);
template void launch_mg_up<float>(const LevelViewT<float>&, const LevelViewT<float>&, const float*,
                                  float*, double, int, int, int, cudaStream_t);
#endif

} // namespace sgpu
