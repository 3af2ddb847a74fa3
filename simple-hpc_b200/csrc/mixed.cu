// mixed.cu — the mixed-precision outer iteration (config key precision = mixed).
//
// Defect correction around FP32 inner solves; everything SIMPLE's stability and stopping test
// depend on stays FP64:
//  * Momentum. The FP64 prep pass computes each cell's coefficients and the residual
//    R = nb(u) + pressure term - AP u exactly as the FP64 path does (momentum_u.cpp:43-59), and
//    sums |R| into res_u / res_v in FP64 (a fixed tree, not the reference's row-by-row chain: the
//    same value to rounding, and no serial pass over the cells). It also stores, per cell, a 40-byte FP32
//    record in three arrays: the 8 neighbour coefficients, 1/AP and R. The maxit_inner
//    multicolour sweeps then run on the correction e = u_new - u in FP32: the reference's update
//    u <- a (nb(u) + pt) / AP + (1 - a) u (momentum_u.cpp:136-137) is, for u = u0 + e, exactly
//    e <- e + a ((R(u0) + nb(e)) / AP - e), applied in the same colour order by the same
//    time-skewed streaming scheme as the FP64 sweep. The field update u += e is FP64.
//  * Pressure correction. assemble_p (pressure.cpp:14-54) stays FP64 for b, its |b| sum (res_p)
//    and its mean (FP64 trees as above); the p' system's operator is stored in FP32 and solved by the FP32 V-cycle
//    (mg_fast.cu / mg.cu, float instantiation). The mean of p' and the velocity / pressure
//    correction (pressure.cpp:136-157) are FP64.
// Fixed points are those of the FP64 iteration: when R and the continuity residual vanish, e and
// p' vanish too, whatever their precision.
#include "kernels.hpp"
#include "blocksum.cuh"
#include "stencil.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

namespace sgpu {

namespace {

__device__ __forceinline__ std::size_t ix(const DevParams& p, int i, int j) {
    return static_cast<std::size_t>(i) * p.pitch + j;
}

// The correction sweep (k_corr_stream and its launchers) is built in the FP32 unit only.
#ifdef SGPU_FLOAT_UNIT
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

#endif

// The tile of one prep block: 32 columns x kTileRows rows, 32 x 8 threads, kTileRows / 8 cells per
// thread. The block's partial sum (a block tree's tail: one thread adding the warps' sums) is paid
// once per tile.
constexpr int kRowsPerThread = 4;
constexpr int kTileRows = 8 * kRowsPerThread;

// One cell of the prep: AP (FP64) and the cell's FP32 record into the tile in shared memory; returns |R|.
template <bool V>
__device__ __forceinline__ double prep_cell(const DevParams& p, const double* __restrict__ x,
                                            const double* __restrict__ oth, const double* __restrict__ pf,
                                            double* __restrict__ AP, float4& near, float4& far, float2& diag,
                                            int i, int j) {
    const std::size_t q = ix(p, i, j), ld = p.pitch;
    double ue, uw, vn, vs;
    if (!V) {
        ue = (x[q] + x[q + 1]) / 2;
        uw = (x[q] + x[q - 1]) / 2;
        vn = (oth[q] + oth[q + 1]) / 2;
        vs = (oth[q + ld] + oth[q + ld + 1]) / 2;
    } else {
        ue = (oth[q - ld] + oth[q]) / 2;
        uw = (oth[q - 1] + oth[q - ld - 1]) / 2;
        vn = (x[q] + x[q - ld]) / 2;
        vs = (x[q] + x[q + ld]) / 2;
    }
    const Coef9 c = momentum_coef(p, ue, uw, vn, vs, i, j);
    const double nb = (c.AE * x[q + 1] + c.AW * x[q - 1] + c.AN * x[q - ld] + c.AS * x[q + ld]) +
                      (c.AEE * x[q + 2] + c.AWW * x[q - 2] + c.ANN * x[q - 2 * ld] +
                       c.ASS * x[q + 2 * ld]);
    const double pt = V ? (pf[q] - pf[q - ld]) * p.dx : (pf[q] - pf[q + 1]) * p.dy;
    const double R = nb + pt - c.AP * x[q];
    AP[q] = c.AP;
    near = make_float4(static_cast<float>(c.AE), static_cast<float>(c.AW), static_cast<float>(c.AN),
                       static_cast<float>(c.AS));
    far = make_float4(static_cast<float>(c.AEE), static_cast<float>(c.AWW), static_cast<float>(c.ANN),
                      static_cast<float>(c.ASS));
    diag = make_float2(static_cast<float>(1.0 / c.AP), static_cast<float>(R));
    return fabs(R);
}

// FP64 prep over the update range: AP (FP64, for assemble_p and correct), the cell's FP32 record
// {AE AW AN AS | AEE AWW ANN ASS | 1/AP R}, and the block's FP64 sum of |R| (each thread's cells in
// row order, then the deterministic tree of blocksum.cuh) into part[block]; k_sum_partials adds the
// blocks' sums into res_u / res_v.
// The records are stored by sweep step (MomRec32): the block stages its tile's records in shared
// memory, then each warp writes whole step rows, the cells of one step row lying on up to five
// field rows of the tile; a step row the tile shares with its neighbour is written in part by each.
template <bool V>
__global__ void __launch_bounds__(256, 4)
    k_mom_prep_mixed(DevParams p, const double* __restrict__ x, const double* __restrict__ oth,
                     const double* __restrict__ pf, double* __restrict__ AP, double* __restrict__ part,
                     MomRec32 rec, Range ur) {
    __shared__ double s_sum[8];
    __shared__ float4 s_near[kTileRows][32], s_far[kTileRows][32];
    __shared__ float2 s_diag[kTileRows][32];
    const int lane = static_cast<int>(threadIdx.x), wy = static_cast<int>(threadIdx.y);
    const int j = ur.j0 + static_cast<int>(blockIdx.x) * 32 + lane;
    const int ib = ur.i0 + static_cast<int>(blockIdx.y) * kTileRows; // the tile's first row
    double a = 0.0;
    if (j <= ur.j1) {
#pragma unroll 1
        for (int k = 0; k < kRowsPerThread; ++k) {
            const int ti = wy + 8 * k;
            if (ib + ti <= ur.i1)
                a += prep_cell<V>(p, x, oth, pf, AP, s_near[ti][lane], s_far[ti][lane], s_diag[ti][lane],
                                  ib + ti, j);
        }
    }
    const double t = block_sum<8>(a, s_sum, wy * 32 + lane); // its barrier also publishes the tile
    if (lane == 0 && wy == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = t;
    // step rows ib .. ib + kTileRows - 1 + 2 (ncol - 1): cell (i, j) of colour c is updated at step
    // i + 2c, and the cell updated at step s in column j has colour (2s + j) mod 5 (five colours) or
    // (s + j) mod 2 (two)
    const int nsteps = kTileRows + 2 * (p.ncol - 1);
    if (j > ur.j1) return;
    for (int k = wy; k < nsteps; k += 8) {
        const int st = ib + k;
        const int c = p.ncol == 5 ? (2 * st + j) % 5 : (st + j) & 1;
        const int ti = k - 2 * c; // the cell's row in the tile
        if (ti < 0 || ti >= kTileRows || ib + ti > ur.i1) continue;
        const std::size_t q = static_cast<std::size_t>(st) * p.pitch + j;
        rec.near_links[q] = s_near[ti][lane];
        rec.far_links[q] = s_far[ti][lane];
        rec.diag[q] = s_diag[ti][lane];
    }
}

#ifdef SGPU_FLOAT_UNIT
// Rows of the e ring (a power of two). A super-step reads rows down to 2 x the colour count behind
// its step and issues rows up to kRecAhead super-steps ahead: 16 rows live at once for five colours.
// Each thread's row copies land in its own column only, and the threads' vertical reads are in their
// own columns, so a slot is refilled as soon as its owner has written the row out.
constexpr int kRing = 16;
constexpr int kRecAhead = 2; // record slots: super-steps whose records are in flight
constexpr int kSpinLimit = 1 << 20; // bounded mbarrier waits (a give-up is reported, never a hang)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(b)) : "memory");
}
// Arrive (count one) and expect `bytes` of bulk copies to complete on b.
__device__ __forceinline__ void mbar_arrive_expect(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* b, unsigned parity) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_u32(b)), "r"(parity)
                 : "memory");
    return done != 0;
}
// Wait for phase `parity` of b to complete, at most kSpinLimit polls. Returns false on a give-up,
// which also sets *err.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, unsigned* err,
                                          int limit = kSpinLimit) {
    for (int it = 0; !mbar_test(b, parity); ++it)
        if (it >= limit) {
            atomicOr(err, 1u);
            return false;
        }
    return true;
}

// The give-up path of mbar_wait, exercised on purpose: one warp waits, at most `polls` polls, for a
// phase of an mbarrier that nothing ever arrives on, so the wait must end by giving up and setting
// *err. No copy is in flight and nothing else waits on this warp: the kernel returns normally.
__global__ void k_wait_selftest(int polls, unsigned* err) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    mbar_wait(&bar, 0, err, polls);
}
// One bulk copy (TMA, no tensor map) of `bytes` from global to this CTA's shared memory, completing
// on mbarrier b. Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}

// Shared memory of k_corr_stream: the e ring (kRing rows of NT floats), then kRecAhead x SPB record
// slots, each one step row of NT cells in three arrays (near links, far links for five colours,
// {1/AP, R}).
template <int NCOL, int NT> struct CorrSmem {
    static constexpr int SPB = NCOL == 5 ? 2 : 1;
    static constexpr int slots = kRecAhead * SPB;
    static constexpr int ring = kRing * NT * 4;
    static constexpr int near = slots * NT * 16;
    static constexpr int far = NCOL == 5 ? slots * NT * 16 : 0;
    static constexpr int diag = slots * NT * 8;
    static constexpr int bytes = ring + near + far + diag;
    // bytes one step row of records brings in
    static constexpr unsigned row_bytes = NT * (NCOL == 5 ? 40 : 24);
};

// One FP32 multicolour correction sweep e_in -> e_out from the stored records; the time-skewed
// streaming of k_mom_stream (fused.cu): cell (r, j) of colour c at step r + 2c, SPB steps per
// barrier (two for five colours), strip halo 2 per colour.
// Records are stored by step (MomRec32), so the records of one step for the CTA's NT columns are
// three contiguous row segments. Thread 0 fetches them for a whole super-step with bulk copies (TMA)
// into one of kRecAhead slot sets, completing on that set's `full` mbarrier; every thread arrives
// on its `empty` mbarrier once it has read the set, and thread 0 refills the set for the super-step
// kRecAhead later only after that. The e rows are per-thread cp.async copies, one group per
// super-step, waited for kRecAhead super-steps later. Waits are bounded (kSpinLimit); a give-up
// sets *err, which the host reports as SGPU_E_TIMEOUT, and stops the CTA cleanly: the barrier of the
// next super-step tells every thread (__syncthreads_or), no further copy is issued and nothing more
// is written, and thread 0 waits (bounded again) for the record copies it has in flight before the
// CTA exits. The output of such a sweep is invalid. e_zero: e_in is zero and is not read.
template <int NCOL, bool V, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_corr_stream(DevParams p, const float* __restrict__ ein, float* __restrict__ eout,
                  MomRec32 rec, int e_zero, int seg_rows, double* __restrict__ xfinal, unsigned* err) {
    using S = CorrSmem<NCOL, NT>;
    constexpr int SPB = S::SPB;
    constexpr int HC = 2 * NCOL;
    constexpr int W = NT - 2 * HC;
    constexpr int D = kRecAhead;
    constexpr int E0 = SPB * D + 2; // e rows issued before the first super-step
    static_assert(D == 2, "the step loop is unrolled over the two record slot sets");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* ring_mem = reinterpret_cast<float*>(smem_raw);
    float4* s_near = reinterpret_cast<float4*>(smem_raw + S::ring);
    float4* s_far = reinterpret_cast<float4*>(smem_raw + S::ring + S::near);
    float2* s_diag = reinterpret_cast<float2*>(smem_raw + S::ring + S::near + S::far);
    __shared__ int s_rmin[NCOL], s_rmax[NCOL];
    __shared__ __align__(8) unsigned long long full[D], empty[D];
    const int tid = threadIdx.x;
    const int j0 = blockIdx.x * W;
    const int C0 = j0 - HC, C1 = j0 + W + HC;
    const int col = C0 + tid;
    const int R0 = blockIdx.y * seg_rows;
    const int R1 = min(R0 + seg_rows, p.nrows);
    const int L0 = max(R0 - HC, 0), L1 = min(R1 + HC, p.nrows);
    const int ld = p.pitch;
    const bool col_in = col >= 0 && col < p.ncols;
    const bool col_out = col_in && col >= j0 && col < j0 + W;
    // the update range (xfinal: the last sweep adds e to the FP64 field there, x += e)
    const int ui0 = V ? p.H + 1 : p.H, ui1 = p.NX + p.H - 1;
    const int uj0 = p.H + 1, uj1 = V ? p.NY + p.H : p.NY + p.H - 1;
    const int H = p.H;
    if (tid < NCOL) {
        const int c = tid;
        int lo = V ? H + 1 : H, hi = p.NX + H - 1;
        if (L0 > 0) lo = max(lo, L0 + 2 + 2 * c);
        if (L1 < p.nrows) hi = min(hi, L1 - 3 - 2 * c);
        s_rmin[c] = lo;
        s_rmax[c] = hi;
    }
    if (tid == 0) {
        for (int d = 0; d < D; ++d) {
            mbar_init(&full[d], 1);
            mbar_init(&empty[d], NT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
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
    const float relax = static_cast<float>(V ? p.av : p.au);
    float* ringc = ring_mem + tid;
    // Running offsets: the next e row to issue and the row the next super-step writes out.
    int next = L0;
    int eo = col + L0 * ld;
    int wo = col + (L0 - 2 * NCOL + 1 - (SPB - 1)) * ld;
    auto issue_row = [&]() {
        if (next < L1 && col_in) {
            float* dst = ringc + (next & (kRing - 1)) * NT;
            if (e_zero) *dst = 0.0f;
            else cp_async(dst, ein + eo);
        }
        ++next;
        eo += ld;
    };
    auto step_cell = [&](int c, int t, int& r) -> bool {
        r = t - 2 * c;
        return ((colmask >> c) & 1u) && r >= s_rmin[c] && r <= s_rmax[c];
    };
    auto next_colour = [&](int c, int steps) {
        return NCOL == 5 ? (c + 2 * steps) % 5 : (c + steps) & 1;
    };
    // Thread 0: the records of the super-step whose first step is t into slot set `slot`, completing
    // phase `parity` of full[slot]. Step rows past the arrays' end hold no cell and are not fetched.
    // `inflight` (thread 0 only) marks the slot sets whose copies thread 0 has not yet seen land.
    const int rec_rows = p.nrows + kRecExtraRows;
    unsigned inflight = 0, inflight_parity = 0;
    auto fill = [&](int slot, int t, unsigned parity) {
        inflight |= 1u << slot;
        inflight_parity = (inflight_parity & ~(1u << slot)) | (parity << slot);
        unsigned bytes = 0;
#pragma unroll
        for (int s = 0; s < SPB; ++s)
            if (t + s < rec_rows) bytes += S::row_bytes;
        mbar_arrive_expect(&full[slot], bytes);
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            if (t + s >= rec_rows) continue;
            const std::ptrdiff_t o = static_cast<std::ptrdiff_t>(t + s) * ld + C0;
            const int q = (slot * SPB + s) * NT;
            bulk_load(s_near + q, rec.near_links + o, NT * 16, &full[slot]);
            if (NCOL == 5) bulk_load(s_far + q, rec.far_links + o, NT * 16, &full[slot]);
            bulk_load(s_diag + q, rec.diag + o, NT * 8, &full[slot]);
        }
    };
    auto update = [&](int r, int q) {
        const float4 a = s_near[q];
        const float2 dg = s_diag[q];
        float* rc = ringc + (r & (kRing - 1)) * NT;
        const float ee = rc[1], ew = rc[-1];
        const float en = ringc[((r - 1) & (kRing - 1)) * NT];
        const float es = ringc[((r + 1) & (kRing - 1)) * NT];
        float nb = a.x * ee + a.y * ew + a.z * en + a.w * es;
        if (NCOL == 5) {
            const float4 b = s_far[q];
            const float eee = rc[2], eww = rc[-2];
            const float enn = ringc[((r - 2) & (kRing - 1)) * NT];
            const float ess = ringc[((r + 2) & (kRing - 1)) * NT];
            nb += b.x * eee + b.y * eww + b.z * enn + b.w * ess;
        }
        const float e0 = rc[0];
        rc[0] = e0 + relax * ((dg.y + nb) * dg.x - e0);
    };
    // The last sweep (xfinal) adds e into x: x of the rows a super-step writes is loaded one
    // super-step ahead, so the read-modify-write does not wait on memory inside the step.
    auto x_row = [&](int rw) {
        return rw >= R0 && rw < R1 && col_out && rw >= ui0 && rw <= ui1 && col >= uj0 && col <= uj1;
    };
    double xpre[SPB];

    __syncthreads(); // s_rmin / s_rmax and the initialised mbarriers
    const int c_start = NCOL == 5 ? (2 * L0 + col + 1000) % 5 : (L0 + col + 1000) & 1;
    const int t_last = R1 + 2 * NCOL - 2 + (SPB - 1);
    // prologue: D e-row groups, the first with E0 rows; the records of super-steps 0 .. D-1
    for (int i = 0; i < E0; ++i) issue_row();
    cp_async_commit();
    cp_async_commit();
    if (tid == 0) {
        fill(0, L0, 0u);
        if (L0 + SPB <= t_last) fill(1, L0 + SPB, 0u);
    }
#pragma unroll
    for (int s = 0; s < SPB; ++s) {
        const int rw = L0 - 2 * NCOL + 1 - (SPB - 1) + s;
        xpre[s] = (xfinal && x_row(rw)) ? xfinal[wo + s * ld] : 0.0;
    }

    int c_cur = c_start;
    bool gave_up = false; // a bounded wait of this thread ran out
    // One super-step; false when a wait of any thread has given up (the CTA then stops).
    auto super_step = [&](int t, int slot, unsigned parity) -> bool {
        cp_async_wait<D - 1>(); // this thread's e rows for this super-step have landed
        if (mbar_wait(&full[slot], parity, err)) { // the slot set's records have landed
            if (tid == 0) inflight &= ~(1u << slot);
        } else {
            gave_up = true;
        }
        if (__syncthreads_or(gave_up ? 1 : 0)) return false; // ... and everyone's e rows
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            int r;
            if (step_cell(next_colour(c_cur, s), t + s, r)) update(r, (slot * SPB + s) * NT + tid);
        }
        mbar_arrive(&empty[slot]); // this thread is done with the slot set
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            const int rw = t - 2 * NCOL + 1 - (SPB - 1) + s;
            const float ev = ringc[(rw & (kRing - 1)) * NT];
            if (!xfinal) {
                if (rw >= R0 && rw < R1 && col_out) eout[wo + s * ld] = ev;
            } else if (x_row(rw)) { // the last sweep: x += e
                xfinal[wo + s * ld] = xpre[s] + static_cast<double>(ev);
            }
        }
        wo += SPB * ld;
        if (xfinal) {
#pragma unroll
            for (int s = 0; s < SPB; ++s) { // the rows the next super-step writes
                const int rw = t + SPB - 2 * NCOL + 1 - (SPB - 1) + s;
                if (x_row(rw)) xpre[s] = xfinal[wo + s * ld];
            }
        }
        // e rows land in ring rows no one reads before the next barriers
#pragma unroll
        for (int s = 0; s < SPB; ++s) issue_row();
        cp_async_commit();
        c_cur = next_colour(c_cur, SPB);
        // Thread 0 refills the slot set for the super-step D later once every thread has read it;
        // a super-step past the last is not fetched, so no copy is in flight when the CTA exits.
        if (tid == 0 && t + SPB * D <= t_last) {
            if (mbar_wait(&empty[slot], parity, err)) fill(slot, t + SPB * D, parity ^ 1u);
            else gave_up = true; // not refilled: the next super-step's barrier stops the CTA
        }
        return true;
    };
    unsigned parity = 0;
    for (int t = L0; t <= t_last; t += 2 * SPB) {
        if (!super_step(t, 0, parity)) break;
        if (t + SPB <= t_last && !super_step(t + SPB, 1, parity)) break;
        parity ^= 1u;
    }
    // After a give-up, record copies may still be in flight into this CTA's shared memory: wait for
    // them (bounded) before exiting. On the normal path nothing is in flight here.
    if (tid == 0)
        for (int sl = 0; sl < D; ++sl)
            if ((inflight >> sl) & 1u) mbar_wait(&full[sl], (inflight_parity >> sl) & 1u, err);
    cp_async_wait<0>();
}

// ---- small grids: all of a component's correction sweeps on one thread-block cluster ----
//
// Where the whole component fits (40 B of records and 4 B of e per cell over kCorrCluster CTAs'
// shared memory), one 16-CTA cluster runs every inner sweep: the update range's rows are split into
// bands, each CTA holding its band's records and its e with two ghost rows on each side (the
// stencil's reach). The sweeps go colour by colour, as the reference's (momentum_u.cpp:123-143), the
// colour-c cells of every band updated with the same expression as k_corr_stream; a cluster barrier
// ends each colour. An update of one of a band's first or last two rows also stores the value into
// the neighbouring band's ghost copy (distributed shared memory): no cell of the stencil shares a
// cell's colour, so within a colour pass no ghost cell that is written is read, and the barrier
// publishes them. e starts at zero (the first sweep's e_in) and the FP64 field takes x += e at the
// end, as the streaming kernels' last sweep does. One launch replaces maxit_inner launches, each of
// which walked its halo and colour skew rows at a barrier per super-step.
constexpr int kCorrCluster = 16;
constexpr int kCorrGhost = 2;

struct CorrClusterPlan {
    int band[kCorrCluster + 1]; // first row of each CTA's band of the update range (band[R]: one past)
    int rows;                   // rows of the largest band
    int bytes;                  // dynamic shared memory per CTA
};

template <int NCOL, bool V>
__global__ void __launch_bounds__(512)
    k_corr_cluster(DevParams p, MomRec32 rec, CorrClusterPlan pl, int nsweeps, double* __restrict__ x) {
    namespace cg = cooperative_groups;
    constexpr int G = kCorrGhost;
    extern __shared__ __align__(16) unsigned char cs_raw[];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = static_cast<int>(cl.block_rank()), R = static_cast<int>(cl.num_blocks());
    const int nc = p.ncols, i0 = pl.band[rank], m = pl.band[rank + 1] - i0;
    const int ne = ((pl.rows + 2 * G) * nc + 3) & ~3;
    float* e = reinterpret_cast<float*>(cs_raw); // rows -G .. rows + G - 1 of the band, all columns
    float4* s_near = reinterpret_cast<float4*>(e + ne);
    float4* s_far = s_near + pl.rows * nc;
    float2* s_diag = reinterpret_cast<float2*>(NCOL == 5 ? s_far + pl.rows * nc : s_far);
    const int uj0 = p.H + 1, uj1 = V ? p.NY + p.H : p.NY + p.H - 1;
    const float relax = static_cast<float>(V ? p.av : p.au);
    cl.sync(); // every CTA of the cluster runs before any touches another's shared memory
    for (int k = threadIdx.x; k < (m + 2 * G) * nc; k += blockDim.x) e[k] = 0.0f;
    for (int k = threadIdx.x; k < m * nc; k += blockDim.x) {
        const int Il = k / nc, j = k - Il * nc, i = i0 + Il;
        if (j < uj0 || j > uj1) continue;
        const int c = NCOL == 5 ? (i + 3 * j) % 5 : (i + j) & 1; // the record sits at step row i + 2c
        const std::size_t q = static_cast<std::size_t>(i + 2 * c) * p.pitch + j;
        s_near[k] = rec.near_links[q];
        if (NCOL == 5) s_far[k] = rec.far_links[q];
        s_diag[k] = rec.diag[q];
    }
    // The band above holds our rows 0 .. G-1 as its bottom ghost rows (its local rows mup ..), the
    // band below our rows m-G .. m-1 as its top ghost rows (its local rows -G .. -1).
    float* eup = rank > 0 ? cl.map_shared_rank(e, rank - 1) : nullptr;
    float* edn = rank < R - 1 ? cl.map_shared_rank(e, rank + 1) : nullptr;
    const int mup = rank > 0 ? i0 - pl.band[rank - 1] : 0;
    cl.sync();
    const int lane = static_cast<int>(threadIdx.x) & 31, w = static_cast<int>(threadIdx.x) >> 5;
    const int nw = static_cast<int>(blockDim.x) >> 5;
    for (int sw = 0; sw < nsweeps; ++sw)
        for (int c = 0; c < NCOL; ++c) {
            for (int Il = w; Il < m; Il += nw) {
                const int i = i0 + Il;
                // the colour-c cells of row i: j = 2 (c - i) mod 5 (five colours), (c - i) mod 2 (two)
                const int res = NCOL == 5 ? ((2 * (c - i)) % 5 + 5) % 5 : ((c - i) & 1);
                for (int j = uj0 + ((res - uj0) % NCOL + NCOL) % NCOL + NCOL * lane; j <= uj1; j += NCOL * 32) {
                    const int k = Il * nc + j;
                    const float4 a = s_near[k];
                    const float2 dg = s_diag[k];
                    float* rc = e + (Il + G) * nc + j;
                    const float ee = rc[1], ew = rc[-1];
                    const float en = rc[-nc], es = rc[nc];
                    float nb = a.x * ee + a.y * ew + a.z * en + a.w * es;
                    if (NCOL == 5) {
                        const float4 b = s_far[k];
                        const float eee = rc[2], eww = rc[-2];
                        const float enn = rc[-2 * nc], ess = rc[2 * nc];
                        nb += b.x * eee + b.y * eww + b.z * enn + b.w * ess;
                    }
                    const float e0 = rc[0];
                    const float v = e0 + relax * ((dg.y + nb) * dg.x - e0);
                    rc[0] = v;
                    if (Il < G && eup) eup[(mup + G + Il) * nc + j] = v;
                    if (Il >= m - G && edn) edn[(Il - m + G) * nc + j] = v;
                }
            }
            cl.sync();
        }
    for (int k = threadIdx.x; k < m * nc; k += blockDim.x) { // x += e (FP64), the own cells
        const int Il = k / nc, j = k - Il * nc;
        if (j < uj0 || j > uj1) continue;
        const std::size_t q = static_cast<std::size_t>(i0 + Il) * p.pitch + j;
        x[q] = x[q] + static_cast<double>(e[(Il + G) * nc + j]);
    }
}

#endif // SGPU_FLOAT_UNIT

// Rows per thread of k_assemble_p_mixed, and the first (even) column of the column pairs that the
// pair kernels (k_assemble_p_mixed, k_correct_mixed) give each thread.
constexpr int kAsmRows = 1;
__host__ __device__ __forceinline__ int pair_col0(const DevParams& p) { return (p.H + 1) & ~1; }
__host__ __device__ __forceinline__ int pair_count(const DevParams& p) { return (p.NY + p.H - pair_col0(p)) / 2 + 1; }
__device__ __forceinline__ double2 ld2(const double* q) { return *reinterpret_cast<const double2*>(q); }

// assemble_p (pressure.cpp:14-54) in FP64 with the p' operator stored in FP32 (level 0 of the FP32
// hierarchy), and the block's FP64 sums of |b| (res_p) and of b (its mean) into part[block] and
// part[nblocks + block] (each thread's cells in a fixed order, then the deterministic trees of
// blocksum.cuh). Each thread takes two adjacent columns (j even: 16-byte pairs of the FP64 arrays)
// in kAsmRows rows, and issues all its loads before the first cell's arithmetic. At 4096^2: 0.20 ms,
// against 0.25 ms for one cell per thread in four rows (and 0.22 ms for pairs in two rows, whose 90
// registers leave two CTAs per SM).
__global__ void __launch_bounds__(256)
    k_assemble_p_mixed(DevParams p, const double* __restrict__ APU, const double* __restrict__ APV,
                       const double* __restrict__ u, const double* __restrict__ v,
                       double* __restrict__ bfield, LevelView32 L0, double* __restrict__ part) {
    constexpr int R = kAsmRows;
    __shared__ double s_abs[8], s_b[8];
    const int H = p.H;
    const int j = pair_col0(p) + 2 * static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I0 = static_cast<int>(blockIdx.y * 8 * R + threadIdx.y);
    const bool jin = j <= p.NY + H; // the pair holds at least one cell
    const std::size_t ld = p.pitch;
    double2 apu[R], apv[R], apvs[R], uu[R], vv[R], vs[R];
    double apuw[R], uw[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int I = I0 + 8 * k;
        if (!jin || I >= p.NX) continue;
        const std::size_t q = ix(p, H + I, j);
        apu[k] = ld2(APU + q);
        apuw[k] = APU[q - 1];
        apv[k] = ld2(APV + q);
        apvs[k] = ld2(APV + q + ld);
        uu[k] = ld2(u + q);
        uw[k] = u[q - 1];
        vv[k] = ld2(v + q);
        vs[k] = ld2(v + q + ld);
    }
    const double dx = p.dx, dy = p.dy;
    double sa = 0.0, sb = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int I = I0 + 8 * k;
        if (!jin || I >= p.NX) continue;
        const int i = H + I;
        const std::size_t q = ix(p, i, j);
        // the pair's two cells: e = 0 at column j, e = 1 at j + 1 (pressure.cpp:22-44)
        const double apu_e[2] = {apu[k].x, apu[k].y}, apu_w[2] = {apuw[k], apu[k].x};
        const double apv_n[2] = {apv[k].x, apv[k].y}, apv_s[2] = {apvs[k].x, apvs[k].y};
        const double u_e[2] = {uu[k].x, uu[k].y}, u_w[2] = {uw[k], uu[k].x};
        const double v_n[2] = {vv[k].x, vv[k].y}, v_s[2] = {vs[k].x, vs[k].y};
        double bq[2];
        bool cell[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int jj = j + e;
            cell[e] = jj >= H + 1 && jj <= p.NY + H;
            if (!cell[e]) continue;
            const double aep = (jj == p.NY + H) ? 0.0 : dy * dy / apu_e[e];
            const double awp = (jj == H + 1) ? 0.0 : dy * dy / apu_w[e];
            const double anp = (i == H) ? 0.0 : dx * dx / apv_n[e];
            const double asp = (i == p.NX + H - 1) ? 0.0 : dx * dx / apv_s[e];
            const int lq = I * L0.stride + (jj - H - 1);
            set_links(L0, lq, static_cast<float>(aep), static_cast<float>(awp), static_cast<float>(anp),
                      static_cast<float>(asp));
            L0.AP[lq] = static_cast<float>(aep + awp + anp + asp);
            bq[e] = -dx * (-v_s[e] + v_n[e]) - dy * (-u_w[e] + u_e[e]);
            sa += fabs(bq[e]);
            sb += bq[e];
        }
        if (cell[0] && cell[1]) *reinterpret_cast<double2*>(bfield + q) = make_double2(bq[0], bq[1]);
        else if (cell[0]) bfield[q] = bq[0];
        else if (cell[1]) bfield[q + 1] = bq[1];
    }
    const int tid = static_cast<int>(threadIdx.y * 32 + threadIdx.x);
    const double ta = block_sum<8>(sa, s_abs, tid);
    const double tb = block_sum<8>(sb, s_b, tid);
    if (tid == 0) {
        const unsigned nb = gridDim.x * gridDim.y, k = blockIdx.y * gridDim.x + blockIdx.x;
        part[k] = ta;
        part[nb + k] = tb;
    }
}

// b32 = b - mean(b), rounded to FP32 (remove_mean0, multigrid.cpp:327-345, in FP64 first).
__global__ void k_b_to_f32(DevParams p, const double* __restrict__ bfield, const double* __restrict__ sum_b,
                           LevelView32 L0) {
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I0 = static_cast<int>(blockIdx.y * kTileRows + threadIdx.y);
    if (J >= p.NY) return;
    const double m = *sum_b / (static_cast<double>(p.NX) * p.NY);
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) { // rows I0, I0 + 8, ...: more loads in flight per thread
        const int I = I0 + 8 * k;
        if (I < p.NX) L0.b[I * L0.stride + J] = static_cast<float>(bfield[ix(p, p.H + I, p.H + 1 + J)] - m);
    }
}

// correct (pressure.cpp:136-157) in FP64 from the FP32 p' minus its FP64 mean (the FP64 p' field
// is formed from it on demand, k_pc_from32). Two adjacent columns per thread: the FP64 arrays are read and written as
// 16-byte pairs (j even; the pitch is even), the FP32 p' as scalars. Elements of a pair that are not
// cells of the correction keep their values (the thread writes back what it read). Against one cell
// per thread with 8-byte accesses (4096^2: 0.26 ms, long-scoreboard bound), the pairs halve the
// load instructions and double the bytes each one has in flight: 0.17 ms.
__global__ void __launch_bounds__(256)
    k_correct_mixed(DevParams p, const float* __restrict__ pc32, int ld32,
                          const double* __restrict__ sum_pc, const double* __restrict__ APU,
                          const double* __restrict__ APV, double* __restrict__ u, double* __restrict__ v,
                          double* __restrict__ pf) {
    const int H = p.H;
    const int j = pair_col0(p) + 2 * static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (I >= p.NX || j > p.NY + H) return;
    const int i = H + I;
    const std::size_t q = ix(p, i, j);
    const double m = *sum_pc / (static_cast<double>(p.NX) * p.NY);
    const double2 pp = *reinterpret_cast<const double2*>(pf + q);
    const double2 uu = *reinterpret_cast<const double2*>(u + q);
    const double2 au = *reinterpret_cast<const double2*>(APU + q);
    double2 vv = make_double2(0.0, 0.0), av = make_double2(1.0, 1.0);
    if (I >= 1) {
        vv = *reinterpret_cast<const double2*>(v + q);
        av = *reinterpret_cast<const double2*>(APV + q);
    }
    const float* pcr = pc32 + I * ld32 + (j - H - 1); // p' of column j; j - H - 1 >= -1 (zero ring)
    const float c0 = pcr[0], c1 = pcr[1], c2 = pcr[2];
    const float n0 = I >= 1 ? pcr[-ld32] : 0.0f, n1 = I >= 1 ? pcr[1 - ld32] : 0.0f;
    double2 pn = pp, un = uu, vn = vv;
    const bool cell0 = j >= H + 1, cell1 = j + 1 <= p.NY + H;
    if (cell0) {
        const double pc = static_cast<double>(c0) - m;
        if (j <= p.NY + H - 1) un.x = uu.x + p.dy * (pc - (static_cast<double>(c1) - m)) / au.x;
        if (I >= 1) vn.x = vv.x + p.dx * (pc - (static_cast<double>(n0) - m)) / av.x;
        pn.x = pp.x + p.ap * pc;
    }
    if (cell1) {
        const double pc = static_cast<double>(c1) - m;
        if (j + 1 <= p.NY + H - 1) un.y = uu.y + p.dy * (pc - (static_cast<double>(c2) - m)) / au.y;
        if (I >= 1) vn.y = vv.y + p.dx * (pc - (static_cast<double>(n1) - m)) / av.y;
        pn.y = pp.y + p.ap * pc;
    }
    *reinterpret_cast<double2*>(pf + q) = pn;
    *reinterpret_cast<double2*>(u + q) = un;
    if (I >= 1) *reinterpret_cast<double2*>(v + q) = vn;
}

// The FP64 p' field as k_correct_mixed uses it (FP32 p' minus its FP64 mean), for a download.
__global__ void k_pc_from32(DevParams p, const float* __restrict__ pc32, int ld32,
                            const double* __restrict__ sum_pc, double* __restrict__ pc64) {
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (I >= p.NX || J >= p.NY) return;
    const double m = *sum_pc / (static_cast<double>(p.NX) * p.NY);
    pc64[ix(p, p.H + I, p.H + 1 + J)] = static_cast<double>(pc32[I * ld32 + J]) - m;
}

// ---- FP64 defect correction of the p' solve (precision = mixed, mg_mode = tolerance) ----
//
// The FP32 V-cycle alone stalls at the FP32 rounding of its operator and iterate: ||b - A p'|| stops
// falling near 1e-6 ||b|| on large grids. In tolerance mode the p' iterate is therefore kept in FP64
// and each V-cycle solves for a correction: r = (b - mean b) - A p' with the FP64 operator of
// assemble_p (its links formed from APU / APV by the expressions of k_assemble_p_mixed,
// pressure.cpp:14-54), rounded to FP32 as the cycle's right-hand side; the cycle, from zero, gives e;
// p' += e in FP64. The tolerance test reads the norm of that FP64 residual.

// The first right-hand side, b - mean(b) rounded to FP32, and per block the FP64 sum of (b - mean b)^2.
__global__ void __launch_bounds__(256)
    k_dc_rhs0(DevParams p, const double* __restrict__ bfield, const double* __restrict__ sum_b, LevelView32 L0,
              double* __restrict__ part) {
    __shared__ double s_bb[8];
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I0 = static_cast<int>(blockIdx.y * kTileRows + threadIdx.y);
    const double m = *sum_b / (static_cast<double>(p.NX) * p.NY);
    double bb = 0.0;
    if (J < p.NY) {
#pragma unroll
        for (int k = 0; k < kRowsPerThread; ++k) {
            const int I = I0 + 8 * k;
            if (I < p.NX) {
                const double b = bfield[ix(p, p.H + I, p.H + 1 + J)] - m;
                L0.b[I * L0.stride + J] = static_cast<float>(b);
                bb += b * b;
            }
        }
    }
    const int tid = static_cast<int>(threadIdx.y * 32 + threadIdx.x);
    const double t = block_sum<8>(bb, s_bb, tid);
    if (tid == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = t;
}

// One defect-correction step over the p' cells (I, J) (field cell (H + I, H + 1 + J)):
// pnew = pold + e (pold = 0 when first), then r = (b - mean b) - (APP pnew - (AEP pE + AWP pW + ASP pS
// + ANP pN)) with the FP64 links (the multigrid residual form, multigrid.cpp:73-87), L0.b = FP32 r,
// and per block the FP64 sums of r^2 (part[k]) and of pnew (part[nblocks + k]). pold and pnew are
// distinct full-grid arrays: a cell's neighbours are read from pold + e, never from pnew.
__global__ void __launch_bounds__(256)
    k_dc_update(DevParams p, const double* __restrict__ APU, const double* __restrict__ APV,
                const double* __restrict__ bfield, const double* __restrict__ sum_b,
                const float* __restrict__ e, int lde, const double* __restrict__ pold,
                double* __restrict__ pnew, int first, LevelView32 L0, double* __restrict__ part) {
    __shared__ double s_rr[8], s_ps[8];
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I0 = static_cast<int>(blockIdx.y * kTileRows + threadIdx.y);
    const double m = *sum_b / (static_cast<double>(p.NX) * p.NY);
    const int H = p.H;
    const std::size_t ld = p.pitch;
    double rr = 0.0, ps = 0.0;
    if (J < p.NY) {
#pragma unroll 1
        for (int k = 0; k < kRowsPerThread; ++k) {
            const int I = I0 + 8 * k;
            if (I >= p.NX) break;
            const int i = H + I, j = H + 1 + J;
            const std::size_t q = ix(p, i, j);
            const float* ec = e + I * lde + J; // e's zero ring covers the neighbours outside
            auto pv = [&](std::size_t qq, const float* ee) {
                return (first ? 0.0 : pold[qq]) + static_cast<double>(*ee);
            };
            const double dx = p.dx, dy = p.dy;
            const double aep = (j == p.NY + H) ? 0.0 : dy * dy / APU[q];
            const double awp = (j == H + 1) ? 0.0 : dy * dy / APU[q - 1];
            const double anp = (i == H) ? 0.0 : dx * dx / APV[q];
            const double asp = (i == p.NX + H - 1) ? 0.0 : dx * dx / APV[q + ld];
            const double app = aep + awp + anp + asp;
            const double pc = pv(q, ec);
            const double pe = aep != 0.0 ? pv(q + 1, ec + 1) : 0.0;
            const double pw = awp != 0.0 ? pv(q - 1, ec - 1) : 0.0;
            const double pn = anp != 0.0 ? pv(q - ld, ec - lde) : 0.0;
            const double psn = asp != 0.0 ? pv(q + ld, ec + lde) : 0.0;
            const double r = (bfield[q] - m) - (app * pc - (aep * pe + awp * pw + asp * psn + anp * pn));
            pnew[q] = pc;
            L0.b[I * L0.stride + J] = static_cast<float>(r);
            rr += r * r;
            ps += pc;
        }
    }
    const int tid = static_cast<int>(threadIdx.y * 32 + threadIdx.x);
    const double trr = block_sum<8>(rr, s_rr, tid);
    const double tps = block_sum<8>(ps, s_ps, tid);
    if (tid == 0) {
        const unsigned nb = gridDim.x * gridDim.y, kb = blockIdx.y * gridDim.x + blockIdx.x;
        part[kb] = trr;
        part[nb + kb] = tps;
    }
}

// correct (pressure.cpp:136-157) in FP64 from the FP64 p' of the defect correction minus its mean.
__global__ void k_correct_dc(DevParams p, const double* __restrict__ pc64, const double* __restrict__ sum_pc,
                             const double* __restrict__ APU, const double* __restrict__ APV, double* u,
                             double* v, double* pf) {
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (I >= p.NX || J >= p.NY) return;
    const int H = p.H, i = H + I, j = H + 1 + J;
    const std::size_t q = ix(p, i, j);
    const double m = *sum_pc / (static_cast<double>(p.NX) * p.NY);
    const double pc = pc64[q] - m;
    if (j <= p.NY + H - 1) u[q] += p.dy * (pc - (pc64[q + 1] - m)) / APU[q];
    if (i >= H + 1) v[q] += p.dx * (pc - (pc64[q - p.pitch] - m)) / APV[q];
    pf[q] += p.ap * pc;
}

// The p' field a download shows: the FP64 iterate minus its mean (src may equal dst).
__global__ void k_pc_from64(DevParams p, const double* src, const double* __restrict__ sum_pc, double* dst) {
    const int J = static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    const int I = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (I >= p.NX || J >= p.NY) return;
    const double m = *sum_pc / (static_cast<double>(p.NX) * p.NY);
    const std::size_t q = ix(p, p.H + I, p.H + 1 + J);
    dst[q] = src[q] - m;
}

Range update_range(const DevParams& p, bool v) {
    const int H = p.H;
    return v ? Range{H + 1, p.NX + H - 1, H + 1, p.NY + H} : Range{H, p.NX + H - 1, H + 1, p.NY + H - 1};
}

#ifdef SGPU_FLOAT_UNIT
// Threads per CTA of the correction sweep and the resident CTAs per SM its registers are bounded
// for: 224 threads (7 warps) keep the e ring and the two record slot sets at 50 KB, so four CTAs
// (28 warps) fit an SM, where 256 threads fit three (24 warps, 3% slower at 4096^2).
constexpr int kCorrNT = 224;
constexpr int kCorrMinb = 4;

template <int NCOL, bool V, int NT, int MINB>
void launch_corr(const DevParams& p, const float* ein, float* eout, MomRec32 rec, bool e_zero,
                 int seg_rows, double* xfinal, unsigned* err, cudaStream_t st) {
    // The bulk copies start at record (t * pitch + first column): 16-byte aligned for every step
    // row t and CTA when the arrays are and the pitch and first columns are even (the strips
    // start at multiples of NT - 4 NCOL, minus 2 NCOL).
    const auto misaligned = [](const void* q) { return (reinterpret_cast<std::uintptr_t>(q) & 15u) != 0; };
    if ((p.pitch & 1) || misaligned(rec.near_links) || misaligned(rec.far_links) || misaligned(rec.diag) || !err)
        throw Error(SGPU_E_INVALID, "correction sweep: records not aligned for bulk copies");
    constexpr int W = NT - 4 * NCOL;
    static_assert(W % 2 == 0 && (2 * NCOL) % 2 == 0, "strip starts must be even");
    static_assert(2 * NCOL <= kRecFrontCols && NT <= kRecBackCols, "copy windows must stay in the margins");
    const dim3 grid((p.ncols + W - 1) / W, (p.nrows + seg_rows - 1) / seg_rows);
    constexpr int smem = CorrSmem<NCOL, NT>::bytes;
    k_corr_stream<NCOL, V, NT, MINB><<<grid, NT, smem, st>>>(p, ein, eout, rec, e_zero ? 1 : 0, seg_rows,
                                                              xfinal, err);
    SGPU_LAUNCH();
}

template <int NCOL, bool V>
void launch_corr_m(const DevParams& p, const float* ein, float* eout, MomRec32 rec, bool e_zero,
                   int seg_rows, double* xfinal, unsigned* err, cudaStream_t st) {
    launch_corr<NCOL, V, kCorrNT, kCorrMinb>(p, ein, eout, rec, e_zero, seg_rows, xfinal, err, st);
}


// The cluster sweep's plan: bands of at least kCorrGhost rows, the shared memory of the largest
// within a CTA's 227 KB; false where the component does not fit.
bool corr_cluster_plan(const DevParams& p, bool v, CorrClusterPlan& pl) {
    const Range ur = update_range(p, v);
    const int n = ur.rows();
    if (n < kCorrGhost * kCorrCluster || ur.cols() <= 0) return false;
    for (int r = 0; r <= kCorrCluster; ++r) pl.band[r] = ur.i0 + (r * n) / kCorrCluster;
    pl.rows = (n + kCorrCluster - 1) / kCorrCluster;
    const long long ne = ((static_cast<long long>(pl.rows) + 2 * kCorrGhost) * p.ncols + 3) / 4 * 4;
    const long long bytes = ne * 4 + static_cast<long long>(pl.rows) * p.ncols * (p.ncol == 5 ? 40 : 24);
    if (bytes > 227 * 1024) return false;
    pl.bytes = static_cast<int>(bytes);
    return true;
}

// Whether this device runs the cluster sweep (its attributes set once per device, one cluster of
// kCorrCluster CTAs with 227 KB each resident). SGPU_CORR_CLUSTER=0 turns it off.
bool corr_cluster_available() {
    if (const char* e = std::getenv("SGPU_CORR_CLUSTER"))
        if (std::atoi(e) == 0) return false;
    static PerDeviceOnce once;
    return once.get([] {
        // a device that refuses either attribute runs the streaming sweep
        auto setup = [](auto kernel) {
            return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) ==
                       cudaSuccess &&
                   cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
        };
        if (!setup(k_corr_cluster<5, false>) || !setup(k_corr_cluster<5, true>) || !setup(k_corr_cluster<2, false>) ||
            !setup(k_corr_cluster<2, true>)) {
            (void)cudaGetLastError();
            return 0;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kCorrCluster);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = 227 * 1024;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kCorrCluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, k_corr_cluster<5, false>, &cfg) != cudaSuccess) {
            (void)cudaGetLastError(); // not supported here: the clear-up of the failed query
            return 0;
        }
        return nclusters > 0 ? 1 : 0;
    }) != 0;
}

template <int NCOL, bool V>
void launch_corr_cluster_t(const DevParams& p, MomRec32 rec, const CorrClusterPlan& pl, int nsweeps, double* x,
                           cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCorrCluster);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = static_cast<std::size_t>(pl.bytes);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kCorrCluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    SGPU_CUDA(cudaLaunchKernelEx(&cfg, k_corr_cluster<NCOL, V>, p, rec, pl, nsweeps, x));
    SGPU_LAUNCH();
}
#endif // SGPU_FLOAT_UNIT

} // namespace

// This file alone defines the FP64 launchers (built without contraction); mixed32.cu includes it
// with SGPU_FLOAT_UNIT for the FP32 correction sweep (contraction allowed).
#ifndef SGPU_FLOAT_UNIT
int launch_mom_prep_mixed(const DevParams& p, bool v_component, const double* x, const double* oth,
                          const double* pf, double* AP, double* part, MomRec32 rec, cudaStream_t st) {
    const Range ur = update_range(p, v_component);
    if (ur.rows() <= 0 || ur.cols() <= 0) return 0;
    const dim3 grid((ur.cols() + 31) / 32, (ur.rows() + 8 * kRowsPerThread - 1) / (8 * kRowsPerThread));
    if (v_component) k_mom_prep_mixed<true><<<grid, dim3(32, 8), 0, st>>>(p, x, oth, pf, AP, part, rec, ur);
    else k_mom_prep_mixed<false><<<grid, dim3(32, 8), 0, st>>>(p, x, oth, pf, AP, part, rec, ur);
    SGPU_LAUNCH();
    return static_cast<int>(grid.x * grid.y);
}

dim3 assemble_grid(const DevParams& p) {
    return dim3((pair_count(p) + 31) / 32, (p.NX + 8 * kAsmRows - 1) / (8 * kAsmRows));
}

int launch_assemble_p_mixed(const DevParams& p, const double* APU, const double* APV, const double* u,
                            const double* v, double* bfield, const LevelView32& L0, double* part,
                            cudaStream_t st) {
    const dim3 grid = assemble_grid(p);
    k_assemble_p_mixed<<<grid, dim3(32, 8), 0, st>>>(p, APU, APV, u, v, bfield, L0, part);
    SGPU_LAUNCH();
    return static_cast<int>(grid.x * grid.y);
}

int mixed_partials(const DevParams& p) {
    // the prep's blocks (one partial each: 32 columns x kTileRows rows over the update range, at most
    // NY + 1 columns and NX rows), the defect-correction update's (two each: 32 x kTileRows cells)
    // and assemble_p's (two each)
    const int prep = ((p.NY + 1 + 31) / 32) * ((p.NX + kTileRows - 1) / kTileRows);
    const int dc = 2 * ((p.NY + 31) / 32) * ((p.NX + kTileRows - 1) / kTileRows);
    const dim3 g = assemble_grid(p);
    return std::max({prep, dc, static_cast<int>(2 * g.x * g.y)});
}

void launch_b_to_f32(const DevParams& p, const double* bfield, const double* sum_b,
                     const LevelView32& L0, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + kTileRows - 1) / kTileRows);
    k_b_to_f32<<<grid, dim3(32, 8), 0, st>>>(p, bfield, sum_b, L0);
    SGPU_LAUNCH();
}

void launch_pc_from32(const DevParams& p, const LevelView32& L0, const double* sum_pc, double* pc64,
                      cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + 7) / 8);
    k_pc_from32<<<grid, dim3(32, 8), 0, st>>>(p, L0.x, L0.stride, sum_pc, pc64);
    SGPU_LAUNCH();
}

int launch_dc_rhs0(const DevParams& p, const double* bfield, const double* sum_b, const LevelView32& L0,
                   double* part, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + kTileRows - 1) / kTileRows);
    k_dc_rhs0<<<grid, dim3(32, 8), 0, st>>>(p, bfield, sum_b, L0, part);
    SGPU_LAUNCH();
    return static_cast<int>(grid.x * grid.y);
}

int launch_dc_update(const DevParams& p, const double* APU, const double* APV, const double* bfield,
                     const double* sum_b, const LevelView32& L0, const double* pold, double* pnew, bool first,
                     double* part, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + kTileRows - 1) / kTileRows);
    k_dc_update<<<grid, dim3(32, 8), 0, st>>>(p, APU, APV, bfield, sum_b, L0.x, L0.stride, pold, pnew,
                                               first ? 1 : 0, L0, part);
    SGPU_LAUNCH();
    return static_cast<int>(grid.x * grid.y);
}

void launch_correct_dc(const DevParams& p, const double* pc64, const double* sum_pc, const double* APU,
                       const double* APV, double* u, double* v, double* pf, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + 7) / 8);
    k_correct_dc<<<grid, dim3(32, 8), 0, st>>>(p, pc64, sum_pc, APU, APV, u, v, pf);
    SGPU_LAUNCH();
}

void launch_pc_from64(const DevParams& p, const double* src, const double* sum_pc, double* dst, cudaStream_t st) {
    const dim3 grid((p.NY + 31) / 32, (p.NX + 7) / 8);
    k_pc_from64<<<grid, dim3(32, 8), 0, st>>>(p, src, sum_pc, dst);
    SGPU_LAUNCH();
}

void launch_correct_mixed(const DevParams& p, const LevelView32& L0, const double* sum_pc,
                          const double* APU, const double* APV, double* u, double* v, double* pf,
                          cudaStream_t st) {
    const dim3 grid((pair_count(p) + 31) / 32, (p.NX + 7) / 8);
    k_correct_mixed<<<grid, dim3(32, 8), 0, st>>>(p, L0.x, L0.stride, sum_pc, APU, APV, u, v, pf);
    SGPU_LAUNCH();
}

#else
void launch_corr_sweep(const DevParams& p, bool v_component, const float* ein, float* eout,
                       MomRec32 rec, bool e_zero, int seg_rows, unsigned* err, cudaStream_t st,
                       double* xfinal) {
    if (p.ncol == 5) {
        if (v_component) launch_corr_m<5, true>(p, ein, eout, rec, e_zero, seg_rows, xfinal, err, st);
        else launch_corr_m<5, false>(p, ein, eout, rec, e_zero, seg_rows, xfinal, err, st);
    } else {
        if (v_component) launch_corr_m<2, true>(p, ein, eout, rec, e_zero, seg_rows, xfinal, err, st);
        else launch_corr_m<2, false>(p, ein, eout, rec, e_zero, seg_rows, xfinal, err, st);
    }
}

bool launch_corr_cluster(const DevParams& p, bool v_component, MomRec32 rec, int nsweeps, double* x,
                         cudaStream_t st) {
    CorrClusterPlan pl{};
    if (nsweeps < 1 || !corr_cluster_available() || !corr_cluster_plan(p, v_component, pl)) return false;
    if (p.ncol == 5) {
        if (v_component) launch_corr_cluster_t<5, true>(p, rec, pl, nsweeps, x, st);
        else launch_corr_cluster_t<5, false>(p, rec, pl, nsweeps, x, st);
    } else {
        if (v_component) launch_corr_cluster_t<2, true>(p, rec, pl, nsweeps, x, st);
        else launch_corr_cluster_t<2, false>(p, rec, pl, nsweeps, x, st);
    }
    return true;
}

void init_mixed_kernels() {
#define SGPU_SMEM(NC, V)                                                                               \
    SGPU_CUDA(cudaFuncSetAttribute(k_corr_stream<NC, V, kCorrNT, kCorrMinb>,                           \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, CorrSmem<NC, kCorrNT>::bytes))
    SGPU_SMEM(5, false); SGPU_SMEM(5, true); SGPU_SMEM(2, false); SGPU_SMEM(2, true);
#undef SGPU_SMEM
}

int corr_threads() { return kCorrNT; }

void launch_wait_selftest(int polls, unsigned* err, cudaStream_t st) {
    k_wait_selftest<<<1, 32, 0, st>>>(polls, err);
    SGPU_LAUNCH();
}

int corr_blocks_per_sm(int ncol) {
    const int smem = ncol == 5 ? CorrSmem<5, kCorrNT>::bytes : CorrSmem<2, kCorrNT>::bytes;
    int n = 0;
    if (ncol == 5)
        SGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_corr_stream<5, false, kCorrNT, kCorrMinb>,
                                                                kCorrNT, smem));
    else
        SGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_corr_stream<2, false, kCorrNT, kCorrMinb>,
                                                                kCorrNT, smem));
    return n > 0 ? n : 1;
}

#endif

} // namespace sgpu
