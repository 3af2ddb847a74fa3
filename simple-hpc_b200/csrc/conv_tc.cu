// conv_tc.cu — the warm-start network's 3x3 convolutions on the Blackwell tensor cores (tcgen05).
//
// Implicit GEMM: Y[p, co] = sum over taps t and input channels ci of X[p + t, ci] W[co, t, ci], with
// M = 128 pixels per CTA (the accumulator's 128 TMEM lanes), N = Cout (16 .. 256, FP32 accumulator
// columns in TMEM) and K = 9 taps x Cin, walked in stages of one tap and Kc <= 64 input channels.
//  * Operands. All 128 threads stage a stage's A tile (128 pixels x Kc channels, zero where the tap
//    falls outside the image) and B tile (N output channels x Kc) into shared memory with 16-byte
//    loads, in the canonical K-major layout without swizzling: 8 x 16-byte core matrices, the rows
//    of a core matrix contiguous, core matrices adjacent in K 128 bytes apart (leading byte offset)
//    and groups of 8 rows Kc x 16 bytes apart (stride byte offset). Two stage buffers alternate.
//  * MMA. Thread 0 issues Kc / 16 `tcgen05.mma.cta_group::1.kind::f16` (BF16 x BF16 -> FP32,
//    K = 16 each) per stage and commits them to that buffer's mbarrier; the buffer is refilled only
//    after that commit has arrived, so loads of stage s + 1 overlap the MMAs of stage s.
//  * Epilogue. After the last commit, warp w reads TMEM lanes 32w .. 32w + 31 (its pixels) with
//    `tcgen05.ld.32x32b`, adds the bias, applies ReLU and stores BF16.
// Every mbarrier wait is bounded: a give-up sets *err, no further MMA is issued, outstanding commits
// are waited for (bounded again), TMEM is freed and the CTA returns. The input-gradient pass is the
// same kernel on the output gradient with flipped weights.
#include "cnn.hpp"

#include <algorithm>
#include <cstdint>

namespace sgpu {

namespace {

using bf16 = __nv_bfloat16;

constexpr int kM = 128;          // pixels per CTA = accumulator rows = TMEM lanes
constexpr int kThreadsTc = 128;  // 4 warps: warp w owns TMEM lanes 32w .. 32w + 31
constexpr int kSpinTc = 1 << 22; // mbarrier polls before a wait gives up

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool bar_test(uint64_t* b, unsigned parity) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_addr(b)), "r"(parity)
                 : "memory");
    return done != 0;
}
// Bounded wait for phase `parity` of b; false (and *err set) on a give-up.
__device__ __forceinline__ bool bar_wait(uint64_t* b, unsigned parity, unsigned* err) {
    for (int it = 0; !bar_test(b, parity); ++it)
        if (it >= kSpinTc) {
            atomicOr(err, 2u);
            return false;
        }
    return true;
}

// Shared-memory matrix descriptor (tcgen05): start address, leading and stride byte offsets (all
// >> 4), the fixed field 0b001 at bits 46-48, base offset 0, no swizzling.
__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N and M.
__host__ __device__ constexpr uint32_t instr_desc(int n, int m) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_addr(b))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor cores' (async proxy) reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 16 FP32 accumulator columns [col, col + 16) of this warp's 32 TMEM lanes: lane i of the warp gets
// row 32 (warp % 4) + i.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                 "%12, %13, %14, %15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Byte offset of row r, 8-channel group g in a K-major no-swizzle tile of Kc channels per row.
__device__ __forceinline__ unsigned core_off(int r, int g, int kc) {
    return static_cast<unsigned>((r >> 3) * (kc * 16) + g * 128 + (r & 7) * 16);
}

// 16-byte asynchronous copy global -> shared; src_bytes 0 writes zeros (no global read).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, unsigned src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stage shape of the forward kernel: kc input channels of nt taps (K = nt kc <= 144 per stage).
struct ConvStages {
    int kc, nt, chunks, tgroups, stages, nbuf, kmax;
};

// 3x3 convolution, zero padding 1: X [N*H*W][Cin] -> Y [N*H*W][Cout] (+ bias, ReLU if relu).
// A stage covers taps [t0, t0 + nt_s) and channels [c0, c0 + kc): K index (local tap, channel) in
// that order, so a weight row's stage slice is contiguous when kc = Cin. Its A and B tiles are copied
// with cp.async (zero-fill where the tap leaves the image) nbuf - 1 stages ahead into a ring of nbuf
// buffers; a buffer is refilled after the MMAs that read it have committed.
__global__ void __launch_bounds__(kThreadsTc)
    k_conv_tc(const bf16* __restrict__ X, int N, int H, int W, int Cin, const bf16* __restrict__ Wt,
              const float* __restrict__ bias, bf16* __restrict__ Y, int Cout, int relu, ConvStages cs,
              uint32_t tmem_cols, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[4];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const unsigned a_bytes = kM * cs.kmax * 2, b_bytes = static_cast<unsigned>(Cout) * cs.kmax * 2;
    auto a_buf = [&](int b) { return smem + b * (a_bytes + b_bytes); };
    auto b_buf = [&](int b) { return smem + b * (a_bytes + b_bytes) + a_bytes; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_addr(&tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < 4; ++k) bar_init(&bars[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    // This thread's pixel (A row) and its coordinates.
    const long npix = static_cast<long>(N) * H * W;
    const long p = static_cast<long>(blockIdx.x) * kM + tid;
    const bool live = p < npix;
    const long q = live ? p : 0;
    const int px = static_cast<int>(q % W), py = static_cast<int>((q / W) % H);
    const long pn = q / (static_cast<long>(W) * H);
    const int gk = cs.kc / 8; // 16-byte groups per tap and stage

    // stage s: channel chunk s / tgroups, taps [t0, t0 + nt_s)
    auto stage_taps = [&](int s, int& t0, int& c0) {
        const int tg = s % cs.tgroups;
        c0 = (s / cs.tgroups) * cs.kc;
        t0 = tg * cs.nt;
        return min(cs.nt, 9 - t0);
    };
    auto issue = [&](int s) {
        if (s < cs.stages) {
            int t0, c0;
            const int nts = stage_taps(s, t0, c0);
            const int kst = nts * cs.kc;
            unsigned char* ab = a_buf(s % cs.nbuf);
            unsigned char* bb = b_buf(s % cs.nbuf);
            for (int tl = 0; tl < nts; ++tl) {
                const int t = t0 + tl;
                const int ys = py + t / 3 - 1, xs = px + t % 3 - 1;
                const bool in = live && ys >= 0 && ys < H && xs >= 0 && xs < W;
                const bf16* src = in ? X + ((pn * H + ys) * W + xs) * Cin + c0 : X;
                for (int g = 0; g < gk; ++g)
                    cp_async16(ab + core_off(tid, tl * gk + g, kst), src + 8 * g, in ? 16u : 0u);
            }
            for (int co = tid; co < Cout; co += kThreadsTc)
                for (int tl = 0; tl < nts; ++tl) {
                    const bf16* w = Wt + (static_cast<long>(co) * 9 + t0 + tl) * Cin + c0;
                    for (int g = 0; g < gk; ++g) cp_async16(bb + core_off(co, tl * gk + g, kst), w + 8 * g, 16u);
                }
        }
        cp_async_commit(); // one group per stage slot, empty past the last stage
    };

    const uint32_t idesc = instr_desc(Cout, kM);
    bool gave_up = false;
    int issued = 0; // stages whose MMAs thread 0 committed
    for (int s = 0; s < cs.nbuf - 1; ++s) issue(s);
    for (int s = 0; s < cs.stages; ++s) {
        const int b = s % cs.nbuf;
        // this thread's copies of stage s have landed (the groups of later stages may still fly)
        if (cs.nbuf == 3) cp_async_wait<1>();
        else cp_async_wait<0>();
        fence_async_smem();
        if (__syncthreads_or(gave_up ? 1 : 0)) {
            gave_up = true;
            break;
        }
        if (tid == 0) {
            fence_after();
            int t0, c0;
            const int kst = stage_taps(s, t0, c0) * cs.kc;
            const unsigned a0 = smem_addr(a_buf(b)), b0 = smem_addr(b_buf(b));
            for (int k = 0; k < kst / 16; ++k) {
                const uint64_t ad = smem_desc(a0 + 256u * k, 128u, static_cast<unsigned>(kst) * 16u);
                const uint64_t bd = smem_desc(b0 + 256u * k, 128u, static_cast<unsigned>(kst) * 16u);
                mma_issue(tmem, ad, bd, idesc, (s > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(&bars[b]);
        }
        issued = s + 1;
        // refill the buffer stage s - 1 used, once its MMAs have committed
        const int nxt = s + cs.nbuf - 1;
        if (nxt < cs.stages && s >= 1) {
            const int pb = (s - 1) % cs.nbuf;
            if (!bar_wait(&bars[pb], static_cast<unsigned>(((s - 1) / cs.nbuf) & 1), err)) gave_up = true;
        }
        if (!gave_up) issue(nxt);
        else cp_async_commit();
    }
    cp_async_wait<0>();

    // The last commit covers every MMA before it.
    if (issued > 0 && !gave_up) {
        const int s = issued - 1;
        if (!bar_wait(&bars[s % cs.nbuf], static_cast<unsigned>((s / cs.nbuf) & 1), err)) gave_up = true;
    }
    if (__syncthreads_or(gave_up ? 1 : 0)) {
        // Drain: wait (bounded) for the commits still outstanding, so no MMA writes TMEM or reads
        // shared memory after the CTA frees them. Stage s's commit is phase s / nbuf of buffer s % nbuf.
        if (tid == 0)
            for (int s = issued - 1; s >= 0 && s >= issued - cs.nbuf; --s)
                bar_wait(&bars[s % cs.nbuf], static_cast<unsigned>((s / cs.nbuf) & 1), err);
    } else {
        fence_after();
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        for (int c0 = 0; c0 < Cout; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + static_cast<uint32_t>(c0), v);
            if (live) {
                uint32_t packed[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    float v0 = v[2 * k] + (bias ? bias[c0 + 2 * k] : 0.0f);
                    float v1 = v[2 * k + 1] + (bias ? bias[c0 + 2 * k + 1] : 0.0f);
                    if (relu) {
                        v0 = fmaxf(v0, 0.0f);
                        v1 = fmaxf(v1, 0.0f);
                    }
                    const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
                    packed[k] = *reinterpret_cast<const uint32_t*>(&h);
                }
                uint4* dst = reinterpret_cast<uint4*>(Y + p * Cout + c0);
                dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols)
                     : "memory");
}

// Weight gradient of a 3x3 convolution: dW[co, t, ci] += sum over pixels p of dZ[p, co] X[p + t, ci],
// for the taps t0 .. t0 + nt - 1 of this CTA (blockIdx.y) and its chunk of `chunk` pixels
// (blockIdx.x). GEMM with M = 128 (output channels co < Cout, the rest zero rows), N = nt x Cin
// (column (t, ci)), K = pixels in stages of kWgPix. Both operands are gathered from the NHWC arrays
// into the K-major core-matrix layout: a thread takes two consecutive pixels of 8 channels (two
// 16-byte loads) and writes the 8 channel rows' (p, p + 1) pairs as 4-byte stores. The chunk's
// result is added into the FP32 dW with atomics (as many adds per weight as pixel chunks).
constexpr int kWgPix = 32; // pixels (K) per stage: two MMAs of K = 16

__global__ void __launch_bounds__(kThreadsTc)
    k_conv_wgrad_tc(const bf16* __restrict__ X, const bf16* __restrict__ dZ, int N, int H, int W, int Cin,
                    int Cout, int taps_per_cta, float* __restrict__ dW, int chunk, uint32_t tmem_cols,
                    unsigned* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int t0 = blockIdx.y * taps_per_cta;
    const int nt = min(taps_per_cta, 9 - t0);
    const int ncols = nt * Cin; // N
    const unsigned a_bytes = kM * kWgPix * 2, b_bytes = static_cast<unsigned>(ncols) * kWgPix * 2;
    unsigned char* a_buf[2] = {smem, smem + a_bytes};
    unsigned char* b_buf[2] = {smem + 2 * a_bytes, smem + 2 * a_bytes + b_bytes};

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_addr(&tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        bar_init(&bars[0], 1);
        bar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // Rows co >= Cout of both A buffers stay zero: clear both A buffers once.
    for (unsigned o = tid * 16u; o < 2 * a_bytes; o += kThreadsTc * 16u)
        *reinterpret_cast<uint4*>(smem + o) = make_uint4(0u, 0u, 0u, 0u);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    const long npix = static_cast<long>(N) * H * W;
    const long pbeg = static_cast<long>(blockIdx.x) * chunk;
    const long pend = min(npix, pbeg + chunk);
    const int stages = static_cast<int>((pend - pbeg + kWgPix - 1) / kWgPix);
    const uint32_t idesc = instr_desc(ncols, kM);
    const int co_groups = Cout / 8, ci_groups = Cin / 8;
    bool gave_up = false;
    int issued = 0;
    // a 16-byte group of 8 channels of pixel p (zero past the chunk), and of the pixel tap t away
    auto zload = [&](long p, int g) -> uint4 {
        return p < pend ? __ldg(reinterpret_cast<const uint4*>(dZ + p * Cout) + g) : make_uint4(0u, 0u, 0u, 0u);
    };
    auto xload = [&](long p, int t, int g) -> uint4 {
        if (p >= pend) return make_uint4(0u, 0u, 0u, 0u);
        const int x = static_cast<int>(p % W), y = static_cast<int>((p / W) % H);
        const long n = p / (static_cast<long>(W) * H);
        const int ys = y + t / 3 - 1, xs = x + t % 3 - 1;
        if (ys < 0 || ys >= H || xs < 0 || xs >= W) return make_uint4(0u, 0u, 0u, 0u);
        return __ldg(reinterpret_cast<const uint4*>(X + ((n * H + ys) * W + xs) * Cin) + g);
    };
    // the pair (k, k + 1) of 8 rows r0 .. r0 + 7 from two 8-channel groups lo (pixel k), hi (k + 1)
    auto scatter = [&](unsigned char* buf, int r0, int k, uint4 lo, uint4 hi) {
        const uint32_t l[4] = {lo.x, lo.y, lo.z, lo.w}, h[4] = {hi.x, hi.y, hi.z, hi.w};
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t a = (l[e >> 1] >> (16 * (e & 1))) & 0xFFFFu;
            const uint32_t b = (h[e >> 1] >> (16 * (e & 1))) & 0xFFFFu;
            *reinterpret_cast<uint32_t*>(buf + core_off(r0 + e, k >> 3, kWgPix) + (k & 7) * 2) = a | (b << 16);
        }
    };

    for (int s = 0; s < stages; ++s) {
        const int b = s & 1;
        if (s >= 2 && !bar_wait(&bars[b], static_cast<unsigned>(((s - 2) >> 1) & 1), err)) gave_up = true;
        if (!gave_up) {
            const long p0 = pbeg + static_cast<long>(s) * kWgPix;
            // A: (k pair, co group) units
            for (int u = tid; u < (kWgPix / 2) * co_groups; u += kThreadsTc) {
                const int k = 2 * (u % (kWgPix / 2)), g = u / (kWgPix / 2);
                scatter(a_buf[b], 8 * g, k, zload(p0 + k, g), zload(p0 + k + 1, g));
            }
            // B: (k pair, tap, ci group) units
            for (int u = tid; u < (kWgPix / 2) * nt * ci_groups; u += kThreadsTc) {
                const int k = 2 * (u % (kWgPix / 2)), rest = u / (kWgPix / 2);
                const int g = rest % ci_groups, t = rest / ci_groups;
                scatter(b_buf[b], t * Cin + 8 * g, k, xload(p0 + k, t0 + t, g), xload(p0 + k + 1, t0 + t, g));
            }
        }
        fence_async_smem();
        if (__syncthreads_or(gave_up ? 1 : 0)) {
            gave_up = true;
            break;
        }
        if (tid == 0) {
            fence_after();
            const unsigned a0 = smem_addr(a_buf[b]), b0 = smem_addr(b_buf[b]);
#pragma unroll
            for (int k = 0; k < kWgPix / 16; ++k) {
                const uint64_t ad = smem_desc(a0 + 256u * k, 128u, kWgPix * 16u);
                const uint64_t bd = smem_desc(b0 + 256u * k, 128u, kWgPix * 16u);
                mma_issue(tmem, ad, bd, idesc, (s > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(&bars[b]);
        }
        issued = s + 1;
    }
    if (issued > 0 && !gave_up) {
        const int s = issued - 1;
        if (!bar_wait(&bars[s & 1], static_cast<unsigned>((s >> 1) & 1), err)) gave_up = true;
    }
    if (__syncthreads_or(gave_up ? 1 : 0)) {
        if (tid == 0)
            for (int s = issued - 1; s >= 0 && s >= issued - 2; --s)
                bar_wait(&bars[s & 1], static_cast<unsigned>((s >> 1) & 1), err);
    } else if (issued > 0) {
        fence_after();
        const int co = warp * 32 + (tid & 31);
        const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
        for (int c0 = 0; c0 < ncols; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + static_cast<uint32_t>(c0), v);
            if (co < Cout) {
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int col = c0 + e, t = t0 + col / Cin, ci = col % Cin;
                    atomicAdd(dW + (static_cast<long>(co) * 9 + t) * Cin + ci, v[e]);
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols)
                     : "memory");
}

// Kernel shared memory available for the stage ring (one CTA's share of an SM).
constexpr int kConvSmemMax = 200 * 1024;

// Stages of the forward kernel: kc = Cin (or the largest multiple of 16 dividing it that is <= 128),
// nt = the taps that keep K = nt kc <= 144, and as many buffers (2 or 3) as the ring allows.
ConvStages conv_stages(int cin, int cout) {
    ConvStages c{};
    c.kc = cin;
    if (c.kc > 128)
        for (int k = 128; k >= 16; k -= 16)
            if (cin % k == 0) {
                c.kc = k;
                break;
            }
    c.nt = std::max(1, std::min(9, 144 / c.kc));
    c.chunks = cin / c.kc;
    c.tgroups = (9 + c.nt - 1) / c.nt;
    c.stages = c.chunks * c.tgroups;
    c.kmax = c.nt * c.kc;
    const int per = (kM + cout) * c.kmax * 2;
    c.nbuf = std::min(3, std::max(2, kConvSmemMax / per));
    if (c.stages < c.nbuf) c.nbuf = std::max(2, c.stages);
    return c;
}

} // namespace

void launch_conv_wgrad_tc(const bf16* X, const bf16* dZ, int N, int H, int W, int Cin, int Cout, float* dW,
                          unsigned* err, cudaStream_t st) {
    if (Cin < 16 || Cin > 256 || Cin % 16 || Cout < 16 || Cout > kM || Cout % 16 || !err)
        throw Error(SGPU_E_INVALID, "tensor-core weight gradient: channels must be multiples of 16, Cout <= 128");
    const auto misaligned = [](const void* q) { return (reinterpret_cast<std::uintptr_t>(q) & 15u) != 0; };
    if (misaligned(X) || misaligned(dZ))
        throw Error(SGPU_E_INVALID, "tensor-core weight gradient: operands must be 16-byte aligned");
    const long npix = static_cast<long>(N) * H * W;
    if (npix <= 0) return;
    const int taps = std::min(9, std::max(1, 256 / Cin)); // N = taps x Cin <= 256
    int ncols_max = taps * Cin;
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(ncols_max)) cols <<= 1;
    const int chunk = 4096;
    const int smem = 2 * (kM * kWgPix * 2) + 2 * (ncols_max * kWgPix * 2);
    static PerDeviceOnce attr;
    attr.get([] {
        SGPU_CUDA(cudaFuncSetAttribute(k_conv_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * (kM * kWgPix * 2) + 2 * (256 * kWgPix * 2)));
        return 0;
    });
    const dim3 grid(static_cast<unsigned>((npix + chunk - 1) / chunk), static_cast<unsigned>((9 + taps - 1) / taps));
    k_conv_wgrad_tc<<<grid, kThreadsTc, smem, st>>>(X, dZ, N, H, W, Cin, Cout, taps, dW, chunk, cols, err);
    SGPU_LAUNCH();
}

void launch_conv_tc(const bf16* X, int N, int H, int W, int Cin, const bf16* Wt, const float* bias, bf16* Y,
                    int Cout, int relu, unsigned* err, cudaStream_t st) {
    if (Cin < 16 || Cin % 16 || Cout < 16 || Cout > 256 || Cout % 16 || !err)
        throw Error(SGPU_E_INVALID, "tensor-core convolution: channels must be multiples of 16, Cout <= 256");
    const auto misaligned = [](const void* q) { return (reinterpret_cast<std::uintptr_t>(q) & 15u) != 0; };
    if (misaligned(X) || misaligned(Wt) || misaligned(Y))
        throw Error(SGPU_E_INVALID, "tensor-core convolution: operands must be 16-byte aligned");
    const long npix = static_cast<long>(N) * H * W;
    if (npix <= 0) return;
    const ConvStages cs = conv_stages(Cin, Cout);
    // buffers a launch actually fills: a one-stage layer (Cin = 16: all 9 taps at once) uses one
    const int smem = std::min(cs.nbuf, cs.stages) * (kM + Cout) * cs.kmax * 2;
    if (smem > kConvSmemMax)
        throw Error(SGPU_E_INVALID, "tensor-core convolution: stage ring exceeds shared memory");
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(Cout)) cols <<= 1;
    static PerDeviceOnce attr;
    attr.get([] {
        SGPU_CUDA(cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmemMax));
        return 0;
    });
    const unsigned grid = static_cast<unsigned>((npix + kM - 1) / kM);
    k_conv_tc<<<grid, kThreadsTc, smem, st>>>(X, N, H, W, Cin, Wt, bias, Y, Cout, relu, cs, cols, err);
    SGPU_LAUNCH();
}

} // namespace sgpu
