// reduce.cu — ordered (bit-reproducible) sums on the device.
//
// The reference sums a per-cell quantity by adding each row left to right from 0.0 and then the
// row sums top to bottom from 0.0 (CellSums::sum and add_rows, src/decomp.cpp:176-205; det_sum,
// src/multigrid.cpp:18-34). Floating-point addition is not associative, so the same bits need the
// same chain: one dependent chain per row, then one chain over the rows.
//
// One lane per row: a warp owns 32 rows and streams them through a ring of 32 x 32 tiles in shared
// memory, filled by cp.async many tiles ahead; each lane then adds its row's 32 values of a tile in
// column order. A tile costs a lane 32 shared loads and 32 adds for 32 rows' worth of data, so the
// kernel is bound by the memory stream and the add latency, not by instruction issue. The last CTA
// to finish adds the row sums in row order. Inputs may be FP64 or FP32 (widened to FP64 when
// added); the sums are FP64.
#include "kernels.hpp"
#include "blocksum.cuh"

#include <algorithm>

namespace sgpu {

namespace {

constexpr int kTile = 32;   // columns per tile (and rows per warp)
constexpr int kStages = 12; // tiles in flight per warp (the standalone sum)
constexpr int kLeanStages = 3; // the lean variant: little shared memory, to run beside other kernels
constexpr int kPitch = kTile + 1; // padded tile row: lanes reading one column hit distinct banks

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

// One warp per CTA (32 rows); the grid covers ceil(nr / 32) x K planes. PAIR: one plane, two sums
// in one pass (out[0] = sum of |v|, out[1] = sum of v, each in the same order).
template <class TIn, int STAGES, bool PAIR>
__global__ void __launch_bounds__(32)
    k_ordered_sum(const TIn* __restrict__ vals, std::size_t plane_stride, int ld, int nr, int nc,
                  double* __restrict__ rows, unsigned int* counter, double* __restrict__ out,
                  const int* skip, int chunk) {
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char tile_raw[];
    TIn(*tile)[kTile][kPitch] = reinterpret_cast<TIn(*)[kTile][kPitch]>(tile_raw);
    __shared__ bool last_block;
    const int m = blockIdx.y;
    const int lane = threadIdx.x;
    const int r0 = blockIdx.x * kTile;
    const int nrow = min(kTile, nr - r0);
    const TIn* src = vals + m * plane_stride + static_cast<std::size_t>(r0) * ld;
    const int ntiles = (nc + kTile - 1) / kTile;

    // Tile k: rows r0 .. r0 + 31, columns 32k .. 32k + 31; lane = column while loading.
    auto issue = [&](int k) {
        if (k < ntiles) {
            const int c = k * kTile + lane;
            if (c < nc)
                for (int rr = 0; rr < nrow; ++rr)
                    cp_async(&tile[k % STAGES][rr][lane], src + static_cast<std::size_t>(rr) * ld + c);
        }
        cp_async_commit();
    };
    for (int k = 0; k < STAGES - 1; ++k) issue(k);

    double s = 0.0;  // this lane's row: r0 + lane
    double sa = 0.0; // PAIR: the sum of |v| of the same row
    for (int k = 0; k < ntiles; ++k) {
        issue(k + STAGES - 1);
        cp_async_wait<STAGES - 1>(); // tile k has landed (this lane's copies)
        __syncwarp();                 // ... and everyone's
        const int cnt = min(kTile, nc - k * kTile);
        const TIn* t = tile[k % STAGES][lane];
        if (cnt == kTile) {
            double v[kTile];
#pragma unroll
            for (int c = 0; c < kTile; ++c) v[c] = static_cast<double>(t[c]); // loads first
#pragma unroll
            for (int c = 0; c < kTile; ++c) {
                s += v[c];
                if (PAIR) sa += fabs(v[c]);
            }
        } else {
            for (int c = 0; c < cnt; ++c) {
                const double x = static_cast<double>(t[c]);
                s += x;
                if (PAIR) sa += fabs(x);
            }
        }
        __syncwarp(); // the slot is refilled by the next issue
    }
    cp_async_wait<0>();
    if (lane < nrow) {
        if (PAIR) {
            rows[r0 + lane] = sa;
            rows[static_cast<std::size_t>(nr) + r0 + lane] = s;
        } else {
            rows[static_cast<std::size_t>(m) * nr + r0 + lane] = s;
        }
    }

    // The last CTA to finish adds every plane's row sums in row order.
    __threadfence();
    __syncwarp();
    if (lane == 0) {
        const unsigned int total = gridDim.x * gridDim.y;
        last_block = (atomicAdd(counter, 1u) == total - 1);
    }
    __syncwarp();
    if (!last_block) return;
    __threadfence();
    // The chain over the rows is serial, so it must not wait on L2 for each term: the warp stages
    // chunks of every plane's row sums in shared memory (the tile ring is free now; many
    // independent loads per lane in flight), then lane m adds plane m's chunk from registers.
    const int K = PAIR ? 2 : static_cast<int>(gridDim.y);
    double* buf = reinterpret_cast<double*>(tile_raw);
    const int cs = chunk + 1; // plane stride in buf: lanes reading one row index hit distinct banks
    double acc = 0.0;
    for (int c0 = 0; c0 < nr; c0 += chunk) {
        const int n = min(chunk, nr - c0);
        __syncwarp();
        for (int m2 = 0; m2 < K; ++m2) {
            const double* rs = rows + static_cast<std::size_t>(m2) * nr + c0;
#pragma unroll 16
            for (int r = lane; r < n; r += kTile) buf[m2 * cs + r] = __ldcg(rs + r); // L2: other CTAs wrote them
        }
        __syncwarp();
        if (lane < K) {
            const double* b = buf + lane * cs;
            int r = 0;
            for (; r + kTile <= n; r += kTile) {
                double v[kTile];
#pragma unroll
                for (int t = 0; t < kTile; ++t) v[t] = b[r + t];
#pragma unroll
                for (int t = 0; t < kTile; ++t) acc += v[t];
            }
            for (; r < n; ++r) acc += b[r];
        }
    }
    if (lane < K) out[lane] = acc;
    if (lane == 0) *counter = 0u; // ready for the next launch on this stream
}

template <class TIn, int STAGES, bool PAIR = false>
void launch_sum(const TIn* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                double* out, const SumScratch& s, const int* skip, cudaStream_t st) {
    const int kout = PAIR ? 2 : K;
    if (K < 1 || K > 32 || kout > s.max_k || nr > s.max_rows || (PAIR && K != 1))
        throw Error(SGPU_E_INVALID, "ordered sum: sizes exceed the scratch");
    if (nr <= 0) {
        SGPU_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * kout, st));
        return;
    }
    const dim3 grid((nr + kTile - 1) / kTile, K);
    constexpr int smem = STAGES * kTile * kPitch * static_cast<int>(sizeof(TIn));
    static PerDeviceOnce attr; // the attribute lives in each device's context
    attr.get([] {
        SGPU_CUDA(cudaFuncSetAttribute(k_ordered_sum<TIn, STAGES, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return 0;
    });
    // Rows per staged chunk of the final pass: K planes of (chunk + 1) doubles fit the tile ring.
    const int chunk = std::min(2048, (smem / (static_cast<int>(sizeof(double)) * kout) - 1) / kTile * kTile);
    k_ordered_sum<TIn, STAGES, PAIR><<<grid, 32, smem, st>>>(vals, plane_stride, ld, nr, nc, s.rows, s.counter,
                                                              out, skip, chunk);
    SGPU_LAUNCH();
}

// ---- deterministic FP64 tree sums (the mixed-precision path) ----

// out_k = the sum of the n partial sums of plane k (block k): thread t adds values t, t + 1024, ...
// in order, then the block tree.
__global__ void __launch_bounds__(1024)
    k_sum_partials(const double* __restrict__ part, int n, int plane, double* out0, double* out1) {
    __shared__ double s[32];
    const double* src = part + static_cast<std::size_t>(blockIdx.x) * plane;
    double a = 0.0;
#pragma unroll 8
    for (int i = static_cast<int>(threadIdx.x); i < n; i += 1024) a += src[i];
    const double t = block_sum<32>(a, s, static_cast<int>(threadIdx.x));
    if (threadIdx.x == 0) *(blockIdx.x == 0 ? out0 : out1) = t;
}

constexpr int kTileRows = 32; // rows per block of k_tile_sum

// Block (bx, by) of an nr x nc array (row stride ld): columns 256 bx .. +255, rows 32 by .. +31.
// Each thread adds its column's values top to bottom in FP64, then the block tree; one partial sum
// per block.
template <class T>
__global__ void __launch_bounds__(256)
    k_tile_sum(const T* __restrict__ vals, int ld, int nr, int nc, double* __restrict__ part) {
    __shared__ double s[8];
    const int c = static_cast<int>(blockIdx.x * 256 + threadIdx.x);
    const int r0 = static_cast<int>(blockIdx.y) * kTileRows, r1 = min(r0 + kTileRows, nr);
    double a = 0.0;
    if (c < nc) {
        const T* src = vals + static_cast<std::size_t>(r0) * ld + c;
#pragma unroll 8
        for (int r = r0; r < r1; ++r, src += ld) a += static_cast<double>(*src);
    }
    const double t = block_sum<8>(a, s, static_cast<int>(threadIdx.x));
    if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = t;
}

} // namespace

void launch_sum_partials(const double* part, int n, int K, int plane, double* out0, double* out1,
                         cudaStream_t st) {
    if (K < 1 || K > 2 || (K == 2 && !out1)) throw Error(SGPU_E_INVALID, "partial sums: 1 or 2 planes");
    k_sum_partials<<<K, 1024, 0, st>>>(part, n, plane, out0, out1);
    SGPU_LAUNCH();
}

int tree_sum_partials(int nr, int nc) {
    return ((nc + 255) / 256) * ((nr + kTileRows - 1) / kTileRows);
}

void launch_tree_sum(const float* vals, int ld, int nr, int nc, double* part, double* out, cudaStream_t st) {
    if (nr <= 0 || nc <= 0) {
        SGPU_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
        return;
    }
    const dim3 grid((nc + 255) / 256, (nr + kTileRows - 1) / kTileRows);
    k_tile_sum<float><<<grid, 256, 0, st>>>(vals, ld, nr, nc, part);
    SGPU_LAUNCH();
    launch_sum_partials(part, static_cast<int>(grid.x * grid.y), 1, 0, out, nullptr, st);
}

void launch_ordered_sum(const double* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                        double* out, const SumScratch& s, const int* skip, cudaStream_t st) {
    launch_sum<double, kStages>(vals, plane_stride, ld, nr, nc, K, out, s, skip, st);
}

void launch_ordered_sum(const float* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                        double* out, const SumScratch& s, const int* skip, cudaStream_t st) {
    launch_sum<float, kStages>(vals, plane_stride, ld, nr, nc, K, out, s, skip, st);
}

void launch_ordered_sum_abs_pair(const double* vals, int ld, int nr, int nc, double* out, const SumScratch& s,
                                 cudaStream_t st) {
    launch_sum<double, kStages, true>(vals, 0, ld, nr, nc, 1, out, s, nullptr, st);
}

void launch_ordered_sum_lean(const double* vals, int ld, int nr, int nc, double* out, const SumScratch& s,
                             cudaStream_t st) {
    launch_sum<double, kLeanStages>(vals, 0, ld, nr, nc, 1, out, s, nullptr, st);
}

} // namespace sgpu
