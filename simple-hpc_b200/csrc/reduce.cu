// reduce.cu — ordered (bit-reproducible) sums on the device.
//
// The reference sums a per-cell quantity by adding each row left to right from 0.0 and then the
// row sums top to bottom from 0.0 (CellSums::sum and add_rows, src/decomp.cpp:176-205; det_sum,
// src/multigrid.cpp:18-34). Floating-point addition is not associative, so the same bits need the
// same chain: one dependent chain per row, then one chain over the rows. This file runs the row
// chains in parallel (one thread per row) over tiles staged through shared memory, so the global
// reads stay coalesced, and the last CTA to finish adds the row sums in order.
#include "kernels.hpp"

namespace sgpu {

namespace {

constexpr int kTileRows = 32; // rows per CTA (one summing lane each)
constexpr int kTileCols = 32; // columns per staged chunk
constexpr int kLoadWarps = 8;

__global__ void __launch_bounds__(32 * kLoadWarps)
    k_ordered_sum(const double* __restrict__ vals, std::size_t plane_stride, int ld, int nr, int nc,
                  double* __restrict__ rows, unsigned int* counter, double* __restrict__ out,
                  const int* skip) {
    if (skip && *skip) return;
    __shared__ double tile[2][kTileRows][kTileCols + 1];
    __shared__ bool last_block;
    const int m = blockIdx.y;
    const double* src = vals + m * plane_stride;
    const int r0 = blockIdx.x * kTileRows;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int nchunks = (nc + kTileCols - 1) / kTileCols;

    auto load = [&](int chunk, int buf) {
        const int c = chunk * kTileCols + tx;
        for (int rr = ty; rr < kTileRows; rr += kLoadWarps) {
            const int r = r0 + rr;
            tile[buf][rr][tx] = (r < nr && c < nc) ? src[static_cast<std::size_t>(r) * ld + c] : 0.0;
        }
    };

    double acc = 0.0;
    if (nchunks > 0) load(0, 0);
    __syncthreads();
    for (int k = 0; k < nchunks; ++k) {
        const int buf = k & 1;
        if (k + 1 < nchunks) load(k + 1, buf ^ 1);
        if (ty == 0) {
            const int cmax = min(kTileCols, nc - k * kTileCols);
            for (int c = 0; c < cmax; ++c) acc += tile[buf][tx][c];
        }
        __syncthreads();
    }
    if (ty == 0 && r0 + tx < nr) rows[static_cast<std::size_t>(m) * nr + r0 + tx] = acc;

    // The last CTA to finish adds every plane's row sums in row order.
    __threadfence();
    __syncthreads();
    if (tx == 0 && ty == 0) {
        const unsigned int total = gridDim.x * gridDim.y;
        last_block = (atomicAdd(counter, 1u) == total - 1);
    }
    __syncthreads();
    if (!last_block) return;
    __threadfence();
    if (ty == 0 && tx < static_cast<int>(gridDim.y)) {
        const double* rs = rows + static_cast<std::size_t>(tx) * nr;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s += __ldcg(rs + r); // L2: written by other CTAs
        out[tx] = s;
    }
    if (tx == 0 && ty == 0) *counter = 0u; // ready for the next launch on this stream
}

} // namespace

void launch_ordered_sum(const double* vals, std::size_t plane_stride, int ld, int nr, int nc, int K,
                        double* out, const SumScratch& s, const int* skip, cudaStream_t st) {
    if (K < 1 || K > 32 || K > s.max_k || nr > s.max_rows)
        throw Error(SGPU_E_INVALID, "ordered sum: sizes exceed the scratch");
    if (nr <= 0) {
        SGPU_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * K, st));
        return;
    }
    const dim3 grid((nr + kTileRows - 1) / kTileRows, K);
    k_ordered_sum<<<grid, dim3(32, kLoadWarps), 0, st>>>(vals, plane_stride, ld, nr, nc, s.rows,
                                                         s.counter, out, skip);
    SGPU_LAUNCH();
}

} // namespace sgpu
