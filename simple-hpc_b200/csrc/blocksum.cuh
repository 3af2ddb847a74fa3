// blocksum.cuh — deterministic block sums in FP64 (the mixed-precision path's residual sums).
//
// A fixed xor-shuffle tree inside each warp, then thread 0 adds the warps' sums in warp order. At
// each tree step lane i forms v_i + v_(i^o) and its partner v_(i^o) + v_i, the same bits, so every
// lane of a warp ends with the same value and the result depends only on the inputs and the block
// shape: repeated runs give the same bits, independent of scheduling. No atomics are involved.
#pragma once

namespace sgpu {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of v over a block of NW full warps (tid: the linear thread index); valid in thread 0.
// s: NW doubles of shared memory. Every thread of the block must call it.
template <int NW>
__device__ __forceinline__ double block_sum(double v, double* s, int tid) {
    v = warp_sum(v);
    if ((tid & 31) == 0) s[tid >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (tid == 0) {
#pragma unroll
        for (int w = 0; w < NW; ++w) t += s[w];
    }
    return t;
}

} // namespace sgpu
