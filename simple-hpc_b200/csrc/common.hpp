// common.hpp — shared host/device definitions of the B200 SIMPLE solver.
#pragma once

#include "../../include/sgpu.h"

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define SGPU_HD __host__ __device__
#else
#define SGPU_HD
#endif

namespace sgpu {

// ---- errors ----

// Exception carrying an sgpu status code; converted to a return value at the C ABI.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);
int fail(int code, const std::string& msg); // sets the message, returns code
// Kernel launches issued by this library (process-wide, for the benchmark's launch count).
void count_launch();

void params_defaults(sgpu_params_t& p);
void params_finalize(sgpu_params_t& p);
void params_from_config(const std::string& text, sgpu_params_t& p);

#ifdef __CUDACC__
#define SGPU_CUDA(x)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess)                                                                \
            throw ::sgpu::Error(e_ == cudaErrorMemoryAllocation ? SGPU_E_NOMEM : SGPU_E_CUDA, \
                                std::string("GPU error: ") + cudaGetErrorString(e_) +         \
                                    " in " #x);                                               \
    } while (0)
#define SGPU_LAUNCH()                                                                         \
    do {                                                                                      \
        ::sgpu::count_launch();                                                               \
        SGPU_CUDA(cudaGetLastError());                                                        \
    } while (0)

// Once-per-device set-up of a kernel: function attributes (cudaFuncSetAttribute) and occupancy
// queries. CUDA keeps a function's attributes in each device's context, so a process that runs on
// several GPUs must set them on every one. The state is one bit per device ordinal; the first call
// on a device runs init() with that device current, under a mutex, so first calls from several
// host threads are safe. init() returns an int that later calls on that device get back (e.g. the
// resident blocks per SM).
struct PerDeviceOnce {
    static constexpr int kMaxDevices = 64;
    std::mutex mu;
    std::atomic<std::uint64_t> done{0};
    int value[kMaxDevices] = {};
    template <class F> int get(F&& init) {
        int dev = 0;
        SGPU_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) throw Error(SGPU_E_INVALID, "device ordinal above 63");
        const std::uint64_t bit = std::uint64_t{1} << dev;
        if (done.load(std::memory_order_acquire) & bit) return value[dev];
        std::lock_guard<std::mutex> lock(mu);
        if (!(done.load(std::memory_order_relaxed) & bit)) {
            value[dev] = init();
            done.fetch_or(bit, std::memory_order_release);
        }
        return value[dev];
    }
};
#endif

// ---- device layout ----
//
// Every full-grid field is stored row-major with a padded row pitch: element (i, j) of the
// reference's nrows x ncols Field2D is at [i * pitch + j]. The pitch is a multiple of 32 doubles, so
// each row starts on a 256-byte boundary; the padding columns are never read as cells.
struct Grid {
    int nrows = 0, ncols = 0, pitch = 0;
    std::size_t elems() const { return static_cast<std::size_t>(nrows) * pitch; }
    std::size_t bytes() const { return elems() * sizeof(double); }
};

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Inclusive cell range [i0, i1] x [j0, j1] of a kernel, in global (i, j) indices.
struct Range {
    int i0, i1, j0, j1;
    SGPU_HD int rows() const { return i1 >= i0 ? i1 - i0 + 1 : 0; }
    SGPU_HD int cols() const { return j1 >= j0 ? j1 - j0 + 1 : 0; }
};

// What the kernels read from the parameters. The diffusive coefficients depend only on whether a
// cell is in the boundary band, so the host evaluates both variants once (with the expressions of
// diffusive_coefficients, src/coefficients.cpp:41-63; IEEE-exact, no contraction) and the kernels
// add them to the per-cell convective part.
struct DevParams {
    int NX, NY, H, Hx, Hy, nrows, ncols, pitch;
    int ncol;  // momentum colours: 5, or 2 for UDS + order 2 (momentum_u.cpp:70-72)
    int uds;   // convection_scheme == UDS
    int order; // diffusion_order
    double dx, dy, nu, au, av, ap;
    double dband[9]; // diffusive coefficients in the boundary band (and for order 2)
    double dint[9];  // diffusive coefficients elsewhere (order 4)
};

// Multigrid level view (the reference's MGView, include/simple/multigrid.hpp:59-66): element
// (I, J), 0 <= I < nx, 0 <= J < ny, of each array is ptr[I * stride + J]; the pointers address
// interior cell (0, 0) and every neighbour of an interior cell lies inside the allocation.
#ifdef __CUDACC__
// The red-black update value of multigrid.cpp:61-63, x = b / AP; x += nb / AP. The double
// instances keep the reference's two divisions (bit parity); the float instances (the mixed-precision
// V-cycle, where no bit parity applies) divide once, (b + nb) / AP, with the fast single-precision
// division (__fdividef, a reciprocal and a multiply: within 2 ulp for AP of any magnitude the
// operator holds). A smoother of a correction solve inside FP64 defect correction needs no correctly
// rounded quotient, and the IEEE division's instruction sequence is a sizeable share of the level
// kernels' issue slots.
__device__ __forceinline__ double rb_value(double b, double nb, double ap) {
    double t = b / ap;
    t += nb / ap;
    return t;
}
__device__ __forceinline__ float rb_value(float b, float nb, float ap) {
    return __fdividef(b + nb, ap);
}
#endif

// The four links of one FP32 multigrid cell, read with one 128-bit load.
struct alignas(16) Link4 {
    float e, w, n, s;
};

// One multigrid level (interior origin at AE..r, row stride `stride`). Double levels (the reference's
// bits) keep the links in the arrays AE, AW, AN, AS; float levels (the mixed-precision V-cycle) keep
// them in L4, one record per cell, and leave those four arrays null.
template <class T> struct LevelViewT {
    int nx, ny, stride;
    T *AE, *AW, *AN, *AS, *AP, *b, *x, *r;
    Link4* L4 = nullptr;
};
using LevelView = LevelViewT<double>;
using LevelView32 = LevelViewT<float>;

#ifdef __CUDACC__
template <class T> struct Links {
    T e, w, n, s;
};
__device__ __forceinline__ Links<double> links(const LevelViewT<double>& L, int q) {
    return {__ldg(L.AE + q), __ldg(L.AW + q), __ldg(L.AN + q), __ldg(L.AS + q)};
}
__device__ __forceinline__ Links<float> links(const LevelViewT<float>& L, int q) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(L.L4) + q);
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ void set_links(const LevelViewT<double>& L, int q, double e, double w, double n,
                                          double s) {
    L.AE[q] = e;
    L.AW[q] = w;
    L.AN[q] = n;
    L.AS[q] = s;
}
__device__ __forceinline__ void set_links(const LevelViewT<float>& L, int q, float e, float w, float n, float s) {
    reinterpret_cast<float4*>(L.L4)[q] = make_float4(e, w, n, s);
}
#endif

} // namespace sgpu
