// noalloc.cu — the ordered sum without any device allocation (sgpu_ordered_sum_noalloc).
//
// Some callers cannot allocate device memory when they need this reduction: a host application
// that reserves all of its device memory up front and runs under a fixed budget, a plugin host that
// forbids libraries from allocating, or a latency-critical loop that cannot afford cudaMalloc's
// implicit device synchronisation. For them this entry point takes device input and output
// pointers and keeps its only scratch — the per-row partial sums and the completion counter of
// the ordered reduction (reduce.cu) — in file-scope __device__ arrays of fixed size. Every GPU that
// loads this library holds those arrays (128 KiB + 256 B) until the process exits.
//
// The array names are host-side stand-ins in host code, not device addresses, so the device
// addresses are fetched with cudaGetSymbolAddress once per device, with that device current, by
// the first call made on that device; that first call should come before any stream capture.
// The addresses are kept for the life of the process, so a cudaDeviceReset after the first call on
// a device (which unloads the module and may move the arrays) is not supported.
#include "kernels.hpp"

#include <mutex>

namespace sgpu {

namespace {

constexpr int kNoAllocMaxRows = 16384; // rows of the summed block (one double of scratch each)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_rows[kNoAllocMaxRows];
static __device__ __align__(256) unsigned int g_noalloc_counter[64];

struct DeviceScratch {
    double* rows = nullptr;
    unsigned int* counter = nullptr;
    bool ready = false;
};

std::mutex g_mutex;
DeviceScratch g_scratch[kMaxDevices];

// Device addresses of the scratch arrays on the current device (looked up once per device).
DeviceScratch scratch_for_current_device() {
    int dev = 0;
    SGPU_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(SGPU_E_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch& s = g_scratch[dev];
    if (!s.ready) {
        void* rows = nullptr;
        void* counter = nullptr;
        SGPU_CUDA(cudaGetSymbolAddress(&rows, g_noalloc_rows));
        SGPU_CUDA(cudaGetSymbolAddress(&counter, g_noalloc_counter));
        s.rows = static_cast<double*>(rows);
        s.counter = static_cast<unsigned int*>(counter);
        s.ready = true;
    }
    return s;
}

} // namespace

} // namespace sgpu

extern "C" int sgpu_ordered_sum_noalloc(const double* values, int nrows, int ncols, int ld,
                                        double* out, void* stream) {
    if (!values || !out) return sgpu::fail(SGPU_E_INVALID, "sgpu_ordered_sum_noalloc: null pointer");
    if (nrows < 0 || ncols < 0 || ld < ncols)
        return sgpu::fail(SGPU_E_INVALID, "sgpu_ordered_sum_noalloc: bad sizes");
    if (nrows > sgpu::kNoAllocMaxRows)
        return sgpu::fail(SGPU_E_INVALID,
                          "sgpu_ordered_sum_noalloc: " + std::to_string(nrows) +
                              " rows exceed the fixed scratch of " +
                              std::to_string(sgpu::kNoAllocMaxRows) + " rows");
    try {
        const sgpu::DeviceScratch s = sgpu::scratch_for_current_device();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // The completion counter must start at zero; the previous call may have been abandoned.
        SGPU_CUDA(cudaMemsetAsync(s.counter, 0, sizeof(unsigned int), st));
        sgpu::SumScratch ss;
        ss.rows = s.rows;
        ss.counter = s.counter;
        ss.max_rows = sgpu::kNoAllocMaxRows;
        ss.max_k = 1;
        sgpu::launch_ordered_sum(values, 0, ld, nrows, ncols, 1, out, ss, nullptr, st);
        return SGPU_OK;
    } catch (const sgpu::Error& e) {
        return sgpu::fail(e.code, e.what());
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}
