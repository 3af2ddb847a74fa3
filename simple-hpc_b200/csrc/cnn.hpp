// cnn.hpp — the learned warm start for the p' solve: a U-Net with its own BF16 tensor-core (tcgen05) kernels.
//
// The network maps the p' system of one multigrid level (right-hand side b and diagonal AP, both
// normalised) to a p' guess on that level. The solver runs it on the finest level of at most
// max_size x max_size cells, injects the guess down to the fine grid and lets the unchanged
// multigrid iterate from there (mg_mode = tolerance: to the same tolerance as from zero).
#pragma once

#include "common.hpp"
#include "kernels.hpp"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

namespace sgpu {

class UNet {
  public:
    // base channels (multiple of 16) on the finest level, doubling per level; levels 1..5.
    UNet(int base, int levels, unsigned seed);
    ~UNet();
    UNet(const UNet&) = delete;
    UNet& operator=(const UNet&) = delete;

    int base() const { return base_; }
    int levels() const { return levels_; }
    long num_params() const { return nparam_; }
    // Height and width of an input must be multiples of this.
    int multiple() const { return 1 << (levels_ - 1); }
    // Multiply-adds x 2 of one forward pass per pixel of the finest level.
    double flops_per_pixel() const;

    // Host-facing calls (n images of h x w; input 2 channels interleaved per pixel, FP32).
    void set_input(const float* host, int n, int h, int w, cudaStream_t st);
    void set_target(const float* host, cudaStream_t st);
    void forward(cudaStream_t st);
    // MSE loss against the target; parameter gradients into the gradient buffer.
    void backward(cudaStream_t st);
    void adam(float lr, cudaStream_t st);
    void get_output(float* host, cudaStream_t st);
    float loss(cudaStream_t st);
    void get_params(float* host) const;
    void set_params(const float* host);
    void get_grads(float* host) const;

    // Warm start on a solver level (element type T): input from L.b and L.AP, output into L.x.
    // cells: scratch of two nx * ny planes (plane apart); sums: two doubles of device scratch.
    template <class T>
    void predict_level(const LevelViewT<T>& L, double* cells, std::size_t plane, double* sums,
                       const SumScratch& ss, cudaStream_t st);

    void save(const std::string& path) const;
    static std::unique_ptr<UNet> load(const std::string& path);
    // Raises SGPU_E_TIMEOUT (and clears the word) if a tensor-core convolution's bounded wait for its
    // MMAs gave up since the last check (its outputs are then not to be trusted). Synchronises st.
    void check_error(cudaStream_t st);

  private:
    struct Conv {
        int cin, cout, level;
        long w_off = 0, b_off = 0;
        __nv_bfloat16* y = nullptr;  // post-ReLU output
        __nv_bfloat16* dy = nullptr; // gradient of the output (then of the pre-activation)
    };
    void shape(int n, int h, int w);
    void free_acts();
    void refresh_bf16(cudaStream_t st);
    void conv_fwd(const Conv& c, const __nv_bfloat16* x, __nv_bfloat16* y, cudaStream_t st);
    void conv_back(const Conv& c, const __nv_bfloat16* x_in, __nv_bfloat16* dx, cudaStream_t st);
    long max_conv_weights() const;
    long px(int l) const { return static_cast<long>(n_) * (h_ >> l) * (wd_ >> l); }

    int base_, levels_;
    long nparam_ = 0, head_w_ = 0, head_b_ = 0;
    std::vector<Conv> convs_;
    float *w_ = nullptr, *g_ = nullptr, *m_ = nullptr, *v_ = nullptr, *loss_ = nullptr;
    __nv_bfloat16* wb_ = nullptr; // BF16 copy of every parameter
    __nv_bfloat16* wf_ = nullptr; // flipped weights of one conv (input-gradient pass)
    unsigned* err_ = nullptr;      // device word: a tensor-core convolution's bounded wait gave up
    int step_ = 0;
    // activations for the current shape
    int n_ = 0, h_ = 0, wd_ = 0;
    std::vector<void*> acts_;
    __nv_bfloat16* in_ = nullptr;
    std::vector<__nv_bfloat16*> pool_, dpool_, cat_, dcat_, skip_;
    float *in32_ = nullptr, *out_ = nullptr, *target_ = nullptr;
};

// 3x3 convolution, zero padding 1, of NHWC BF16 X [N*H*W][Cin] with W [Cout][9][Cin] (+ bias when not
// null, ReLU when relu) into Y [N*H*W][Cout], as a tcgen05 implicit GEMM with the accumulator in TMEM
// (conv_tc.cu). Cin and Cout multiples of 16, Cout <= 256. *err (device) gets a bit if a bounded
// wait for the MMAs gave up.
void launch_conv_tc(const __nv_bfloat16* X, int N, int H, int W, int Cin, const __nv_bfloat16* Wt,
                    const float* bias, __nv_bfloat16* Y, int Cout, int relu, unsigned* err, cudaStream_t st);

// Weight gradient of that convolution, dW [Cout][9][Cin] += sum over pixels of dZ[p, co] X[p + t, ci]
// (dZ: the pre-activation gradient), as tcgen05 GEMMs over pixel chunks added with FP32 atomics.
// Cin multiple of 16 up to 256, Cout multiple of 16 up to 128.
void launch_conv_wgrad_tc(const __nv_bfloat16* X, const __nv_bfloat16* dZ, int N, int H, int W, int Cin,
                          int Cout, float* dW, unsigned* err, cudaStream_t st);

// Warm-start plumbing on a multigrid hierarchy (element type T).
// C.b = sum of the four children of F.b (the restriction of the right-hand side itself).
template <class T> void launch_restrict_b(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st);
// F.x = C.x of the parent cell (piecewise-constant injection).
template <class T> void launch_inject_x(const LevelViewT<T>& C, const LevelViewT<T>& F, cudaStream_t st);
// L.x = 0 over the interior.
template <class T> void launch_zero_x(const LevelViewT<T>& L, cudaStream_t st);
// Training pair of a level: input (b, AP) as the network sees it and the target p' block average
// of the fine p' (x0 of level 0, averaged over 2^l x 2^l blocks), normalised the same way. in: h x
// w x 2 FP32, target: h x w FP32 (device buffers).
template <class T>
void launch_make_pair(const LevelViewT<T>& L, const LevelViewT<T>& L0, int l, const double* sums,
                      float* in, float* target, cudaStream_t st);
// Per-cell b^2 and AP of a level into two compact planes (for the normalisation sums).
template <class T>
void launch_level_stats(const LevelViewT<T>& L, double* cells, std::size_t plane, cudaStream_t st);

} // namespace sgpu
