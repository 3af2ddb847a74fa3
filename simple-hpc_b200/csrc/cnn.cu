// cnn.cu — the learned warm start for p': a U-Net trained and run with this file's own kernels.
//
// Network (levels L, base channels c): encoder level l applies two 3x3 convolutions with c * 2^l
// output channels and ReLU; levels are joined by 2x2 average pooling; the decoder upsamples (nearest),
// concatenates the encoder output of its level and applies two 3x3 convolutions with ReLU; a 1x1
// convolution gives the one output channel. Activations are NHWC BF16 with channel counts that are
// multiples of 16; the convolutions use BF16 copies of FP32 master weights and accumulate in FP32 on
// the 5th-generation tensor cores (tcgen05, TMEM accumulators: conv_tc.cu). Training: mean-squared
// error, Adam.
//
// The convolutions are implicit GEMMs. Forward: Y[p, co] = sum over taps t and input channels ci of
// X[p + t, ci] W[co, t, ci]. The input gradient is the same kernel on the output gradient with the
// flipped weights W'[ci, 8 - t, co]. The weight gradient is a GEMM over pixels: dW[co, t, ci] = sum
// over p of dZ[p, co] X[p + t, ci], over chunks of pixels added into FP32 with atomics. This file
// holds the rest of the network: pooling, upsampling and concatenation, the head, the loss, Adam and
// the solver-level plumbing.
//
// Inputs (2 channels, zero-padded to 16): b / s_b and AP / m_a - 1 of the p' system of one multigrid
// level (b and AP as pressure.cpp:39-47 forms them, restricted like multigrid.cpp:232-261), with s_b
// = sqrt(mean b^2) and m_a = mean AP. Output: p' * m_a / s_b, i.e. p' in units where the system has
// unit diagonal and unit right-hand side.
#include "cnn.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <stdexcept>

namespace sgpu {

namespace {

using bf16 = __nv_bfloat16;

// W'[ci][tap'][co] = W[co][8 - tap'][ci]: the weights of the input-gradient convolution.
__global__ void k_flip_weights(const bf16* __restrict__ W, bf16* __restrict__ Wf, int Cout, int Cin) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long>(Cout) * 9 * Cin) return;
    const int ci = static_cast<int>(i % Cin);
    const int tap = static_cast<int>((i / Cin) % 9);
    const int co = static_cast<int>(i / (9L * Cin));
    Wf[(static_cast<long>(ci) * 9 + (8 - tap)) * Cout + co] = W[i];
}

// dZ = dY where the post-activation output Y > 0, else 0 (ReLU backward, in place allowed).
__global__ void k_relu_back(const bf16* __restrict__ Y, const bf16* dY, bf16* dZ, long n) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dZ[i] = __bfloat162float(Y[i]) > 0.0f ? dY[i] : __float2bfloat16(0.0f);
}

// db[c] += sum over pixels of dZ[p, c].
__global__ void k_bias_grad(const bf16* __restrict__ dZ, long npix, int C, float* __restrict__ db) {
    const int c = threadIdx.x;
    if (c >= C) return;
    float s = 0.0f;
    for (long p = blockIdx.x; p < npix; p += gridDim.x) s += __bfloat162float(dZ[p * C + c]);
    atomicAdd(db + c, s);
}

// 2x2 average pooling, 8 channels (16 bytes) per thread, 32-bit indices (images of up to 2^31
// channel values): the forward pass's pooling.
__global__ void k_pool8(const bf16* __restrict__ X, bf16* __restrict__ Y, int N, int H, int W, int C) {
    const int g8 = C / 8;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int Ho = H / 2, Wo = W / 2;
    if (i >= N * Ho * Wo * g8) return;
    const int g = i % g8, q = i / g8;
    const int x = q % Wo, y = (q / Wo) % Ho, b = q / (Wo * Ho);
    const uint4* src = reinterpret_cast<const uint4*>(X);
    const int base = ((b * H + 2 * y) * W + 2 * x) * g8 + g, row = W * g8;
    const uint4 v[4] = {src[base], src[base + g8], src[base + row], src[base + row + g8]};
    uint32_t out[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float lo = 0.0f, hi = 0.0f;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t w = (&v[e].x)[k];
            const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w);
            lo += __low2float(h);
            hi += __high2float(h);
        }
        const __nv_bfloat162 r = __floats2bfloat162_rn(0.25f * lo, 0.25f * hi);
        out[k] = *reinterpret_cast<const uint32_t*>(&r);
    }
    reinterpret_cast<uint4*>(Y)[i] = make_uint4(out[0], out[1], out[2], out[3]);
}

// Backward of the 2x2 average pooling.
__global__ void k_pool_back(const bf16* __restrict__ dY, bf16* __restrict__ dX, int N, int H, int W, int C) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long>(N) * H * W * C) return;
    const int c = static_cast<int>(i % C);
    const long q = i / C;
    const int x = static_cast<int>(q % W), y = static_cast<int>((q / W) % H);
    const long b = q / (static_cast<long>(W) * H);
    dX[i] = __float2bfloat16(0.25f * __bfloat162float(dY[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]));
}

// Y (H x W, Ca + Cb channels) = [nearest 2x upsampling of A (H/2 x W/2, Ca channels), B (Cb)], 8
// channels (16 bytes) per thread, 32-bit indices (Ca, Cb multiples of 8).
__global__ void k_up_concat8(const bf16* __restrict__ A, int Ca, const bf16* __restrict__ B, int Cb,
                             bf16* __restrict__ Y, int N, int H, int W) {
    const int ga = Ca / 8, gb = Cb / 8, gc = ga + gb;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= N * H * W * gc) return;
    const int g = i % gc, q = i / gc;
    const int x = q % W, y = (q / W) % H, b = q / (W * H);
    reinterpret_cast<uint4*>(Y)[i] =
        g < ga ? reinterpret_cast<const uint4*>(A)[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * ga + g]
               : reinterpret_cast<const uint4*>(B)[q * gb + (g - ga)];
}

// Backward of k_up_concat8: dA = sum over the 4 children, dB = copy. One thread per element of dB
// (dB has twice as many elements as dA).
__global__ void k_up_concat_back(const bf16* __restrict__ dY, bf16* __restrict__ dA, int Ca,
                                 bf16* __restrict__ dB, int Cb, int N, int H, int W) {
    const int C = Ca + Cb;
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long nb = static_cast<long>(N) * H * W * Cb;
    const long na = static_cast<long>(N) * (H / 2) * (W / 2) * Ca;
    if (i < nb) dB[i] = dY[(i / Cb) * C + Ca + (i % Cb)];
    if (i < na) {
        const int c = static_cast<int>(i % Ca);
        const long q = i / Ca;
        const int Wo = W / 2, Ho = H / 2;
        const int x = static_cast<int>(q % Wo), y = static_cast<int>((q / Wo) % Ho);
        const long b = q / (static_cast<long>(Wo) * Ho);
        float s = 0.0f;
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
                s += __bfloat162float(dY[((b * H + 2 * y + dy) * W + 2 * x + dx) * C + c]);
        dA[i] = __float2bfloat16(s);
    }
}

// a += b (the skip connection's gradient joins the encoder output's).
__global__ void k_add_bf16(bf16* __restrict__ a, const bf16* __restrict__ b, long n) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] = __float2bfloat16(__bfloat162float(a[i]) + __bfloat162float(b[i]));
}

// 1x1 head: out[p] = b + sum over c of w[c] X[p, c] (FP32).
__global__ void k_head_fwd(const bf16* __restrict__ X, int C, const float* __restrict__ w,
                           const float* __restrict__ b, float* __restrict__ out, long npix) {
    const long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float s = b[0];
    for (int c = 0; c < C; ++c) s += w[c] * __bfloat162float(X[p * C + c]);
    out[p] = s;
}
// Head backward with the mean-squared error folded in: d = 2 (out - t) / npix; dX = d w; dw, db
// summed over pixels; loss = sum of (out - t)^2 / npix.
__global__ void k_head_back_mse(const bf16* __restrict__ X, int C, const float* __restrict__ w,
                                const float* __restrict__ out, const float* __restrict__ target,
                                bf16* __restrict__ dX, float* __restrict__ dw, float* __restrict__ db,
                                float* __restrict__ loss, long npix) {
    __shared__ float sw[128];
    __shared__ float sb, sl;
    const long p = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (threadIdx.x < C) sw[threadIdx.x] = 0.0f;
    if (threadIdx.x == 0) sb = sl = 0.0f;
    __syncthreads();
    if (p < npix) {
        const float diff = out[p] - target[p];
        const float d = 2.0f * diff / static_cast<float>(npix);
        for (int c = 0; c < C; ++c) {
            dX[p * C + c] = __float2bfloat16(d * w[c]);
            atomicAdd(&sw[c], d * __bfloat162float(X[p * C + c]));
        }
        atomicAdd(&sb, d);
        atomicAdd(&sl, diff * diff / static_cast<float>(npix));
    }
    __syncthreads();
    if (threadIdx.x < C) atomicAdd(dw + threadIdx.x, sw[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(db, sb);
        atomicAdd(loss, sl);
    }
}

// Adam (bias-corrected by c1 = 1 - b1^t, c2 = 1 - b2^t) on the FP32 master parameters.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_bf16(const float* __restrict__ a, bf16* __restrict__ b, long n) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

// 2-channel FP32 pixels -> 16-channel BF16 pixels (channels 2..15 zero).
__global__ void k_pack_input(const float* __restrict__ in, bf16* __restrict__ X, long npix) {
    const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix * 16) return;
    const long p = i / 16;
    const int c = static_cast<int>(i % 16);
    X[i] = __float2bfloat16(c < 2 ? in[p * 2 + c] : 0.0f);
}

// ---- solver-level plumbing ----

template <class T> __global__ void k_restrict_b(LevelViewT<T> F, LevelViewT<T> C) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= C.nx || J >= C.ny) return;
    const int f = 2 * I * F.stride + 2 * J, fs = F.stride;
    C.b[I * C.stride + J] = F.b[f] + F.b[f + 1] + F.b[f + fs] + F.b[f + fs + 1];
}
template <class T> __global__ void k_inject_x(LevelViewT<T> C, LevelViewT<T> F) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= F.nx || J >= F.ny) return;
    F.x[I * F.stride + J] = C.x[(I / 2) * C.stride + J / 2];
}
template <class T> __global__ void k_zero_x(LevelViewT<T> L) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    L.x[I * L.stride + J] = T(0);
}
template <class T> __global__ void k_level_stats(LevelViewT<T> L, double* cells, std::size_t plane) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const int q = I * L.stride + J;
    const double b = L.b[q];
    cells[static_cast<std::size_t>(I) * L.ny + J] = b * b;
    cells[plane + static_cast<std::size_t>(I) * L.ny + J] = static_cast<double>(L.AP[q]);
}

struct Scale {
    double sb, ma;
};
__device__ __forceinline__ Scale scale_of(const double* sums, int nx, int ny) {
    const double n = static_cast<double>(nx) * ny;
    return {sqrt(sums[0] / n), sums[1] / n};
}

// Network input of a level, zero-padded to hc x wc (16-channel BF16 pixels).
template <class T>
__global__ void k_make_input(LevelViewT<T> L, const double* sums, bf16* __restrict__ X, int hc, int wc) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= hc || J >= wc) return;
    const Scale s = scale_of(sums, L.nx, L.ny);
    float c0 = 0.0f, c1 = 0.0f;
    if (I < L.nx && J < L.ny) {
        const int q = I * L.stride + J;
        c0 = s.sb > 0.0 ? static_cast<float>(L.b[q] / s.sb) : 0.0f;
        c1 = s.ma > 0.0 ? static_cast<float>(L.AP[q] / s.ma - 1.0) : 0.0f;
    }
    bf16* x = X + (static_cast<long>(I) * wc + J) * 16;
    x[0] = __float2bfloat16(c0);
    x[1] = __float2bfloat16(c1);
    for (int c = 2; c < 16; ++c) x[c] = __float2bfloat16(0.0f);
}
// L.x = out * s_b / m_a over the level (out is hc x wc).
template <class T>
__global__ void k_take_output(LevelViewT<T> L, const double* sums, const float* __restrict__ out, int wc) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const Scale s = scale_of(sums, L.nx, L.ny);
    const double k = s.ma > 0.0 ? s.sb / s.ma : 0.0;
    L.x[I * L.stride + J] = static_cast<T>(out[static_cast<long>(I) * wc + J] * k);
}
// Training pair of level l (input as k_make_input without padding; target = block mean of L0.x).
template <class T>
__global__ void k_make_pair(LevelViewT<T> L, LevelViewT<T> L0, int l, const double* sums,
                            float* __restrict__ in, float* __restrict__ target) {
    const int J = blockIdx.x * 32 + threadIdx.x, I = blockIdx.y * 8 + threadIdx.y;
    if (I >= L.nx || J >= L.ny) return;
    const Scale s = scale_of(sums, L.nx, L.ny);
    const int q = I * L.stride + J;
    const long o = static_cast<long>(I) * L.ny + J;
    in[2 * o] = s.sb > 0.0 ? static_cast<float>(L.b[q] / s.sb) : 0.0f;
    in[2 * o + 1] = s.ma > 0.0 ? static_cast<float>(L.AP[q] / s.ma - 1.0) : 0.0f;
    const int k = 1 << l;
    double acc = 0.0;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) acc += static_cast<double>(L0.x[(I * k + a) * L0.stride + J * k + b]);
    acc /= static_cast<double>(k) * k;
    target[o] = s.sb > 0.0 ? static_cast<float>(acc * s.ma / s.sb) : 0.0f;
}

unsigned blocks(long n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }
dim3 grid2(int nx, int ny) { return dim3((ny + 31) / 32, (nx + 7) / 8); }

} // namespace

// ---- solver-level launchers ----

template <class T> void launch_restrict_b(const LevelViewT<T>& F, const LevelViewT<T>& C, cudaStream_t st) {
    k_restrict_b<T><<<grid2(C.nx, C.ny), dim3(32, 8), 0, st>>>(F, C);
    SGPU_LAUNCH();
}
template <class T> void launch_inject_x(const LevelViewT<T>& C, const LevelViewT<T>& F, cudaStream_t st) {
    k_inject_x<T><<<grid2(F.nx, F.ny), dim3(32, 8), 0, st>>>(C, F);
    SGPU_LAUNCH();
}
template <class T> void launch_zero_x(const LevelViewT<T>& L, cudaStream_t st) {
    k_zero_x<T><<<grid2(L.nx, L.ny), dim3(32, 8), 0, st>>>(L);
    SGPU_LAUNCH();
}
template <class T>
void launch_level_stats(const LevelViewT<T>& L, double* cells, std::size_t plane, cudaStream_t st) {
    k_level_stats<T><<<grid2(L.nx, L.ny), dim3(32, 8), 0, st>>>(L, cells, plane);
    SGPU_LAUNCH();
}
template <class T>
void launch_make_pair(const LevelViewT<T>& L, const LevelViewT<T>& L0, int l, const double* sums,
                      float* in, float* target, cudaStream_t st) {
    k_make_pair<T><<<grid2(L.nx, L.ny), dim3(32, 8), 0, st>>>(L, L0, l, sums, in, target);
    SGPU_LAUNCH();
}

#define SGPU_CNN_INST(T)                                                                               \
    template void launch_restrict_b<T>(const LevelViewT<T>&, const LevelViewT<T>&, cudaStream_t);      \
    template void launch_inject_x<T>(const LevelViewT<T>&, const LevelViewT<T>&, cudaStream_t);        \
    template void launch_zero_x<T>(const LevelViewT<T>&, cudaStream_t);                                \
    template void launch_level_stats<T>(const LevelViewT<T>&, double*, std::size_t, cudaStream_t);     \
    template void launch_make_pair<T>(const LevelViewT<T>&, const LevelViewT<T>&, int, const double*, \
                                      float*, float*, cudaStream_t);
SGPU_CNN_INST(double)
SGPU_CNN_INST(float)
#undef SGPU_CNN_INST

// ---- the network ----

UNet::UNet(int base, int levels, unsigned seed) : base_(base), levels_(levels) {
    if (base < 16 || base > 128 || base % 16 || levels < 1 || levels > 5)
        throw Error(SGPU_E_INVALID, "cnn: base channels must be a multiple of 16 in [16, 128] and levels 1..5");
    auto ch = [&](int l) { return base << l; };
    for (int l = 0; l < levels; ++l) {
        convs_.push_back({l == 0 ? 16 : ch(l - 1), ch(l), l});
        convs_.push_back({ch(l), ch(l), l});
    }
    for (int l = levels - 2; l >= 0; --l) {
        convs_.push_back({ch(l + 1) + ch(l), ch(l), l});
        convs_.push_back({ch(l), ch(l), l});
    }
    // One FP32 array: per convolution W [Cout][9][Cin] then bias [Cout]; head w [base], b.
    long off = 0;
    for (auto& c : convs_) {
        c.w_off = off;
        off += static_cast<long>(c.cout) * 9 * c.cin;
        c.b_off = off;
        off += c.cout;
    }
    head_w_ = off;
    off += base;
    head_b_ = off;
    off += 1;
    nparam_ = off;
    // He-normal initialisation over the real fan-in (the padded input channels stay zero).
    std::vector<float> h(static_cast<std::size_t>(nparam_), 0.0f);
    std::mt19937 rng(seed);
    for (std::size_t k = 0; k < convs_.size(); ++k) {
        const Conv& c = convs_[k];
        const int real_in = k == 0 ? 2 : c.cin;
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * real_in)));
        for (int co = 0; co < c.cout; ++co)
            for (int t = 0; t < 9; ++t)
                for (int ci = 0; ci < real_in; ++ci)
                    h[static_cast<std::size_t>(c.w_off + (static_cast<long>(co) * 9 + t) * c.cin + ci)] = nd(rng);
    }
    std::normal_distribution<float> nh(0.0f, std::sqrt(1.0f / base));
    for (int c = 0; c < base; ++c) h[static_cast<std::size_t>(head_w_ + c)] = nh(rng);
    SGPU_CUDA(cudaMalloc(&w_, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMalloc(&g_, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMalloc(&m_, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMalloc(&v_, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMalloc(&wb_, sizeof(bf16) * nparam_));
    SGPU_CUDA(cudaMalloc(&wf_, sizeof(bf16) * max_conv_weights()));
    SGPU_CUDA(cudaMalloc(&loss_, sizeof(float)));
    SGPU_CUDA(cudaMalloc(&err_, sizeof(unsigned)));
    SGPU_CUDA(cudaMemset(err_, 0, sizeof(unsigned)));
    SGPU_CUDA(cudaMemcpy(w_, h.data(), sizeof(float) * nparam_, cudaMemcpyHostToDevice));
    SGPU_CUDA(cudaMemset(g_, 0, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMemset(m_, 0, sizeof(float) * nparam_));
    SGPU_CUDA(cudaMemset(v_, 0, sizeof(float) * nparam_));
    refresh_bf16(nullptr);
    SGPU_CUDA(cudaDeviceSynchronize());
}

UNet::~UNet() {
    cudaDeviceSynchronize();
    free_acts();
    cudaFree(w_);
    cudaFree(g_);
    cudaFree(m_);
    cudaFree(v_);
    cudaFree(wb_);
    cudaFree(wf_);
    cudaFree(loss_);
    cudaFree(err_);
}

void UNet::check_error(cudaStream_t st) {
    unsigned h = 0;
    SGPU_CUDA(cudaMemcpyAsync(&h, err_, sizeof h, cudaMemcpyDeviceToHost, st));
    SGPU_CUDA(cudaStreamSynchronize(st));
    if (h) {
        SGPU_CUDA(cudaMemsetAsync(err_, 0, sizeof h, st));
        throw Error(SGPU_E_TIMEOUT, "tensor-core convolution: a bounded wait for its MMAs ran out");
    }
}

void UNet::free_acts() {
    for (void* p : acts_) cudaFree(p);
    acts_.clear();
    n_ = h_ = wd_ = 0;
}

long UNet::max_conv_weights() const {
    long m = 0;
    for (const auto& c : convs_) m = std::max(m, static_cast<long>(c.cout) * 9 * c.cin);
    return m;
}

double UNet::flops_per_pixel() const {
    double f = 0.0;
    for (const auto& c : convs_) f += 2.0 * 9.0 * c.cin * c.cout / static_cast<double>(1 << (2 * c.level));
    return f + 2.0 * base_;
}

void UNet::refresh_bf16(cudaStream_t st) {
    k_to_bf16<<<blocks(nparam_), 256, 0, st>>>(w_, wb_, nparam_);
    SGPU_LAUNCH();
}

// Activation and gradient buffers for n images of h x w (reallocated when the shape changes).
void UNet::shape(int n, int h, int w) {
    if (n == n_ && h == h_ && w == wd_) return;
    if (n < 1 || h < 1 || w < 1 || h % multiple() || w % multiple())
        throw Error(SGPU_E_INVALID, "cnn: image height and width must be positive multiples of " +
                                        std::to_string(multiple()));
    if (static_cast<long>(n) * h * w * 256 > 0x7fffffffL)
        throw Error(SGPU_E_INVALID, "cnn: images too large (the pooling and concatenation kernels index in 32 bits)");
    SGPU_CUDA(cudaDeviceSynchronize());
    free_acts();
    n_ = n;
    h_ = h;
    wd_ = w;
    auto alloc = [&](long elems, std::size_t size) {
        void* p = nullptr;
        SGPU_CUDA(cudaMalloc(&p, size * static_cast<std::size_t>(std::max(1L, elems))));
        acts_.push_back(p);
        return p;
    };
    auto abf = [&](long elems) { return static_cast<bf16*>(alloc(elems, sizeof(bf16))); };
    in_ = abf(px(0) * 16);
    for (auto& c : convs_) {
        c.y = abf(px(c.level) * c.cout);
        c.dy = abf(px(c.level) * c.cout);
    }
    const int L = levels_;
    pool_.assign(L, nullptr);
    dpool_.assign(L, nullptr);
    cat_.assign(L, nullptr);
    dcat_.assign(L, nullptr);
    skip_.assign(L, nullptr);
    for (int l = 1; l < L; ++l) {
        pool_[l] = abf(px(l) * (base_ << (l - 1)));
        dpool_[l] = abf(px(l) * (base_ << (l - 1)));
    }
    for (int l = 0; l + 1 < L; ++l) {
        const long c = (base_ << (l + 1)) + (base_ << l);
        cat_[l] = abf(px(l) * c);
        dcat_[l] = abf(px(l) * c);
        skip_[l] = abf(px(l) * (base_ << l));
    }
    in32_ = static_cast<float*>(alloc(2 * px(0), sizeof(float)));
    out_ = static_cast<float*>(alloc(px(0), sizeof(float)));
    target_ = static_cast<float*>(alloc(px(0), sizeof(float)));
}

void UNet::conv_fwd(const Conv& c, const bf16* x, bf16* y, cudaStream_t st) {
    launch_conv_tc(x, n_, h_ >> c.level, wd_ >> c.level, c.cin, wb_ + c.w_off, w_ + c.b_off, y, c.cout, 1, err_, st);
}

void UNet::forward(cudaStream_t st) {
    if (!n_) throw Error(SGPU_E_INVALID, "cnn: forward before an input was set");
    const int L = levels_;
    const bf16* x = in_;
    std::size_t k = 0;
    for (int l = 0; l < L; ++l) {
        if (l > 0) {
            const Conv& prev = convs_[k - 1];
            k_pool8<<<blocks(px(l) * prev.cout / 8), 256, 0, st>>>(prev.y, pool_[l], n_, h_ >> (l - 1),
                                                                  wd_ >> (l - 1), prev.cout);
            SGPU_LAUNCH();
            x = pool_[l];
        }
        conv_fwd(convs_[k], x, convs_[k].y, st);
        conv_fwd(convs_[k + 1], convs_[k].y, convs_[k + 1].y, st);
        x = convs_[k + 1].y;
        k += 2;
    }
    for (int l = L - 2; l >= 0; --l) {
        const int ca = base_ << (l + 1), cb = base_ << l;
        k_up_concat8<<<blocks(px(l) * (ca + cb) / 8), 256, 0, st>>>(x, ca, convs_[2 * l + 1].y, cb, cat_[l],
                                                                   n_, h_ >> l, wd_ >> l);
        SGPU_LAUNCH();
        conv_fwd(convs_[k], cat_[l], convs_[k].y, st);
        conv_fwd(convs_[k + 1], convs_[k].y, convs_[k + 1].y, st);
        x = convs_[k + 1].y;
        k += 2;
    }
    k_head_fwd<<<blocks(px(0)), 256, 0, st>>>(x, base_, w_ + head_w_, w_ + head_b_, out_, px(0));
    SGPU_LAUNCH();
}

// Gradient through conv c given c.dy (gradient of its post-ReLU output): ReLU mask, weight and bias
// gradients, and (dx != null) the gradient of its input.
void UNet::conv_back(const Conv& c, const bf16* x_in, bf16* dx, cudaStream_t st) {
    const int h = h_ >> c.level, w = wd_ >> c.level;
    const long np = px(c.level);
    k_relu_back<<<blocks(np * c.cout), 256, 0, st>>>(c.y, c.dy, c.dy, np * c.cout);
    SGPU_LAUNCH();
    launch_conv_wgrad_tc(x_in, c.dy, n_, h, w, c.cin, c.cout, g_ + c.w_off, err_, st);
    k_bias_grad<<<static_cast<unsigned>(std::min<long>(np, 1024)), std::max(32, c.cout), 0, st>>>(c.dy, np, c.cout,
                                                                                               g_ + c.b_off);
    SGPU_LAUNCH();
    if (!dx) return;
    const long nw = static_cast<long>(c.cout) * 9 * c.cin;
    k_flip_weights<<<blocks(nw), 256, 0, st>>>(wb_ + c.w_off, wf_, c.cout, c.cin);
    SGPU_LAUNCH();
    launch_conv_tc(c.dy, n_, h, w, c.cout, wf_, nullptr, dx, c.cin, 0, err_, st);
}

void UNet::backward(cudaStream_t st) {
    if (!n_) throw Error(SGPU_E_INVALID, "cnn: backward before an input was set");
    const int L = levels_;
    SGPU_CUDA(cudaMemsetAsync(g_, 0, sizeof(float) * nparam_, st));
    SGPU_CUDA(cudaMemsetAsync(loss_, 0, sizeof(float), st));
    std::size_t k = convs_.size();
    const Conv& last = convs_[k - 1];
    k_head_back_mse<<<blocks(px(0)), 256, 0, st>>>(last.y, base_, w_ + head_w_, out_, target_, last.dy,
                                                  g_ + head_w_, g_ + head_b_, loss_, px(0));
    SGPU_LAUNCH();
    // Decoder, finest level first (the reverse of the forward order).
    for (int l = 0; l <= L - 2; ++l) {
        k -= 2;
        const Conv& c1 = convs_[k];
        const Conv& c2 = convs_[k + 1];
        conv_back(c2, c1.y, c1.dy, st);
        conv_back(c1, cat_[l], dcat_[l], st);
        // Upsampled part -> the producing convolution's output gradient; skip part -> stashed for
        // the encoder output of level l.
        const int ca = base_ << (l + 1), cb = base_ << l;
        k_up_concat_back<<<blocks(px(l) * cb), 256, 0, st>>>(dcat_[l], convs_[k - 1].dy, ca, skip_[l], cb, n_,
                                                            h_ >> l, wd_ >> l);
        SGPU_LAUNCH();
    }
    // Encoder, coarsest level first.
    for (int l = L - 1; l >= 0; --l) {
        k -= 2;
        const Conv& c1 = convs_[k];
        const Conv& c2 = convs_[k + 1];
        if (l < L - 1) {
            k_add_bf16<<<blocks(px(l) * c2.cout), 256, 0, st>>>(c2.dy, skip_[l], px(l) * c2.cout);
            SGPU_LAUNCH();
        }
        conv_back(c2, c1.y, c1.dy, st);
        conv_back(c1, l == 0 ? in_ : pool_[l], l == 0 ? nullptr : dpool_[l], st);
        if (l > 0) {
            const Conv& prev = convs_[k - 1];
            k_pool_back<<<blocks(px(l - 1) * prev.cout), 256, 0, st>>>(dpool_[l], prev.dy, n_, h_ >> (l - 1),
                                                                      wd_ >> (l - 1), prev.cout);
            SGPU_LAUNCH();
        }
    }
}

void UNet::adam(float lr, cudaStream_t st) {
    ++step_;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(step_));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(step_));
    k_adam<<<blocks(nparam_), 256, 0, st>>>(w_, g_, m_, v_, nparam_, lr, b1, b2, 1e-8f, c1, c2);
    SGPU_LAUNCH();
    refresh_bf16(st);
}

void UNet::set_input(const float* host, int n, int h, int w, cudaStream_t st) {
    shape(n, h, w);
    SGPU_CUDA(cudaMemcpyAsync(in32_, host, sizeof(float) * 2 * px(0), cudaMemcpyHostToDevice, st));
    k_pack_input<<<blocks(px(0) * 16), 256, 0, st>>>(in32_, in_, px(0));
    SGPU_LAUNCH();
}

void UNet::set_target(const float* host, cudaStream_t st) {
    if (!n_) throw Error(SGPU_E_INVALID, "cnn: target before an input was set");
    SGPU_CUDA(cudaMemcpyAsync(target_, host, sizeof(float) * px(0), cudaMemcpyHostToDevice, st));
}

void UNet::get_output(float* host, cudaStream_t st) {
    SGPU_CUDA(cudaMemcpyAsync(host, out_, sizeof(float) * px(0), cudaMemcpyDeviceToHost, st));
    check_error(st);
}

float UNet::loss(cudaStream_t st) {
    float l = 0.0f;
    SGPU_CUDA(cudaMemcpyAsync(&l, loss_, sizeof(float), cudaMemcpyDeviceToHost, st));
    check_error(st);
    return l;
}

void UNet::get_params(float* host) const {
    SGPU_CUDA(cudaDeviceSynchronize());
    SGPU_CUDA(cudaMemcpy(host, w_, sizeof(float) * nparam_, cudaMemcpyDeviceToHost));
}
void UNet::set_params(const float* host) {
    SGPU_CUDA(cudaDeviceSynchronize());
    SGPU_CUDA(cudaMemcpy(w_, host, sizeof(float) * nparam_, cudaMemcpyHostToDevice));
    refresh_bf16(nullptr);
    SGPU_CUDA(cudaDeviceSynchronize());
}
void UNet::get_grads(float* host) const {
    SGPU_CUDA(cudaDeviceSynchronize());
    SGPU_CUDA(cudaMemcpy(host, g_, sizeof(float) * nparam_, cudaMemcpyDeviceToHost));
}

template <class T>
void UNet::predict_level(const LevelViewT<T>& L, double* cells, std::size_t plane, double* sums,
                         const SumScratch& ss, cudaStream_t st) {
    const int m = multiple();
    const int hc = (L.nx + m - 1) / m * m, wc = (L.ny + m - 1) / m * m;
    shape(1, hc, wc);
    launch_level_stats(L, cells, plane, st);
    launch_ordered_sum(cells, plane, L.ny, L.nx, L.ny, 2, sums, ss, nullptr, st);
    k_make_input<T><<<grid2(hc, wc), dim3(32, 8), 0, st>>>(L, sums, in_, hc, wc);
    SGPU_LAUNCH();
    forward(st);
    k_take_output<T><<<grid2(L.nx, L.ny), dim3(32, 8), 0, st>>>(L, sums, out_, wc);
    SGPU_LAUNCH();
}
template void UNet::predict_level<double>(const LevelViewT<double>&, double*, std::size_t, double*,
                                          const SumScratch&, cudaStream_t);
template void UNet::predict_level<float>(const LevelViewT<float>&, double*, std::size_t, double*,
                                         const SumScratch&, cudaStream_t);

// Weights file: four int32 (magic "UNET", base, levels, parameter count), then the FP32 parameters.
void UNet::save(const std::string& path) const {
    std::vector<float> h(static_cast<std::size_t>(nparam_));
    get_params(h.data());
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw Error(SGPU_E_INVALID, "cnn: cannot write " + path);
    const int hdr[4] = {0x54454e55, base_, levels_, static_cast<int>(nparam_)};
    const bool ok = std::fwrite(hdr, sizeof hdr, 1, f) == 1 &&
                    std::fwrite(h.data(), sizeof(float), h.size(), f) == h.size();
    std::fclose(f);
    if (!ok) throw Error(SGPU_E_INVALID, "cnn: short write to " + path);
}

std::unique_ptr<UNet> UNet::load(const std::string& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(SGPU_E_INVALID, "cnn: cannot read weights file " + path);
    int hdr[4] = {0, 0, 0, 0};
    if (std::fread(hdr, sizeof hdr, 1, f) != 1 || hdr[0] != 0x54454e55) {
        std::fclose(f);
        throw Error(SGPU_E_INVALID, "cnn: not a weights file: " + path);
    }
    std::unique_ptr<UNet> net;
    try {
        net = std::make_unique<UNet>(hdr[1], hdr[2], 0u);
    } catch (...) {
        std::fclose(f);
        throw;
    }
    if (net->nparam_ != hdr[3]) {
        std::fclose(f);
        throw Error(SGPU_E_INVALID, "cnn: weights file does not match its network shape: " + path);
    }
    std::vector<float> h(static_cast<std::size_t>(net->nparam_));
    const std::size_t got = std::fread(h.data(), sizeof(float), h.size(), f);
    std::fclose(f);
    if (got != h.size()) throw Error(SGPU_E_INVALID, "cnn: truncated weights file: " + path);
    net->set_params(h.data());
    return net;
}

} // namespace sgpu
