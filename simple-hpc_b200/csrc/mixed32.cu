// mixed32.cu — the FP32 correction sweep of mixed.cu (k_corr_stream and its launchers), in a
// translation unit of its own so that it is built with fused multiply-add contraction; mixed.cu's
// FP64 kernels (coefficients, residuals, corrections) are built without it.
#define SGPU_FLOAT_UNIT 1
#include "mixed.cu"
