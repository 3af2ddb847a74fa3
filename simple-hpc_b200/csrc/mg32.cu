// mg32.cu — the float (mixed-precision) instances of mg.cu, in a translation unit of their own
// so that they are built with fused multiply-add contraction; mg.cu's double instances keep the
// reference's bits without it.
#define SGPU_FLOAT_UNIT 1
#include "mg.cu"
