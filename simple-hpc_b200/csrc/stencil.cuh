// stencil.cuh — per-cell arithmetic shared by every FP64 kernel.
//
// The expressions keep the reference's operation order exactly and every translation unit that
// includes this file is compiled with --fmad=false, so a cell's result has the same bits as the
// reference's serial C++ (built with -ffp-contract=off, CMakeLists.txt:34).
#pragma once

#include "common.hpp"

namespace sgpu {

// std::max(0.0, a) is (0.0 < a) ? a : 0.0, signed zeros included (coefficients.cpp:19).
__device__ __forceinline__ double mx0(double a) { return (0.0 < a) ? a : 0.0; }

// in_boundary_band (coefficients.cpp:10-13): j is tested against N_halo_y, i against N_halo_x.
__device__ __forceinline__ bool in_band(const DevParams& p, int i, int j) {
    return j == p.Hy + 1 || j == p.NY + p.Hy || i == p.NX + p.Hx - 1 || i == p.Hx;
}

// The 9 coefficients of one momentum cell: convective_coefficients (coefficients.cpp:15-39) plus
// diffusive_coefficients (coefficients.cpp:41-63, precomputed per band), summed component-wise as
// Coef9 operator+ does (coefficients.cpp:5-8). Order: AE AW AN AS AEE AWW ANN ASS AP.
struct Coef9 {
    double AE, AW, AN, AS, AEE, AWW, ANN, ASS, AP;
};

__device__ __forceinline__ Coef9 momentum_coef(const DevParams& p, double ue, double uw, double vn,
                                               double vs, int i, int j) {
    const double dx = p.dx, dy = p.dy;
    const bool band = in_band(p, i, j);
    double AE, AW, AN, AS, AEE, AWW, ANN, ASS;
    if (p.uds || band) {
        AE = dy * mx0(-ue);
        AW = dy * mx0(uw);
        AN = dx * mx0(-vn);
        AS = dx * mx0(vs);
        AEE = AWW = ANN = ASS = 0.0;
    } else {
        AE = -dy * (-0.75 * mx0(-ue) + 0.375 * mx0(ue) - 0.125 * mx0(-uw));
        AW = -dy * (-0.125 * mx0(ue) + 0.375 * mx0(-uw) - 0.75 * mx0(uw));
        AN = -dx * (-0.75 * mx0(-vn) + 0.375 * mx0(vn) - 0.125 * mx0(-vs));
        AS = -dx * (-0.125 * mx0(vn) + 0.375 * mx0(-vn) - 0.75 * mx0(vs));
        AEE = -0.125 * dy * mx0(-ue);
        AWW = -0.125 * dy * mx0(uw);
        ANN = -0.125 * dx * mx0(-vn);
        ASS = -0.125 * dx * mx0(vs);
    }
    const double APc = AS + AW + AN + AE + ASS + AWW + ANN + AEE;
    const double* d = (p.order == 2 || band) ? p.dband : p.dint;
    Coef9 c;
    c.AE = AE + d[0];
    c.AW = AW + d[1];
    c.AN = AN + d[2];
    c.AS = AS + d[3];
    c.AEE = AEE + d[4];
    c.AWW = AWW + d[5];
    c.ANN = ANN + d[6];
    c.ASS = ASS + d[7];
    c.AP = APc + d[8];
    return c;
}

// Colour of a momentum cell (momentum_u.hpp:15-17).
__device__ __forceinline__ int momentum_colour(int ncol, int i, int j) {
    return ncol == 2 ? (i + j) % 2 : (i + 3 * j) % 5;
}

} // namespace sgpu
