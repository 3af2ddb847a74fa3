// cg.cu — Jacobi-preconditioned conjugate gradient for p' on the device (solve_pc_cg,
// src/pressure.cpp:208-317), FP64 and bit-identical to the reference.
//
// The scalars (alpha, beta, the mean corrections, the stopping test) live in device memory and are
// updated by one-thread kernels between the per-cell passes, so an iteration needs no host round
// trip; once the solve stops, every later kernel of the launch sequence sees `done` and returns.
// Sums of per-cell values go through the ordered reduction (reduce.cu) in CellSums order.
#include "kernels.hpp"

namespace sgpu {

namespace {

constexpr int BX = 32, BY = 8;

__device__ __forceinline__ bool cell_p(const DevParams& p, int& i, int& j) {
    j = p.H + 1 + static_cast<int>(blockIdx.x * BX + threadIdx.x);
    i = p.H + static_cast<int>(blockIdx.y * BY + threadIdx.y);
    return i <= p.NX + p.H - 1 && j <= p.NY + p.H;
}

dim3 grid_p(const DevParams& p) { return dim3((p.NY + BX - 1) / BX, (p.NX + BY - 1) / BY); }

// Plane offset of cell (i, j) in the compact NX x NY cell buffer.
__device__ __forceinline__ std::size_t cell_ix(const DevParams& p, int i, int j) {
    return static_cast<std::size_t>(i - p.H) * p.NY + (j - p.H - 1);
}

// r = b - mb, z = r / APP; values rr, z, r.z, r (pressure.cpp:230-245).
__global__ void k_cg_init(DevParams p, PressurePtr w, CgPtr cg, const CgScalars* sc,
                          double* cells, std::size_t plane) {
    int i, j;
    if (!cell_p(p, i, j)) return;
    const std::size_t q = static_cast<std::size_t>(i) * p.pitch + j, c = cell_ix(p, i, j);
    const double ri = w.b[q] - sc->mb;
    cg.r[q] = ri;
    const double zi = ri / w.APP[q];
    cg.z[q] = zi;
    cells[c] = ri * ri;
    cells[plane + c] = zi;
    cells[2 * plane + c] = ri * zi;
    cells[3 * plane + c] = ri;
}

// d = z - mz (pressure.cpp:253-256).
__global__ void k_cg_dinit(DevParams p, CgPtr cg, const CgScalars* sc) {
    if (sc->done) return;
    int i, j;
    if (!cell_p(p, i, j)) return;
    const std::size_t q = static_cast<std::size_t>(i) * p.pitch + j;
    cg.d[q] = cg.z[q] - sc->mz;
}

// q = A d, value d.q (pressure.cpp:263-274).
__global__ void k_cg_dq(DevParams p, PressurePtr w, CgPtr cg, const CgScalars* sc, double* cells) {
    if (sc->done) return;
    int i, j;
    if (!cell_p(p, i, j)) return;
    const std::size_t q = static_cast<std::size_t>(i) * p.pitch + j, ld = p.pitch;
    const double* d = cg.d;
    const double qi = w.APP[q] * d[q] -
                      (w.AEP[q] * d[q + 1] + w.AWP[q] * d[q - 1] + w.ASP[q] * d[q + ld] +
                       w.ANP[q] * d[q - ld]);
    cg.q[q] = qi;
    cells[cell_ix(p, i, j)] = d[q] * qi;
}

// x += alpha d; r -= alpha q; z = r / APP; values rr, z, r.z, r (pressure.cpp:278-292).
__global__ void k_cg_update(DevParams p, PressurePtr w, CgPtr cg, const CgScalars* sc,
                            double* cells, std::size_t plane) {
    if (sc->done) return;
    int i, j;
    if (!cell_p(p, i, j)) return;
    const std::size_t q = static_cast<std::size_t>(i) * p.pitch + j, c = cell_ix(p, i, j);
    const double alpha = sc->alpha;
    w.pc[q] += alpha * cg.d[q];
    const double ri = cg.r[q] - alpha * cg.q[q];
    cg.r[q] = ri;
    const double zi = ri / w.APP[q];
    cg.z[q] = zi;
    cells[c] = ri * ri;
    cells[plane + c] = zi;
    cells[2 * plane + c] = ri * zi;
    cells[3 * plane + c] = ri;
}

// d = (z - mz) + beta d (pressure.cpp:306-309).
__global__ void k_cg_dir(DevParams p, CgPtr cg, const CgScalars* sc) {
    if (sc->done) return;
    int i, j;
    if (!cell_p(p, i, j)) return;
    const std::size_t q = static_cast<std::size_t>(i) * p.pitch + j;
    cg.d[q] = (cg.z[q] - sc->mz) + sc->beta * cg.d[q];
}

// Scalar steps between the passes. sums holds the ordered sums of the preceding pass.
//  0: mb = sum(b) / n                                  (pressure.cpp:226-228)
//  1: after the init pass: rr == 0 -> done; nb, mz, rz (pressure.cpp:246-252)
//  2: after the d.q pass: breakdown test, alpha        (pressure.cpp:275-277)
//  3: after the update pass: k, rel, stop test, beta   (pressure.cpp:293-305)
__global__ void k_cg_scalars(int stage, CgScalars* sc, const double* sums) {
    if (stage == 0) {
        sc->k = 0;
        sc->done = 0;
        sc->rel = 0.0;
        sc->mb = sums[0] / sc->n;
        return;
    }
    if (sc->done) return;
    if (stage == 1) {
        const double rr = sums[0], sz = sums[1], rz = sums[2], sr = sums[3];
        if (rr == 0.0) {
            sc->done = 1; // ||b|| == 0: p' = 0
            return;
        }
        sc->nb = sqrt(rr);
        sc->mz = sz / sc->n;
        sc->rz = rz - sc->mz * sr;
        sc->rel = 1.0;
        if (sc->maxit <= 0) sc->done = 1;
    } else if (stage == 2) {
        const double dq = sums[0];
        if (!(dq > 0.0)) {
            sc->done = 1; // breakdown: stop with the current x
            return;
        }
        sc->alpha = sc->rz / dq;
    } else {
        const double rr = sums[0], sz = sums[1], sr = sums[3];
        double rzn = sums[2];
        sc->k += 1;
        sc->rel = sqrt(rr) / sc->nb;
        if (sc->rel <= sc->tol) {
            sc->done = 1;
            return;
        }
        sc->mz = sz / sc->n;
        rzn -= sc->mz * sr;
        sc->beta = rzn / sc->rz;
        sc->rz = rzn;
        // The reference still updates d before its loop test fails; d is not read afterwards.
        if (sc->k >= sc->maxit) sc->done = 2;
    }
}

} // namespace

void launch_cg_init(const DevParams& p, PressurePtr w, CgPtr cg, CgScalars* sc, double* cells,
                    std::size_t plane, cudaStream_t st) {
    k_cg_init<<<grid_p(p), dim3(BX, BY), 0, st>>>(p, w, cg, sc, cells, plane);
    SGPU_LAUNCH();
}
void launch_cg_scalars(int stage, CgScalars* sc, const double* sums, cudaStream_t st) {
    k_cg_scalars<<<1, 1, 0, st>>>(stage, sc, sums);
    SGPU_LAUNCH();
}
void launch_cg_dinit(const DevParams& p, CgPtr cg, const CgScalars* sc, cudaStream_t st) {
    k_cg_dinit<<<grid_p(p), dim3(BX, BY), 0, st>>>(p, cg, sc);
    SGPU_LAUNCH();
}
void launch_cg_dq(const DevParams& p, PressurePtr w, CgPtr cg, const CgScalars* sc, double* cells,
                  cudaStream_t st) {
    k_cg_dq<<<grid_p(p), dim3(BX, BY), 0, st>>>(p, w, cg, sc, cells);
    SGPU_LAUNCH();
}
void launch_cg_update(const DevParams& p, PressurePtr w, CgPtr cg, const CgScalars* sc,
                      double* cells, std::size_t plane, cudaStream_t st) {
    k_cg_update<<<grid_p(p), dim3(BX, BY), 0, st>>>(p, w, cg, sc, cells, plane);
    SGPU_LAUNCH();
}
void launch_cg_dir(const DevParams& p, CgPtr cg, const CgScalars* sc, cudaStream_t st) {
    k_cg_dir<<<grid_p(p), dim3(BX, BY), 0, st>>>(p, cg, sc);
    SGPU_LAUNCH();
}

} // namespace sgpu
