// solver.cu — device state, phase orchestration and the C ABI (include/sgpu.h).
//
// Replaces the reference's HipSolver (src/hip/solver_hip.hip:326-550). Differences by design:
//  - every State array lives on the device for the whole run (as in the reference), with a padded
//    row pitch (Grid) instead of the host's packed rows;
//  - residual sums use the reference CPU's fixed order (reduce.cu), so res_u, res_v, res_p and the
//    stopping iteration are bit-identical to the serial code, not just close;
//  - momentum_solver jacobi and pressure_solver jacobi, cg and mg run on the GPU too (the reference
//    GPU backend accepts gs_multicolour + gs_redblack only, solver_hip.hip:373-377);
//  - one CUDA stream per handle; an outer iteration ends with one device->host copy of the three
//    residuals instead of a device synchronisation per phase.
#include "cnn.hpp"
#include "kernels.hpp"

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

namespace sgpu {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_last_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// Relative tolerance of the coarsest-level solve: the reference's kCoarseTol (multigrid.cpp:11)
// in FP64; the FP32 V-cycle of the mixed-precision mode stops at a tolerance FP32 can reach.
constexpr double kCoarseTol64 = 1e-10;
constexpr double kCoarseTol32 = 1e-5;

// Host evaluation of diffusive_coefficients (src/coefficients.cpp:41-63) for the two cell kinds.
static void diffusive_host(const sgpu_params_t& p, bool band_or_order2, double out[9]) {
    const double dx = p.dx, dy = p.dy, nu = p.nu;
    if (band_or_order2) {
        out[0] = dy * nu / dx;
        out[1] = dy * nu / dx;
        out[2] = dx * nu / dy;
        out[3] = dx * nu / dy;
        out[4] = out[5] = out[6] = out[7] = 0.0;
        out[8] = -nu * (-2 * dx / dy - 2 * dy / dx);
    } else {
        out[0] = 4.0 / 3 * dy * nu / dx;
        out[1] = 4.0 / 3 * dy * nu / dx;
        out[2] = 4.0 / 3 * dx * nu / dy;
        out[3] = 4.0 / 3 * dx * nu / dy;
        out[4] = -1.0 / 12 * dy * nu / dx;
        out[5] = -1.0 / 12 * dy * nu / dx;
        out[6] = -1.0 / 12 * dx * nu / dy;
        out[7] = -1.0 / 12 * dx * nu / dy;
        out[8] = -nu * (-2.5 * dx / dy - 2.5 * dy / dx);
    }
}

// One CUDA graph that runs outer iterations of one or more solvers with the stopping test on the
// device (defined with the batch kernels below); sgpu_run and sgpu_batch_run launch it.
struct IterGraph;
void destroy_iter_graph(IterGraph* g);

struct Solver {
    sgpu_params_t prm{};
    DevParams dp{};
    Grid g;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    std::size_t bytes = 0;

    double *u = nullptr, *v = nullptr, *pf = nullptr;
    Coef9Ptr cu{}, cv{};
    PressurePtr w{};
    double* scratch = nullptr; // Jacobi previous iterate (u, v and p')
    CgPtr cg{};
    CgScalars* cgs = nullptr;
    double* cells = nullptr; // 4 planes of NX x NY per-cell values for the ordered sums
    std::size_t plane = 0;
    double* sums = nullptr;  // 32 device doubles: results of ordered sums
    double* res_dev = nullptr; // res_u, res_v, res_p of the current iteration
    SumScratch ss;
    int* stats = nullptr;      // device ints: [0] coarse sweeps
    double* host_res = nullptr; // pinned: 3 residuals

    // multigrid
    std::vector<LevelView> lv;
    double* mg_r0 = nullptr;
    double* coarse_rowbuf = nullptr;
    bool mg_fast = false;            // streaming level kernels (mg_fast.cu) + single-CTA tail
    int mg_tail = 0;                 // first level handled by the tail kernel
    // first level of the float V-cycle's tail: the cluster tail's (mg.cu, k_mg_tail_cluster) where
    // the device and the grid allow it, else mg_tail
    int mg_tail32 = 0;
    std::vector<double*> mg_x2;      // second iterate buffer per streamed level (interior (0,0))
    MgLevels mgl{};
    // build: form the coarse operators inside the cycle (the streamed levels' down kernels, then the
    // tail's levels) instead of before it.
    void mg_vcycle_fast(bool x_is_zero, bool build = false);

    // fused fast path (multicolour momentum): frozen velocity copy and the sweep ping-pong buffer
    bool fast = false;
    double* xF = nullptr;
    double* tmp = nullptr;
    int sms = 148;
    int seg_rows = 64;
    // Minimum rows per CTA segment of the streaming kernels. A single solve owns the GPU and is
    // bound by each CTA's per-step latency on small grids, so it takes short segments (8 rows); a
    // batch fills the GPU with many cavities and keeps the kernels' defaults (0), which bound the
    // halo and skew work per row (use_batch_shape).
    int min_seg = 8;
    void use_batch_shape() {
        min_seg = 0;
        // A batch fills the GPU with many cavities' kernels, so SM time, not latency, bounds it: the
        // single-CTA tail (one SM) instead of the cluster tail (16 SMs for a shorter time).
        mg_tail32 = mg_tail;
        if (fast)
            seg_rows = mixed ? stream_seg_rows(dp, sms, corr_blocks_per_sm(dp.ncol), 0, corr_threads())
                             : stream_seg_rows(dp, sms, 2, 0);
    }

    int ncol = 5;
    IterGraph* run_graph = nullptr; // sgpu_run's graph (built on first use)

    // learned warm start (warm_start = cnn, or a network attached through the C ABI)
    std::unique_ptr<UNet> own_net;
    UNet* net = nullptr;
    int cnn_max = 256; // the network runs on the finest level of at most cnn_max x cnn_max cells
    long long ws_used = 0, ws_fallbacks = 0;
    float* pair_buf = nullptr; // training pair of the last sgpu_cnn_sample (input 2 planes, target)
    template <class T> int cnn_level(const std::vector<LevelViewT<T>>& L) const {
        int l = 0;
        while (l + 1 < static_cast<int>(L.size()) && std::max(L[l].nx, L[l].ny) > cnn_max) ++l;
        return l;
    }
    template <class T> bool warm_start_on(std::vector<LevelViewT<T>>& L);
    template <class T> void sample_pair(std::vector<LevelViewT<T>>& L, float* hin, float* htarget);

    int last_cg_iterations = 0, last_vcycles = 0, last_coarse_sweeps = 0;
    double last_rel = 0.0;
    bool cg_stats_pending = false;

    template <class T> T* dalloc(std::size_t count) {
        void* p = nullptr;
        const std::size_t nb = count * sizeof(T);
        SGPU_CUDA(cudaMalloc(&p, nb > 0 ? nb : 1));
        allocs.push_back(p);
        bytes += nb;
        SGPU_CUDA(cudaMemsetAsync(p, 0, nb > 0 ? nb : 1, st));
        return static_cast<T*>(p);
    }
    double* field() { return dalloc<double>(g.elems()); }

    Solver(const sgpu_params_t& p, const double* hu, const double* hv, const double* hp);
    ~Solver();

    void upload(double* dst, const double* host) {
        SGPU_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * g.pitch, host, sizeof(double) * g.ncols,
                                    sizeof(double) * g.ncols, g.nrows, cudaMemcpyHostToDevice, st));
    }
    void download(const double* src, double* host) {
        SGPU_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * g.ncols, src, sizeof(double) * g.pitch,
                                    sizeof(double) * g.ncols, g.nrows, cudaMemcpyDeviceToHost, st));
        SGPU_CUDA(cudaStreamSynchronize(st));
    }
    double* field_ptr(int id) {
        if (id == SGPU_F_U) return u;
        if (id == SGPU_F_V) return v;
        if (id == SGPU_F_P) return pf;
        if (id >= SGPU_F_CU_AE && id <= SGPU_F_CU_AP) return cu.a[id - SGPU_F_CU_AE];
        if (id >= SGPU_F_CV_AE && id <= SGPU_F_CV_AP) return cv.a[id - SGPU_F_CV_AE];
        switch (id) {
        case SGPU_F_AEP: return w.AEP;
        case SGPU_F_AWP: return w.AWP;
        case SGPU_F_ANP: return w.ANP;
        case SGPU_F_ASP: return w.ASP;
        case SGPU_F_APP: return w.APP;
        case SGPU_F_B: return w.b;
        case SGPU_F_PC: return w.pc;
        default: return nullptr;
        }
    }
    // Offset of the first p' cell (H, H + 1) in a full-grid array.
    std::size_t p_origin() const { return static_cast<std::size_t>(prm.H) * g.pitch + prm.H + 1; }
    double* at(double* f, int i, int j) const {
        return f + static_cast<std::size_t>(i) * g.pitch + j;
    }

    // ---- phases (enqueue only) ----
    void assemble_u() { launch_assemble_u(dp, u, v, cu, st); }
    void bc_u() { launch_bc_u(dp, u, st); }
    void residual_u(double* out) {
        launch_residual_u_cells(dp, cu, u, pf, cells, st);
        launch_ordered_sum(cells, 0, prm.NY - 1, prm.NX, prm.NY - 1, 1, out, ss, nullptr, st);
    }
    void sweep_u(int n);
    void assemble_v() { launch_assemble_v(dp, u, v, cv, st); }
    void bc_v() { launch_bc_v(dp, v, st); }
    void residual_v(double* out) {
        launch_residual_v_cells(dp, cv, v, pf, cells, st);
        launch_ordered_sum(cells, 0, prm.NY, prm.NX - 1, prm.NY, 1, out, ss, nullptr, st);
    }
    void sweep_v(int n);
    void assemble_p(double* out) {
        launch_assemble_p(dp, cu.a[8], cv.a[8], u, v, w, cells, nullptr, st);
        p_links_stale = false;
        launch_ordered_sum(cells, 0, prm.NY, prm.NX, prm.NY, 1, out, ss, nullptr, st);
    }
    void solve_p();
    void correct() { launch_correct(dp, w, cu.a[8], cv.a[8], u, v, pf, st); }

    void solve_redblack();
    void solve_jacobi();
    void solve_cg();
    void solve_mg();
    void mg_vcycle();
    // remove_mean0 (multigrid.cpp:327-345). known_sum: the ordered sum of f's p' cells if it is
    // already formed (it is then not summed again).
    void remove_mean0(double* f, const double* known_sum = nullptr);
    // Set while the fast iteration's pressure solve runs: the ordered sum of b, formed by the |b| / b
    // pair sum in the same order, for the multigrid's mean removal of b.
    const double* b_sum = nullptr;

    // One momentum phase on the fused path: bc, residual + AP + frozen copy, n streaming sweeps.
    void fast_momentum(bool vcomp, double* res) {
        double* x = vcomp ? v : u;
        const double* oth = vcomp ? u : v;
        double* AP = vcomp ? cv.a[8] : cu.a[8];
        // Phase attribution: the prep pass is the assembly, the ordered sum the residual.
        mark(vcomp ? SGPU_PH_BC_V : SGPU_PH_BC_U);
        if (vcomp) launch_bc_v(dp, v, st);
        else launch_bc_u(dp, u, st);
        mark(vcomp ? SGPU_PH_ASSEMBLE_V : SGPU_PH_ASSEMBLE_U);
        double* cplane = cells + (vcomp ? plane : 0);
        launch_mom_prep(dp, vcomp, x, oth, pf, xF, AP, cplane, st);
        mark(vcomp ? SGPU_PH_RESIDUAL_V : SGPU_PH_RESIDUAL_U);
        const bool deferred = defer_sums();
        if (!deferred) momentum_sum(vcomp, res, cplane, false);
        mark(vcomp ? SGPU_PH_SWEEP_V : SGPU_PH_SWEEP_U);
        const int n = vcomp ? prm.maxit_inner_v : prm.maxit_inner_u;
        double* in = x;
        double* out = tmp;
        sweep_mark(vcomp, 0, n);
        for (int k = 0; k < n; ++k) {
            launch_mom_sweep(dp, vcomp, in, out, xF, oth, pf, seg_rows, st);
            std::swap(in, out);
        }
        sweep_mark(vcomp, 1, n);
        if (in != x) launch_copy(in, x, g.elems(), st);
        if (deferred) momentum_sum(vcomp, res, cplane, true); // beside the next prep / assemble_p
    }

    // res_u / res_v: the ordered sum of |R| over the residual range. The sums feed only the stopping
    // test at the end of the iteration, so on the FP64 fast path they run on a side stream, forked
    // after the component's sweeps: res_u beside the v prep, res_v beside assemble_p and the
    // V-cycle, joined before the iteration ends. Beside the sweeps themselves they would cost more
    // than they save: a co-resident sum CTA stops the sweep's one-wave grid from fitting. The side
    // sums have their own scratch (the main stream's sums run at the same time) and read the |R|
    // planes, which nothing else writes until the next iteration's prep when the pressure solve is
    // a fixed-cycle multigrid without a warm start; otherwise the sums stay on the solver's stream.
    // SGPU_SIDE_SUMS=0 keeps them there always (a tuning switch: the bits are the same).
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork[2] = {}, ev_done[2] = {};
    bool side_sums = true;
    bool side_pending = false;
    SumScratch ss_side;
    bool defer_sums() const {
        return side_sums && side && prm.pressure_solver == SGPU_P_MG && prm.mg_mode == SGPU_MG_FIXED && !net;
    }
    void momentum_sum(bool vcomp, double* res, const double* vals, bool on_side) {
        const int nr = vcomp ? prm.NX - 1 : prm.NX, nc = vcomp ? prm.NY : prm.NY - 1;
        if (!on_side) {
            launch_ordered_sum(vals, 0, nc, nr, nc, 1, res, ss, nullptr, st);
            return;
        }
        const int k = vcomp ? 1 : 0;
        SGPU_CUDA(cudaEventRecord(ev_fork[k], st));
        SGPU_CUDA(cudaStreamWaitEvent(side, ev_fork[k], 0));
        launch_ordered_sum_lean(vals, nc, nr, nc, res, ss_side, side);
        SGPU_CUDA(cudaEventRecord(ev_done[k], side));
        side_pending = true;
    }
    void join_sums() {
        if (!side_pending) return;
        SGPU_CUDA(cudaStreamWaitEvent(st, ev_done[0], 0));
        SGPU_CUDA(cudaStreamWaitEvent(st, ev_done[1], 0));
        side_pending = false;
    }

    void fast_iteration_enqueue(double* res3) {
        fast_momentum(false, res3 + 0);
        fast_momentum(true, res3 + 1);
        mark(SGPU_PH_ASSEMBLE_P);
        launch_assemble_p_fused(dp, cu.a[8], cv.a[8], u, v, w, nullptr, nullptr, st);
        // res_p = the ordered sum of |b| over the p' cells, read from b itself (res3[3] gets the sum of b)
        launch_ordered_sum_abs_pair(w.b + p_origin(), g.pitch, prm.NX, prm.NY, res3 + 2, ss, st);
        mark(SGPU_PH_SOLVE_P);
        b_sum = res3 + 3; // the multigrid's mean of b reuses the pair's sum of b
        solve_p();
        b_sum = nullptr;
        mark(SGPU_PH_CORRECT);
        correct();
        join_sums(); // res_u, res_v from the side stream
        mark(SGPU_PH_COUNT);
    }

    // ---- per-phase device timing (CUDA events on the solver's stream) ----
    bool profiling = false;
    // Sampled timers (sgpu_set_profiling(h, 2)): sgpu_run times the phases of its first
    // kSampledIterations iterations (host-issued, between events) and replays the graph for the rest.
    bool sampled = false;
    cudaEvent_t ev[SGPU_PH_COUNT + 1] = {};
    bool ev_used[SGPU_PH_COUNT + 1] = {};
    int ev_order[SGPU_PH_COUNT + 2] = {};
    int ev_n = 0;
    double phase_acc[SGPU_PH_COUNT] = {};
    // Record the start of phase ph (SGPU_PH_COUNT marks the end of the iteration).
    void mark(int ph) {
        if (!profiling) return;
        if (!ev[ph]) SGPU_CUDA(cudaEventCreate(&ev[ph]));
        SGPU_CUDA(cudaEventRecord(ev[ph], st));
        ev_order[ev_n++] = ph;
    }
    // The streaming sweep kernels alone (k_mom_stream or k_corr_stream, back to back on the stream):
    // events before the first and after the last sweep of each component.
    cudaEvent_t sw_ev[4] = {};
    int sw_pending[2] = {0, 0};
    double sweep_acc = 0.0;
    long long sweep_launches = 0;
    void sweep_mark(bool vcomp, int end, int n) {
        if (!profiling || n <= 0) return;
        cudaEvent_t& e = sw_ev[2 * (vcomp ? 1 : 0) + end];
        if (!e) SGPU_CUDA(cudaEventCreate(&e));
        SGPU_CUDA(cudaEventRecord(e, st));
        if (end) sw_pending[vcomp ? 1 : 0] = n;
    }
    // After the stream is synchronised: add each phase's time to phase_acc (and to out if given).
    void collect_phases(double* out) {
        if (!profiling) return;
        for (int c = 0; c < 2; ++c) {
            if (!sw_pending[c]) continue;
            float ms = 0.0f;
            SGPU_CUDA(cudaEventElapsedTime(&ms, sw_ev[2 * c], sw_ev[2 * c + 1]));
            sweep_acc += ms * 1e-3;
            sweep_launches += sw_pending[c];
            sw_pending[c] = 0;
        }
        for (int k = 0; k + 1 < ev_n; ++k) {
            float ms = 0.0f;
            SGPU_CUDA(cudaEventElapsedTime(&ms, ev[ev_order[k]], ev[ev_order[k + 1]]));
            phase_acc[ev_order[k]] += ms * 1e-3;
            if (out) out[ev_order[k]] += ms * 1e-3;
        }
        ev_n = 0;
    }

    void iteration_enqueue(double* res3) {
        ev_n = 0;
        if (mixed) mixed_iteration_enqueue(res3);
        else if (fast) fast_iteration_enqueue(res3);
        else outer_iteration_enqueue(res3);
    }

    // ---- mixed precision (precision = mixed): FP32 inner solves inside FP64 defect correction ----
    bool mixed = false;
    // The mixed iteration keeps the p' operator in FP32 only; the FP64 links and APP are formed from
    // APU / APV when a caller downloads one of them.
    bool p_links_stale = false;
    bool pc_stale = false; // the mixed iteration keeps p' in FP32; the FP64 field is formed on download
    void form_p_links_if_stale(int id) {
        if (pc_stale && id == SGPU_F_PC) { // p' of the last mixed iteration, kept in FP32 (or FP64)
            if (pc_dc_src) launch_pc_from64(dp, pc_dc_src, sums + 26, w.pc, st);
            else launch_pc_from32(dp, lv32[0], sums + 26, w.pc, st);
            pc_stale = false;
            return;
        }
        if (!p_links_stale || id < SGPU_F_AEP || id > SGPU_F_APP) return;
        launch_p_links_app(dp, cu.a[8], cv.a[8], w, st);
        p_links_stale = false;
    }
    MomRec32 rec32{};                 // per-cell FP32 records: coefficients, 1/AP, R
    unsigned* corr_err = nullptr;     // device word: a correction sweep's bounded wait gave up
    // Raises SGPU_E_TIMEOUT if a correction sweep since the last check gave up waiting for its
    // record copies (its results are then not to be trusted); clears the word.
    void check_pipeline() {
        if (net) net->check_error(st);
        if (!corr_err) return;
        unsigned h = 0;
        SGPU_CUDA(cudaMemcpyAsync(&h, corr_err, sizeof h, cudaMemcpyDeviceToHost, st));
        sync();
        if (h) {
            SGPU_CUDA(cudaMemsetAsync(corr_err, 0, sizeof h, st));
            throw Error(SGPU_E_TIMEOUT, "correction sweep: a bounded wait for its record copies ran out");
        }
    }
    // FP64 defect correction of the p' solve in tolerance mode: the FP64 iterate ping-pongs between
    // two full-grid arrays (allocated on first use); pc_dc_src is the last iteration's final iterate.
    double* dc[2] = {nullptr, nullptr};
    const double* pc_dc_src = nullptr;
    double* part = nullptr;           // per-block partial sums of the FP64 tree sums
    float* e32[2] = {nullptr, nullptr}; // correction ping-pong
    std::vector<LevelView32> lv32;    // FP32 multigrid hierarchy (level 0: the p' operator)
    std::vector<float*> mg32_x2;
    MgLevelsT<float> mgl32{};

    void mixed_momentum(bool vcomp, double* res) {
        double* x = vcomp ? v : u;
        const double* oth = vcomp ? u : v;
        double* AP = vcomp ? cv.a[8] : cu.a[8];
        mark(vcomp ? SGPU_PH_BC_V : SGPU_PH_BC_U);
        if (vcomp) launch_bc_v(dp, v, st);
        else launch_bc_u(dp, u, st);
        mark(vcomp ? SGPU_PH_ASSEMBLE_V : SGPU_PH_ASSEMBLE_U);
        const int nparts = launch_mom_prep_mixed(dp, vcomp, x, oth, pf, AP, part, rec32, st);
        mark(vcomp ? SGPU_PH_RESIDUAL_V : SGPU_PH_RESIDUAL_U);
        launch_sum_partials(part, nparts, 1, 0, res, nullptr, st); // res_u / res_v: FP64 tree
        mark(vcomp ? SGPU_PH_SWEEP_V : SGPU_PH_SWEEP_U);
        const int n = vcomp ? prm.maxit_inner_v : prm.maxit_inner_u;
        int cur = 0; // e32[cur] holds the current correction (zero before the first sweep)
        sweep_mark(vcomp, 0, n);
        // small grids: every sweep in one cluster launch where the component fits
        if (launch_corr_cluster(dp, vcomp, rec32, n, x, st)) {
            sweep_mark(vcomp, 1, n);
            return;
        }
        for (int k = 0; k < n; ++k) {
            launch_corr_sweep(dp, vcomp, e32[cur], e32[1 - cur], rec32, k == 0, seg_rows, corr_err, st,
                              k == n - 1 ? x : nullptr); // the last sweep adds e into x
            cur = 1 - cur;
        }
        sweep_mark(vcomp, 1, n);
    }

    void mixed_iteration_enqueue(double* res3) {
        p_links_stale = true;
        pc_stale = true;
        mixed_momentum(false, res3 + 0);
        mixed_momentum(true, res3 + 1);
        mark(SGPU_PH_ASSEMBLE_P);
        const int nparts = launch_assemble_p_mixed(dp, cu.a[8], cv.a[8], u, v, w.b, lv32[0], part, st);
        // res_p = the sum of |b|, and the sum of b (its mean), from the blocks' partial sums
        launch_sum_partials(part, nparts, 2, nparts, res3 + 2, sums + 25, st);
        mark(SGPU_PH_SOLVE_P);
        // The coarse operators are built inside the V-cycle (fused_build: by the down kernel of the
        // level above for the streamed levels, then the tail's levels), unless a warm start reads
        // them before the first cycle.
        const bool fused_build = !net;
        if (!fused_build)
            for (std::size_t l = 1; l < lv32.size(); ++l) launch_mg_build<float>(lv32[l - 1], lv32[l], st);
        const bool dc_mode = prm.mg_mode == SGPU_MG_TOLERANCE;
        pc_dc_src = nullptr;
        int nbb = 0;
        if (dc_mode) {
            if (!dc[0]) {
                dc[0] = field();
                dc[1] = field();
            }
            nbb = launch_dc_rhs0(dp, w.b, sums + 25, lv32[0], part, st);
        } else {
            launch_b_to_f32(dp, w.b, sums + 25, lv32[0], st);
        }
        const LevelView32& L0 = lv32[0];
        // p' starts from zero. The streaming level kernels need no cleared array for that: the
        // first cycle's k_mg_down does not read x (x_zero), a warm start writes every interior cell,
        // and the zero ring is never written after allocation. Level 0 inside the tail kernel
        // (a grid of mg_tail32 = 0) reads x, so it is cleared there.
        if (mg_tail32 == 0)
            SGPU_CUDA(cudaMemsetAsync(L0.x - (L0.stride + 1), 0,
                                      sizeof(float) * (L0.nx + 2) * static_cast<std::size_t>(L0.stride), st));
        const bool guess = apply_warm_start(L0);
        auto vcycle32 = [&](bool x_zero) {
            for (int l = 0; l < mg_tail32; ++l)
                launch_mg_down<float>(lv32[l], lv32[l + 1], mg32_x2[l], prm.mg_pre, x_zero || l > 0, sms,
                                      min_seg, st, fused_build);
            if (fused_build)
                for (std::size_t l = static_cast<std::size_t>(mg_tail32) + 1; l < lv32.size(); ++l)
                    launch_mg_build<float>(lv32[l - 1], lv32[l], st);
            if (mg_tail32 == mg_tail ||
                !launch_mg_tail_cluster(mgl32, mg_tail32, prm.mg_pre, prm.mg_post, prm.mg_omega, kCoarseTol32,
                                        stats, st))
                launch_mg_tail<float>(mgl32, mg_tail32, prm.mg_pre, prm.mg_post, prm.mg_omega, kCoarseTol32,
                                      coarse_rowbuf, stats, st);
            for (int l = mg_tail32 - 1; l >= 0; --l)
                launch_mg_up<float>(lv32[l + 1], lv32[l], mg32_x2[l], lv32[l].x, prm.mg_omega,
                                    prm.mg_post, sms, min_seg, st);
        };
        if (dc_mode) {
            last_vcycles = run_cycles_dc(L0, guess, nbb, vcycle32); // p' in FP64, its sum in sums[26]
            mark(SGPU_PH_CORRECT);
            launch_correct_dc(dp, pc_dc_src, sums + 26, cu.a[8], cv.a[8], u, v, pf, st);
        } else {
            last_vcycles = run_cycles(L0, !guess, vcycle32);
            launch_tree_sum(L0.x, L0.stride, L0.nx, L0.ny, part, sums + 26, st); // the mean of p'
            mark(SGPU_PH_CORRECT);
            launch_correct_mixed(dp, L0, sums + 26, cu.a[8], cv.a[8], u, v, pf, st);
        }
        mark(SGPU_PH_COUNT);
    }

    // mg_mode = tolerance with precision = mixed: each V-cycle, from zero, solves in FP32 for the
    // correction of an FP64 iterate (mixed.cu, k_dc_update): L0.b holds (b - mean b) in FP32 on entry
    // and the blocks' sums of its square (nbb partials); L0.x holds the warm start when guess (the
    // first cycle then starts from it and is judged as in run_cycles). Cycles repeat until the FP64
    // norm ||r|| <= pressure_tolerance ||b - mean b||, at most pressure_maxit. Leaves the final
    // iterate in pc_dc_src and its sum in sums[26]; returns the cycles run.
    template <class Cycle> int run_cycles_dc(const LevelView32& L0, bool guess, int nbb, Cycle&& vcycle) {
        launch_sum_partials(part, nbb, 1, 0, sums + 28, nullptr, st);
        const double bb = fetch(sums + 28);
        if (!(bb > 0.0)) { // b = mean: p' = 0
            SGPU_CUDA(cudaMemsetAsync(dc[0], 0, g.bytes(), st));
            SGPU_CUDA(cudaMemsetAsync(sums + 26, 0, sizeof(double), st));
            pc_dc_src = dc[0];
            last_rel = 0.0;
            return 0;
        }
        const double target = prm.pressure_tolerance * std::sqrt(bb);
        last_rel_initial = 1.0;
        int c = 0, run = 0, cur = 0;
        bool first = true, from_guess = guess;
        while (c < prm.pressure_maxit) {
            if (mg_tail32 == 0 && !from_guess) launch_zero_x(L0, st); // the tail kernel reads level 0's x
            vcycle(!from_guess);
            ++c;
            ++run;
            const int nb = launch_dc_update(dp, cu.a[8], cv.a[8], w.b, sums + 25, L0, dc[1 - cur], dc[cur],
                                            first, part, st);
            launch_sum_partials(part, nb, 2, nb, sums + 29, sums + 26, st);
            pc_dc_src = dc[cur];
            cur = 1 - cur;
            first = false;
            const double rr = fetch(sums + 29);
            last_rel = std::sqrt(rr) / std::sqrt(bb);
            if (from_guess) {
                from_guess = false;
                last_rel_initial = last_rel;
                if (!(rr < bb)) { // no better than a zero start: discard the guess, restart from zero
                    ++ws_fallbacks;
                    launch_dc_rhs0(dp, w.b, sums + 25, L0, part, st);
                    first = true;
                    c = 0;
                    continue;
                }
            }
            if (std::sqrt(rr) <= target) break;
        }
        return run;
    }

    // V-cycles on level 0 (iterate L0.x, right-hand side L0.b). mg_mode = fixed: mg_cycles cycles
    // (the reference, multigrid.cpp:349-354). mg_mode = tolerance: cycles until the FP64 norm
    // ||b - A x|| <= pressure_tolerance ||b||, at most pressure_maxit; each norm is an ordered sum
    // read back by the host. Returns the number of cycles run. first_zero: L0.x is zero on entry.
    // Otherwise L0.x is a warm start. It is judged after its first cycle, not before: a network guess
    // carries rounding noise at the grid scale that the operator amplifies but the first smoothing
    // removes. If the residual after that cycle is still not below ||b|| (what a zero start has
    // before any cycle), the guess is discarded and the cycles start again from zero.
    template <class T, class Cycle>
    int run_cycles(const LevelViewT<T>& L0, bool first_zero, Cycle&& vcycle) {
        const bool tol_mode = prm.mg_mode == SGPU_MG_TOLERANCE;
        const bool judge = !first_zero;
        const int nr = L0.nx;
        auto norm2 = [&](bool residual, double* slot) {
            if (residual) launch_mg_residual_sq(L0, cells, st);
            else launch_mg_b_sq(L0, cells, st);
            launch_ordered_sum(cells, 0, L0.ny, nr, L0.ny, 1, slot, ss, nullptr, st);
            return fetch(slot);
        };
        if (!tol_mode && !judge) { // the reference's fixed cycle count from zero
            for (int c = 0; c < prm.mg_cycles; ++c) vcycle(c == 0);
            return prm.mg_cycles;
        }
        const double bb = norm2(false, sums + 28);
        if (!(bb > 0.0)) { // b = 0: p' = 0
            if (!first_zero) launch_zero_x(L0, st);
            last_rel = 0.0;
            return 0;
        }
        const int maxc = tol_mode ? prm.pressure_maxit : prm.mg_cycles;
        const double target = prm.pressure_tolerance * std::sqrt(bb);
        last_rel_initial = 1.0;
        int c = 0, run = 0;
        bool zero = first_zero;
        while (c < maxc) {
            vcycle(zero && c == 0);
            ++c;
            ++run;
            const bool need = tol_mode || (judge && c == 1);
            if (!need) continue;
            const double rr = norm2(true, sums + 29);
            last_rel = std::sqrt(rr) / std::sqrt(bb);
            if (judge && c == 1 && !zero) {
                last_rel_initial = last_rel;
                if (!(rr < bb)) { // no better than a zero start: discard the guess
                    launch_zero_x(L0, st);
                    ++ws_fallbacks;
                    zero = true;
                    c = 0;
                    continue;
                }
            }
            if (tol_mode && std::sqrt(rr) <= target) break;
        }
        return run;
    }

    // Learned warm start (warm_start = cnn): writes the network's p' guess into L0.x. Returns whether
    // a guess was written (false: L0.x stays zero).
    double last_rel_initial = 1.0;
    bool apply_warm_start(const LevelViewT<double>& L0);
    bool apply_warm_start(const LevelViewT<float>& L0);

    void outer_iteration_enqueue(double* res3) {
        mark(SGPU_PH_ASSEMBLE_U);
        assemble_u();
        mark(SGPU_PH_BC_U);
        bc_u();
        mark(SGPU_PH_RESIDUAL_U);
        residual_u(res3 + 0);
        mark(SGPU_PH_SWEEP_U);
        sweep_u(prm.maxit_inner_u);
        mark(SGPU_PH_ASSEMBLE_V);
        assemble_v();
        mark(SGPU_PH_BC_V);
        bc_v();
        mark(SGPU_PH_RESIDUAL_V);
        residual_v(res3 + 1);
        mark(SGPU_PH_SWEEP_V);
        sweep_v(prm.maxit_inner_v);
        mark(SGPU_PH_ASSEMBLE_P);
        assemble_p(res3 + 2);
        mark(SGPU_PH_SOLVE_P);
        solve_p();
        mark(SGPU_PH_CORRECT);
        correct();
        join_sums(); // res_u, res_v from the side stream
        mark(SGPU_PH_COUNT);
    }
    void sync() { SGPU_CUDA(cudaStreamSynchronize(st)); }
    double fetch(const double* dev) {
        SGPU_CUDA(cudaMemcpyAsync(host_res, dev, sizeof(double), cudaMemcpyDeviceToHost, st));
        sync();
        return host_res[0];
    }
    void finish_stats() {
        if (prm.pressure_solver == SGPU_P_MG) {
            int h = 0;
            SGPU_CUDA(cudaMemcpyAsync(&h, stats, sizeof(int), cudaMemcpyDeviceToHost, st));
            sync();
            last_coarse_sweeps = h;
        }
    }
};

Solver::Solver(const sgpu_params_t& p, const double* hu, const double* hv, const double* hp)
    : prm(p) {
    // Solver check of the reference GPU backend (solver_hip.hip:373-377), widened to every solver
    // this backend implements.
    if (p.momentum_solver == SGPU_MOM_GS_LEX || p.pressure_solver == SGPU_P_GS_LEX)
        throw Error(SGPU_E_INVALID,
                    "backend = gpu supports momentum_solver = gs_multicolour or jacobi with "
                    "pressure_solver = gs_redblack, jacobi, cg or mg (gs_lex is sequential)");
    if (p.nrows != p.NX + 2 * p.H + 1 || p.ncols != p.NY + 2 * p.H + 1 || p.NX < 1 || p.NY < 1 ||
        p.H < 2)
        throw Error(SGPU_E_INVALID, "sgpu_create: parameters are not finalised (call sgpu_params_finalize)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        (void)cudaGetLastError();
        throw Error(SGPU_E_NODEVICE, "GPU error: no CUDA device is visible");
    }
    SGPU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    g.nrows = p.nrows;
    g.ncols = p.ncols;
    g.pitch = round_up(p.ncols, 32);
    ncol = (p.convection_scheme == SGPU_UDS && p.diffusion_order == 2) ? 2 : 5;

    dp.NX = p.NX;
    dp.NY = p.NY;
    dp.H = p.H;
    dp.Hx = p.N_halo_x;
    dp.Hy = p.N_halo_y;
    dp.nrows = p.nrows;
    dp.ncols = p.ncols;
    dp.pitch = g.pitch;
    dp.ncol = ncol;
    dp.uds = p.convection_scheme == SGPU_UDS ? 1 : 0;
    dp.order = p.diffusion_order;
    dp.dx = p.dx;
    dp.dy = p.dy;
    dp.nu = p.nu;
    dp.au = p.relaxation_factor_u;
    dp.av = p.relaxation_factor_v;
    dp.ap = p.relaxation_factor_p;
    diffusive_host(p, true, dp.dband);
    diffusive_host(p, false, dp.dint);

    u = field();
    v = field();
    pf = field();
    for (int k = 0; k < 9; ++k) cu.a[k] = field();
    for (int k = 0; k < 9; ++k) cv.a[k] = field();
    w.AEP = field();
    w.AWP = field();
    w.ANP = field();
    w.ASP = field();
    w.APP = field();
    w.b = field();
    w.pc = field();
    if (p.momentum_solver == SGPU_MOM_JACOBI || p.pressure_solver == SGPU_P_JACOBI)
        scratch = field();
    fast = p.momentum_solver == SGPU_MOM_GS_MULTICOLOUR;
    if (fast) {
        xF = field();
        tmp = field();
        int dev = 0;
        SGPU_CUDA(cudaGetDevice(&dev));
        SGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        seg_rows = stream_seg_rows(dp, sms, 2, min_seg);
        if (const char* e = std::getenv("SGPU_SIDE_SUMS")) side_sums = std::atoi(e) != 0;
        ss_side.max_rows = p.nrows;
        ss_side.max_k = 1;
        ss_side.rows = dalloc<double>(static_cast<std::size_t>(p.nrows));
        ss_side.counter = dalloc<unsigned int>(1);
        SGPU_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            SGPU_CUDA(cudaEventCreateWithFlags(&ev_fork[k], cudaEventDisableTiming));
            SGPU_CUDA(cudaEventCreateWithFlags(&ev_done[k], cudaEventDisableTiming));
        }
    }
    plane = static_cast<std::size_t>(p.NX) * p.NY;
    const int kplanes = p.pressure_solver == SGPU_P_CG ? 4 : 2;
    cells = dalloc<double>(plane * kplanes);
    if (p.pressure_solver == SGPU_P_CG) {
        cg.r = field();
        cg.z = field();
        cg.d = field();
        cg.q = field();
        cgs = dalloc<CgScalars>(1);
        CgScalars init{};
        init.n = static_cast<double>(p.NX) * p.NY;
        init.tol = p.pressure_tolerance;
        init.maxit = p.pressure_maxit;
        SGPU_CUDA(cudaMemcpyAsync(cgs, &init, sizeof init, cudaMemcpyHostToDevice, st));
    }
    sums = dalloc<double>(32);
    res_dev = dalloc<double>(4);
    stats = dalloc<int>(8);
    ss.max_rows = p.nrows;
    ss.max_k = 4;
    ss.rows = dalloc<double>(static_cast<std::size_t>(ss.max_rows) * ss.max_k);
    ss.counter = dalloc<unsigned int>(1);
    SGPU_CUDA(cudaMallocHost(&host_res, sizeof(double) * 8));

    if (p.pressure_solver == SGPU_P_MG) {
        int dims[128];
        int nl = 0;
        sgpu_mg_levels(p.NX, p.NY, &nl, dims);
        mg_r0 = field();
        lv.resize(nl);
        int maxnx = 1;
        for (int l = 0; l < nl; ++l) {
            LevelView& L = lv[l];
            L.nx = dims[2 * l];
            L.ny = dims[2 * l + 1];
            if (L.nx > maxnx) maxnx = L.nx;
            if (l == 0) {
                // Level 0 aliases the PressureWork arrays (mg_view, multigrid.cpp:193-206).
                const std::size_t base = static_cast<std::size_t>(p.H) * g.pitch + p.H + 1;
                L.stride = g.pitch;
                L.AE = w.AEP + base;
                L.AW = w.AWP + base;
                L.AN = w.ANP + base;
                L.AS = w.ASP + base;
                L.AP = w.APP + base;
                L.b = w.b + base;
                L.x = w.pc + base;
                L.r = mg_r0 + base;
            } else {
                // Coarse levels: (nx + 2) x (ny + 2) with a zero halo (MGWork, multigrid.cpp:176-184).
                L.stride = L.ny + 2;
                const std::size_t n = static_cast<std::size_t>(L.nx + 2) * L.stride;
                const std::size_t base = static_cast<std::size_t>(L.stride) + 1;
                double* a[8];
                for (int k = 0; k < 8; ++k) a[k] = dalloc<double>(n) + base;
                L.AE = a[0];
                L.AW = a[1];
                L.AN = a[2];
                L.AS = a[3];
                L.AP = a[4];
                L.b = a[5];
                L.x = a[6];
                L.r = a[7];
            }
        }
        coarse_rowbuf = dalloc<double>(static_cast<std::size_t>(maxnx) + 1);
        // Streaming V-cycle: levels above tail_cells cells get a second iterate buffer; the rest
        // run in the single-CTA tail kernel. SGPU_MG_TAIL_CELLS overrides the split (tuning).
        int kTailCells = 4096;
        if (const char* e = std::getenv("SGPU_MG_TAIL_CELLS")) kTailCells = std::max(16, std::atoi(e));
        mg_fast = mg_fast_supported(p.mg_pre, p.mg_post) && p.mg_pre >= 1 && nl <= 24;
        mg_tail = 0;
        while (mg_tail < nl - 1 && lv[mg_tail].nx * lv[mg_tail].ny > kTailCells) ++mg_tail;
        mg_x2.assign(nl, nullptr);
        for (int l = 0; mg_fast && l < mg_tail; ++l) {
            if (l == 0) {
                mg_x2[0] = field() + (lv[0].x - w.pc);
            } else {
                const std::size_t n = static_cast<std::size_t>(lv[l].nx + 2) * lv[l].stride;
                mg_x2[l] = dalloc<double>(n) + (lv[l].stride + 1);
            }
        }
        mgl.n = nl;
        for (int l = 0; l < nl && l < 24; ++l) mgl.L[l] = lv[l];
    }

    if (p.precision == SGPU_PREC_MIXED) {
        if (p.momentum_solver != SGPU_MOM_GS_MULTICOLOUR || p.pressure_solver != SGPU_P_MG ||
            !mg_fast)
            throw Error(SGPU_E_INVALID,
                        "precision = mixed needs momentum_solver = gs_multicolour, pressure_solver = "
                        "mg and 1 <= mg_pre <= 4, 0 <= mg_post <= 4");
        mixed = true;
        init_mixed_kernels();
        seg_rows = stream_seg_rows(dp, sms, corr_blocks_per_sm(dp.ncol), min_seg, corr_threads());
        const std::size_t nrec =
            g.elems() + static_cast<std::size_t>(kRecExtraRows) * g.pitch + kRecFrontCols + kRecBackCols;
        rec32.near_links = dalloc<float4>(nrec) + kRecFrontCols;
        rec32.far_links = dalloc<float4>(nrec) + kRecFrontCols;
        rec32.diag = dalloc<float2>(nrec) + kRecFrontCols;
        corr_err = dalloc<unsigned>(1);
        part = dalloc<double>(static_cast<std::size_t>(std::max(mixed_partials(dp), tree_sum_partials(p.NX, p.NY))));
        e32[0] = dalloc<float>(g.elems());
        e32[1] = dalloc<float>(g.elems());
        const int nl = static_cast<int>(lv.size());
        lv32.resize(nl);
        mg32_x2.assign(nl, nullptr);
        for (int l = 0; l < nl; ++l) {
            LevelView32& L = lv32[l];
            L.nx = lv[l].nx;
            L.ny = lv[l].ny;
            L.stride = L.ny + 2;
            const std::size_t n = static_cast<std::size_t>(L.nx + 2) * L.stride;
            const std::size_t base = static_cast<std::size_t>(L.stride) + 1;
            // links as one 16-byte record per cell (AE..AS stay null), AP, b, x, r as arrays
            L.L4 = dalloc<Link4>(n) + base;
            L.AE = L.AW = L.AN = L.AS = nullptr;
            L.AP = dalloc<float>(n) + base;
            L.b = dalloc<float>(n) + base;
            L.x = dalloc<float>(n) + base;
            L.r = dalloc<float>(n) + base;
            if (l < mg_tail) mg32_x2[l] = dalloc<float>(n) + base;
        }
        mgl32.n = nl;
        for (int l = 0; l < nl && l < 24; ++l) mgl32.L[l] = lv32[l];
        mg_tail32 = mg_cluster_tail_first(mgl32, mg_tail);
    }

    if (p.warm_start == 1) {
        if (p.pressure_solver != SGPU_P_MG)
            throw Error(SGPU_E_INVALID, "warm_start = cnn needs pressure_solver = mg");
        if (!p.cnn_weights[0])
            throw Error(SGPU_E_INVALID, "warm_start = cnn needs cnn_weights = <file written by sgpu_cnn_write>");
        own_net = UNet::load(p.cnn_weights);
        net = own_net.get();
    }

    if (hu) upload(u, hu);
    if (hv) upload(v, hv);
    if (hp) upload(pf, hp);
    sync();
}

Solver::~Solver() {
    if (st) cudaStreamSynchronize(st);
    destroy_iter_graph(run_graph);
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : sw_ev)
        if (e) cudaEventDestroy(e);
    if (side) cudaStreamSynchronize(side);
    for (int k = 0; k < 2; ++k) {
        if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
        if (ev_done[k]) cudaEventDestroy(ev_done[k]);
    }
    if (side) cudaStreamDestroy(side);

    for (void* q : allocs) cudaFree(q);
    if (host_res) cudaFreeHost(host_res);
    if (st) cudaStreamDestroy(st);
}

// sweep_u_batch (momentum_u.cpp:162-171).
void Solver::sweep_u(int n) {
    if (n <= 0) return;
    if (prm.momentum_solver == SGPU_MOM_JACOBI) {
        launch_copy(u, scratch, g.elems(), st);
        for (int k = 0; k < n; ++k) {
            const bool to_u = (n - k) % 2 == 1;
            launch_sweep_u_jacobi(dp, cu, to_u ? scratch : u, to_u ? u : scratch, pf, st);
        }
        return;
    }
    for (int s = 0; s < n; ++s)
        for (int c = 0; c < ncol; ++c) launch_sweep_u_colour(dp, cu, u, pf, c, st);
}

// sweep_v_batch (momentum_v.cpp:164-173).
void Solver::sweep_v(int n) {
    if (n <= 0) return;
    if (prm.momentum_solver == SGPU_MOM_JACOBI) {
        launch_copy(v, scratch, g.elems(), st);
        for (int k = 0; k < n; ++k) {
            const bool to_v = (n - k) % 2 == 1;
            launch_sweep_v_jacobi(dp, cv, to_v ? scratch : v, to_v ? v : scratch, pf, st);
        }
        return;
    }
    for (int s = 0; s < n; ++s)
        for (int c = 0; c < ncol; ++c) launch_sweep_v_colour(dp, cv, v, pf, c, st);
}

// solve_pc_redblack (pressure.cpp:114-134).
void Solver::solve_redblack() {
    SGPU_CUDA(cudaMemsetAsync(w.pc, 0, g.bytes(), st));
    for (int k = 0; k < prm.maxit_inner_p; ++k)
        for (int c = 0; c < 2; ++c) launch_pc_redblack(dp, w, c, st);
}

// solve_pc_jacobi (pressure.cpp:77-112).
void Solver::solve_jacobi() {
    SGPU_CUDA(cudaMemsetAsync(w.pc, 0, g.bytes(), st));
    SGPU_CUDA(cudaMemsetAsync(scratch, 0, g.bytes(), st));
    const int n = prm.maxit_inner_p;
    for (int k = 0; k < n; ++k) {
        const bool to_pc = (n - k) % 2 == 1;
        launch_pc_jacobi(dp, w, to_pc ? scratch : w.pc, to_pc ? w.pc : scratch, st);
    }
}

// solve_pc_cg (pressure.cpp:208-317) with device-resident scalars.
void Solver::solve_cg() {
    SGPU_CUDA(cudaMemsetAsync(w.pc, 0, g.bytes(), st));
    const double* b0 = at(w.b, prm.H, prm.H + 1);
    launch_ordered_sum(b0, 0, g.pitch, prm.NX, prm.NY, 1, sums, ss, nullptr, st);
    launch_cg_scalars(0, cgs, sums, st);
    launch_cg_init(dp, w, cg, cgs, cells, plane, st);
    launch_ordered_sum(cells, plane, prm.NY, prm.NX, prm.NY, 4, sums, ss, nullptr, st);
    launch_cg_scalars(1, cgs, sums, st);
    launch_cg_dinit(dp, cg, cgs, st);
    const int* done = &cgs->done;
    // Iterations are enqueued in chunks; between chunks the host reads `done` once.
    const int chunk = 16;
    int enqueued = 0;
    while (enqueued < prm.pressure_maxit) {
        const int m = std::min(chunk, prm.pressure_maxit - enqueued);
        for (int it = 0; it < m; ++it) {
            launch_cg_dq(dp, w, cg, cgs, cells, st);
            launch_ordered_sum(cells, plane, prm.NY, prm.NX, prm.NY, 1, sums, ss, done, st);
            launch_cg_scalars(2, cgs, sums, st);
            launch_cg_update(dp, w, cg, cgs, cells, plane, st);
            launch_ordered_sum(cells, plane, prm.NY, prm.NX, prm.NY, 4, sums, ss, done, st);
            launch_cg_scalars(3, cgs, sums, st);
            launch_cg_dir(dp, cg, cgs, st);
        }
        enqueued += m;
        int h = 0;
        SGPU_CUDA(cudaMemcpyAsync(&h, done, sizeof(int), cudaMemcpyDeviceToHost, st));
        sync();
        if (h) break;
    }
    // Remove the mean of the solution (pressure.cpp:311-316).
    const double* x0 = at(w.pc, prm.H, prm.H + 1);
    launch_ordered_sum(x0, 0, g.pitch, prm.NX, prm.NY, 1, sums + 8, ss, nullptr, st);
    LevelView L0{prm.NX, prm.NY, g.pitch, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 nullptr, nullptr};
    launch_mg_sub_mean(L0, at(w.pc, prm.H, prm.H + 1), sums + 8, st);
    cg_stats_pending = true;
}

// remove_mean0 (multigrid.cpp:327-345) on the p' interior.
void Solver::remove_mean0(double* f, const double* known_sum) {
    double* f0 = at(f, prm.H, prm.H + 1);
    if (!known_sum) {
        launch_ordered_sum(f0, 0, g.pitch, prm.NX, prm.NY, 1, sums + 16, ss, nullptr, st);
        known_sum = sums + 16;
    }
    LevelView L0{prm.NX, prm.NY, g.pitch, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 nullptr, nullptr};
    launch_mg_sub_mean(L0, f0, known_sum, st);
}

// mg_vcycle (multigrid.cpp:299-323).
void Solver::mg_vcycle() {
    const int nl = static_cast<int>(lv.size());
    for (int l = 0; l + 1 < nl; ++l) {
        for (int s = 0; s < prm.mg_pre; ++s) {
            launch_mg_smooth_colour(lv[l], 0, st);
            launch_mg_smooth_colour(lv[l], 1, st);
        }
        launch_mg_residual(lv[l], st);
        launch_mg_restrict(lv[l], lv[l + 1], st);
    }
    launch_mg_coarse(lv[nl - 1], coarse_rowbuf, kCoarseTol64, stats, st);
    for (int l = nl - 2; l >= 0; --l) {
        launch_mg_prolong(lv[l + 1], lv[l], prm.mg_omega, st);
        for (int s = 0; s < prm.mg_post; ++s) {
            launch_mg_smooth_colour(lv[l], 0, st);
            launch_mg_smooth_colour(lv[l], 1, st);
        }
    }
}

// solve_pc_mg (multigrid.cpp:347-357).
void Solver::solve_mg() {
    // The streaming V-cycle builds the coarse operators itself unless a warm start reads them first.
    const bool fused_build = mg_fast && !net;
    if (!fused_build)
        for (std::size_t l = 1; l < lv.size(); ++l) launch_mg_build(lv[l - 1], lv[l], st);
    SGPU_CUDA(cudaMemsetAsync(w.pc, 0, g.bytes(), st));
    remove_mean0(w.b, b_sum);
    const bool guess = apply_warm_start(lv[0]);
    last_vcycles = run_cycles(lv[0], !guess, [&](bool x_zero) {
        if (mg_fast) mg_vcycle_fast(x_zero, fused_build);
        else mg_vcycle();
    });
    remove_mean0(w.pc);
}

bool Solver::apply_warm_start(const LevelViewT<double>&) { return net && warm_start_on(lv); }
bool Solver::apply_warm_start(const LevelViewT<float>&) { return net && warm_start_on(lv32); }

// The network's guess on the finest level of at most cnn_max^2 cells (its b restricted from level 0
// by 2x2 sums, its operator the multigrid one), injected back to level 0 as the initial iterate.
template <class T> bool Solver::warm_start_on(std::vector<LevelViewT<T>>& L) {
    const int l = cnn_level(L);
    for (int k = 0; k < l; ++k) launch_restrict_b(L[k], L[k + 1], st);
    net->predict_level(L[l], cells, plane, sums + 30, ss, st);
    for (int k = l - 1; k >= 0; --k) launch_inject_x(L[k + 1], L[k], st);
    ++ws_used;
    return true;
}

// Training pair from the last p' solve: the network input of the warm-start level and the block
// mean of the solved p' there (both normalised as the network sees them).
template <class T> void Solver::sample_pair(std::vector<LevelViewT<T>>& L, float* hin, float* htarget) {
    const int l = cnn_level(L);
    for (int k = 0; k < l; ++k) launch_restrict_b(L[k], L[k + 1], st);
    launch_level_stats(L[l], cells, plane, st);
    launch_ordered_sum(cells, plane, L[l].ny, L[l].nx, L[l].ny, 2, sums + 30, ss, nullptr, st);
    const std::size_t n = static_cast<std::size_t>(L[l].nx) * L[l].ny;
    if (!pair_buf) pair_buf = dalloc<float>(3 * plane);
    launch_make_pair(L[l], L[0], l, sums + 30, pair_buf, pair_buf + 2 * n, st);
    SGPU_CUDA(cudaMemcpyAsync(hin, pair_buf, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, st));
    SGPU_CUDA(cudaMemcpyAsync(htarget, pair_buf + 2 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    SGPU_CUDA(cudaStreamSynchronize(st));
}

// mg_vcycle with the streaming level kernels: levels [0, mg_tail) go down and up in one pass
// each, the rest (and the coarse solve) in the single-CTA tail kernel.
void Solver::mg_vcycle_fast(bool x_is_zero, bool build) {
    const int nl = static_cast<int>(lv.size());
    for (int l = 0; l < mg_tail; ++l)
        launch_mg_down(lv[l], lv[l + 1], mg_x2[l], prm.mg_pre, x_is_zero || l > 0, sms, min_seg, st, build);
    if (build)
        for (int l = mg_tail + 1; l < nl; ++l) launch_mg_build(lv[l - 1], lv[l], st);
    launch_mg_tail(mgl, mg_tail, prm.mg_pre, prm.mg_post, prm.mg_omega, kCoarseTol64, coarse_rowbuf,
                   stats, st);
    for (int l = mg_tail - 1; l >= 0; --l)
        launch_mg_up(lv[l + 1], lv[l], mg_x2[l], lv[l].x, prm.mg_omega, prm.mg_post, sms, min_seg, st);
    (void)nl;
}

void Solver::solve_p() {
    pc_stale = false; // the FP64 p' field is written by this solve
    switch (prm.pressure_solver) {
    case SGPU_P_JACOBI: solve_jacobi(); break;
    case SGPU_P_GS_REDBLACK: solve_redblack(); break;
    case SGPU_P_CG: solve_cg(); break;
    case SGPU_P_MG: solve_mg(); break;
    default: throw Error(SGPU_E_INVALID, "unsupported pressure_solver");
    }
}

} // namespace sgpu

namespace sgpu {

// ---- batched cavities: device-side stopping test inside one graph launch ----

struct BatchDev {
    int n;
    const int* limit;           // a cavity stops after *limit iterations at most
    double* const* res;         // per cavity: its res_u, res_v, res_p of the current iteration
    const double* tol;          // error_tolerance per cavity
    const int* runmax;          // residual_normalisation = running_max per cavity
    double* maxr;               // 3 running maxima per cavity
    int* iters;                 // iterations done per cavity
    int* active;                // 1 while a cavity iterates
    int* converged;             // 1 converged, -1 stopped because a residual became NaN or Inf
    double* last;               // 3 residuals of the last iteration per cavity
    double* log;                // log_cap x 4 per cavity (iteration, res_u, res_v, res_p), or null
    int log_cap;
    cudaGraphConditionalHandle* h; // the IF node of each cavity
    cudaGraphConditionalHandle hw; // the WHILE node around the batch iteration
};

// Start of a batch iteration: each cavity's IF node runs iff the cavity is still active and below
// the iteration limit of this launch.
__global__ void k_batch_pre(const BatchDev* bp) {
    const BatchDev& b = *bp;
    for (int c = threadIdx.x; c < b.n; c += blockDim.x)
        cudaGraphSetConditional(b.h[c], b.active[c] && b.iters[c] < *b.limit ? 1u : 0u);
}

// End of a batch iteration: the stopping rule of run_outer_loop (solver.cpp:117-129) per active
// cavity, with the same arithmetic as the host loop of sgpu_run; the loop continues while any
// cavity is active. A cavity whose residuals are no longer finite stops (converged = -1): the
// reference would run such a diverged cavity on to maxit (its NaNs never pass the test).
__global__ void k_batch_step(const BatchDev* bp) {
    const BatchDev& b = *bp;
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int c = threadIdx.x; c < b.n; c += blockDim.x) {
        if (!b.active[c] || b.iters[c] >= *b.limit) continue; // its IF branch did not run
        const int it = ++b.iters[c];
        const double ru = b.res[c][0], rv = b.res[c][1], rp = b.res[c][2];
        b.last[3 * c + 0] = ru;
        b.last[3 * c + 1] = rv;
        b.last[3 * c + 2] = rp;
        if (b.log && it <= b.log_cap) {
            double* l = b.log + (static_cast<std::size_t>(c) * b.log_cap + (it - 1)) * 4;
            l[0] = it;
            l[1] = ru;
            l[2] = rv;
            l[3] = rp;
        }
        if (!(isfinite(ru) && isfinite(rv) && isfinite(rp))) {
            b.active[c] = 0;
            b.converged[c] = -1;
            continue;
        }
        double tu = ru, tv = rv, tp = rp;
        if (b.runmax[c]) {
            double* m = b.maxr + 3 * c;
            m[0] = m[0] < ru ? ru : m[0];
            m[1] = m[1] < rv ? rv : m[1];
            m[2] = m[2] < rp ? rp : m[2];
            tu = m[0] > 0.0 ? ru / m[0] : 0.0;
            tv = m[1] > 0.0 ? rv / m[1] : 0.0;
            tp = m[2] > 0.0 ? rp / m[2] : 0.0;
        }
        double m = tu;
        if (m < tv) m = tv;
        if (m < tp) m = tp;
        const bool conv = m <= b.tol[c] && it > 1;
        if (conv) { // finished
            b.active[c] = 0;
            b.converged[c] = 1;
        } else if (it < *b.limit) {
            any = 1;
        } // else paused at the limit: a later launch with a higher limit continues it
    }
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(b.hw, any ? 1u : 0u);
}

__global__ void k_set_ints(int* p, int n, int v) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

// WHILE (any solver active) { pre; per solver IF (active) { one outer iteration }; stopping test }.
// Each solver's iteration is captured from its own stream into the body of its IF node, so several
// solvers run as independent branches. The graph is reusable: reset() zeroes the counters and
// launch(limit) runs until every solver has stopped or reached `limit` iterations in total.
struct IterGraph {
    std::vector<Solver*> sv;
    std::vector<void*> dev;
    BatchDev bd{};                // host mirror of the control block
    BatchDev* d_bd = nullptr;     // the kernels read this copy (so the log can grow without a new graph)
    int* d_limit = nullptr;
    double* d_log = nullptr;
    cudaGraphExec_t exec = nullptr;
    int log_cap = 0;
    long long kernels_per_iteration = 0; // launches one captured outer iteration holds, all solvers

    template <class T> T* alloc(std::size_t n) {
        void* p = nullptr;
        SGPU_CUDA(cudaMalloc(&p, sizeof(T) * (n ? n : 1)));
        SGPU_CUDA(cudaMemset(p, 0, sizeof(T) * (n ? n : 1)));
        dev.push_back(p);
        return static_cast<T*>(p);
    }

    IterGraph(std::vector<Solver*> solvers, int cap) : sv(std::move(solvers)) {
        const int n = static_cast<int>(sv.size());
        std::vector<double*> res(n);
        std::vector<double> tol(n);
        std::vector<int> runmax(n);
        for (int c = 0; c < n; ++c) {
            sv[c]->sync();
            res[c] = sv[c]->res_dev;
            tol[c] = sv[c]->prm.error_tolerance;
            runmax[c] = sv[c]->prm.residual_normalisation == SGPU_NORM_RUNNING_MAX ? 1 : 0;
        }
        bd.n = n;
        double** d_res = alloc<double*>(n);
        double* d_tol = alloc<double>(n);
        int* d_runmax = alloc<int>(n);
        SGPU_CUDA(cudaMemcpy(d_res, res.data(), sizeof(double*) * n, cudaMemcpyHostToDevice));
        SGPU_CUDA(cudaMemcpy(d_tol, tol.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        SGPU_CUDA(cudaMemcpy(d_runmax, runmax.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        d_limit = alloc<int>(1);
        bd.limit = d_limit;
        bd.res = d_res;
        bd.tol = d_tol;
        bd.runmax = d_runmax;
        bd.maxr = alloc<double>(3 * static_cast<std::size_t>(n));
        bd.iters = alloc<int>(n);
        bd.active = alloc<int>(n);
        bd.converged = alloc<int>(n);
        bd.last = alloc<double>(3 * static_cast<std::size_t>(n));
        bd.log = nullptr;
        bd.log_cap = 0;
        d_bd = alloc<BatchDev>(1);

        cudaGraph_t g = nullptr;
        try {
            SGPU_CUDA(cudaGraphCreate(&g, 0));
            SGPU_CUDA(cudaGraphConditionalHandleCreate(&bd.hw, g, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams wp{};
            wp.type = cudaGraphNodeTypeConditional;
            wp.conditional.handle = bd.hw;
            wp.conditional.type = cudaGraphCondTypeWhile;
            wp.conditional.size = 1;
            cudaGraphNode_t wnode;
            SGPU_CUDA(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp));
            cudaGraph_t body = wp.conditional.phGraph_out[0];
            std::vector<cudaGraphConditionalHandle> hs(n);
            for (int c = 0; c < n; ++c) SGPU_CUDA(cudaGraphConditionalHandleCreate(&hs[c], body, 0, 0));
            auto* d_h = alloc<cudaGraphConditionalHandle>(n);
            SGPU_CUDA(cudaMemcpy(d_h, hs.data(), sizeof(cudaGraphConditionalHandle) * n, cudaMemcpyHostToDevice));
            bd.h = d_h;
            SGPU_CUDA(cudaMemcpy(d_bd, &bd, sizeof bd, cudaMemcpyHostToDevice));
            void* args[] = {&d_bd};
            cudaKernelNodeParams kp{};
            kp.func = reinterpret_cast<void*>(&k_batch_pre);
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(256);
            kp.kernelParams = args;
            cudaGraphNode_t pre;
            SGPU_CUDA(cudaGraphAddKernelNode(&pre, body, nullptr, 0, &kp));
            std::vector<cudaGraphNode_t> ifs(n);
            for (int c = 0; c < n; ++c) {
                cudaGraphNodeParams ip{};
                ip.type = cudaGraphNodeTypeConditional;
                ip.conditional.handle = hs[c];
                ip.conditional.type = cudaGraphCondTypeIf;
                ip.conditional.size = 1;
                SGPU_CUDA(cudaGraphAddNode(&ifs[c], body, &pre, 1, &ip));
                cudaGraph_t ib = ip.conditional.phGraph_out[0];
                Solver& s = *sv[c];
                SGPU_CUDA(cudaStreamBeginCaptureToGraph(s.st, ib, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
                try {
                    const long long before = g_launches.load();
                    s.iteration_enqueue(s.res_dev);
                    const long long captured = g_launches.load() - before;
                    kernels_per_iteration += captured;
                    count_launches(-captured); // captured, not run: counted when the graph runs
                } catch (...) {
                    cudaGraph_t tmp = nullptr;
                    cudaStreamEndCapture(s.st, &tmp);
                    throw;
                }
                cudaGraph_t captured = nullptr;
                SGPU_CUDA(cudaStreamEndCapture(s.st, &captured));
            }
            kp.func = reinterpret_cast<void*>(&k_batch_step);
            cudaGraphNode_t step;
            SGPU_CUDA(cudaGraphAddKernelNode(&step, body, ifs.data(), ifs.size(), &kp));
            SGPU_CUDA(cudaGraphInstantiate(&exec, g, 0));
        } catch (...) {
            if (g) cudaGraphDestroy(g);
            release();
            throw;
        }
        cudaGraphDestroy(g);
        ensure_log(cap);
    }
    // Residual log of at least cap rows per solver (rows past a solver's iteration count stay zero).
    void ensure_log(int cap) {
        if (cap <= log_cap) return;
        if (d_log) cudaFree(d_log);
        d_log = nullptr;
        const std::size_t n = static_cast<std::size_t>(bd.n) * cap * 4;
        SGPU_CUDA(cudaMalloc(&d_log, sizeof(double) * n));
        SGPU_CUDA(cudaMemset(d_log, 0, sizeof(double) * n));
        log_cap = cap;
        bd.log = d_log;
        bd.log_cap = cap;
        SGPU_CUDA(cudaMemcpy(d_bd, &bd, sizeof bd, cudaMemcpyHostToDevice));
    }
    ~IterGraph() { release(); }
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        for (void* p : dev) cudaFree(p);
        dev.clear();
        if (d_log) cudaFree(d_log);
        d_log = nullptr;
    }
    void reset(cudaStream_t st) {
        const int n = bd.n;
        SGPU_CUDA(cudaMemsetAsync(bd.iters, 0, sizeof(int) * n, st));
        SGPU_CUDA(cudaMemsetAsync(bd.converged, 0, sizeof(int) * n, st));
        SGPU_CUDA(cudaMemsetAsync(bd.last, 0, sizeof(double) * 3 * n, st));
        SGPU_CUDA(cudaMemsetAsync(bd.maxr, 0, sizeof(double) * 3 * n, st));
        if (bd.log) SGPU_CUDA(cudaMemsetAsync(bd.log, 0, sizeof(double) * 4 * n * static_cast<std::size_t>(log_cap), st));
        k_set_ints<<<1, 256, 0, st>>>(bd.active, n, 1);
        SGPU_LAUNCH();
    }
    // Continue a single solver's run that has done `iters` iterations on the host, with the running
    // maxima maxr[3] of its stopping rule (a graph of one solver only). Host copies from pageable
    // memory: synchronous with respect to the host, ordered on st.
    void resume(cudaStream_t st, int iters, const double* maxr) {
        SGPU_CUDA(cudaMemcpyAsync(bd.iters, &iters, sizeof(int), cudaMemcpyHostToDevice, st));
        SGPU_CUDA(cudaMemcpyAsync(bd.maxr, maxr, sizeof(double) * 3, cudaMemcpyHostToDevice, st));
        SGPU_CUDA(cudaStreamSynchronize(st));
    }
    void launch(int limit, cudaStream_t st) {
        k_set_ints<<<1, 32, 0, st>>>(d_limit, 1, limit);
        SGPU_LAUNCH();
        SGPU_CUDA(cudaGraphLaunch(exec, st));
    }
    // Kernel launches the graph performed for `rounds` WHILE iterations that ran `iterations` solver
    // iterations in total: the captured kernels of each solver iteration, and 2 per round.
    void count(long long rounds, long long iterations) const {
        const long long per = sv.empty() ? 0 : kernels_per_iteration / static_cast<long long>(sv.size());
        count_launches(2 * rounds + iterations * per);
    }
};

void destroy_iter_graph(IterGraph* g) {
    if (!g) return;
    cudaDeviceSynchronize();
    delete g;
}

} // namespace sgpu

struct sgpu_handle {
    std::unique_ptr<sgpu::Solver> s;
};
struct sgpu_batch {
    std::vector<std::unique_ptr<sgpu::Solver>> s;
    cudaStream_t st = nullptr;
    std::unique_ptr<sgpu::IterGraph> g; // the graph of the last run (its counters are the results)
    int ran = 0;                        // 1 after sgpu_batch_run
    int last_log_cap = 0;               // log_cap of the last run
    std::vector<int> seg_tuned;         // autotuned row segment per cavity (0: heuristic)
    ~sgpu_batch() {
        if (st) cudaStreamSynchronize(st);
        g.reset();
        s.clear();
        if (st) cudaStreamDestroy(st);
    }
};
struct sgpu_cnn {
    std::unique_ptr<sgpu::UNet> net;
    cudaStream_t st = nullptr;
};

namespace {

template <class F> int guarded(F&& f) {
    try {
        f();
        return SGPU_OK;
    } catch (const sgpu::Error& e) {
        return sgpu::fail(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return sgpu::fail(SGPU_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}

#define SGPU_NEED_HANDLE(h)                                                                  \
    if (!(h) || !(h)->s) return sgpu::fail(SGPU_E_INVALID, "null sgpu handle")

} // namespace

extern "C" {

const char* sgpu_last_error(void) { return sgpu::g_last_error.c_str(); }
const char* sgpu_version(void) { return "simple-b200 0.1 (sm_100a)"; }

int sgpu_create(const sgpu_params_t* p, const double* u, const double* v, const double* pf,
                sgpu_handle** out) {
    if (!p || !out) return sgpu::fail(SGPU_E_INVALID, "sgpu_create: null argument");
    *out = nullptr;
    return guarded([&] {
        auto h = std::make_unique<sgpu_handle>();
        h->s = std::make_unique<sgpu::Solver>(*p, u, v, pf);
        *out = h.release();
    });
}

int sgpu_destroy(sgpu_handle* h) {
    if (!h) return SGPU_OK;
    const int rc = guarded([&] { h->s.reset(); });
    delete h;
    return rc;
}

int sgpu_assemble_u(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->assemble_u(); h->s->sync(); });
}
int sgpu_bc_u(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->bc_u(); h->s->sync(); });
}
int sgpu_residual_u(sgpu_handle* h, double* res) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        h->s->residual_u(h->s->res_dev);
        const double r = h->s->fetch(h->s->res_dev);
        if (res) *res = r;
    });
}
int sgpu_sweep_u(sgpu_handle* h, int n) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->sweep_u(n); h->s->sync(); });
}
int sgpu_assemble_v(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->assemble_v(); h->s->sync(); });
}
int sgpu_bc_v(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->bc_v(); h->s->sync(); });
}
int sgpu_residual_v(sgpu_handle* h, double* res) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        h->s->residual_v(h->s->res_dev + 1);
        const double r = h->s->fetch(h->s->res_dev + 1);
        if (res) *res = r;
    });
}
int sgpu_sweep_v(sgpu_handle* h, int n) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->sweep_v(n); h->s->sync(); });
}
int sgpu_assemble_p(sgpu_handle* h, double* res) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        h->s->assemble_p(h->s->res_dev + 2);
        const double r = h->s->fetch(h->s->res_dev + 2);
        if (res) *res = r;
    });
}
int sgpu_solve_p(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        h->s->solve_p();
        h->s->sync();
        h->s->finish_stats();
    });
}
int sgpu_correct(sgpu_handle* h) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] { h->s->correct(); h->s->sync(); });
}

int sgpu_outer_iteration(sgpu_handle* h, double res[3], double* phase_seconds) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        const bool was = s.profiling;
        if (phase_seconds) s.profiling = true;
        s.iteration_enqueue(s.res_dev);
        SGPU_CUDA(cudaMemcpyAsync(s.host_res, s.res_dev, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                  s.st));
        s.sync();
        s.collect_phases(phase_seconds);
        s.profiling = was;
        if (res) {
            res[0] = s.host_res[0];
            res[1] = s.host_res[1];
            res[2] = s.host_res[2];
        }
    });
}

// sgpu_run without per-iteration host round trips: the iterations run inside one graph launch per
// print interval (sgpu::IterGraph), the stopping rule and the residual log on the device. Used when
// every outer iteration is a fixed sequence of launches (no CG, no tolerance-driven multigrid, no
// warm start) and the per-phase timers are off.
static bool graphable(const sgpu::Solver& s) {
    return s.prm.pressure_solver != SGPU_P_CG && s.prm.mg_mode != SGPU_MG_TOLERANCE && !s.net;
}

// start > 0: the run continues one whose first `start` iterations ran on the host (sampled timers),
// with the stopping rule's running maxima maxr[3]; the log rows from `start` on are filled here.
static bool run_graphed(sgpu::Solver& s, int maxit, double* log, int print_every, sgpu_result_t& out,
                        bool& diverged, int start = 0, const double* maxr = nullptr) {
    if (s.profiling || maxit < 1 || start >= maxit || !graphable(s)) return false;
    if (!s.run_graph) s.run_graph = new sgpu::IterGraph({&s}, maxit);
    sgpu::IterGraph& g = *s.run_graph;
    g.ensure_log(maxit);
    g.reset(s.st);
    if (start > 0) g.resume(s.st, start, maxr);
    const int chunk = print_every > 0 ? print_every : maxit;
    int done = start, conv = 0;
    std::vector<double> rows;
    while (done < maxit) {
        const int lim = std::min(maxit, done + chunk);
        g.launch(lim, s.st);
        int it = 0;
        SGPU_CUDA(cudaMemcpyAsync(&it, g.bd.iters, sizeof(int), cudaMemcpyDeviceToHost, s.st));
        SGPU_CUDA(cudaMemcpyAsync(&conv, g.bd.converged, sizeof(int), cudaMemcpyDeviceToHost, s.st));
        s.sync();
        if (print_every > 0 && it > done) {
            rows.resize(4 * static_cast<std::size_t>(it - done));
            SGPU_CUDA(cudaMemcpy(rows.data(), g.bd.log + 4 * static_cast<std::size_t>(done),
                                 sizeof(double) * rows.size(), cudaMemcpyDeviceToHost));
            for (int k = done + 1; k <= it; ++k)
                if (k == 1 || k % print_every == 0) {
                    const double* r = rows.data() + 4 * static_cast<std::size_t>(k - 1 - done);
                    std::printf("iter %d  res_u %.6e  res_v %.6e  res_p %.6e\n", k, r[1], r[2], r[3]);
                }
        }
        const bool stopped = conv || it < lim;
        done = it;
        if (stopped) break;
    }
    if (log && done > start)
        SGPU_CUDA(cudaMemcpy(log + 4 * static_cast<std::size_t>(start), g.bd.log + 4 * static_cast<std::size_t>(start),
                             sizeof(double) * 4 * static_cast<std::size_t>(done - start), cudaMemcpyDeviceToHost));
    g.count(done - start, done - start);
    out.iterations = done;
    out.converged = conv == 1 ? 1 : 0;
    diverged = conv < 0;
    if (s.prm.pressure_solver == SGPU_P_MG) out.mg_vcycles = static_cast<long long>(done) * s.prm.mg_cycles;
    return true;
}

// Iterations whose phases sampled timers measure (host-issued launches between CUDA events).
constexpr int kSampledIterations = 10;

// A residual that is NaN or Inf ends the run (the reference has no such test and runs a diverged
// case on to maxit, src/solver.cpp:106-132): the result and the log hold the iterations up to and
// including the one that produced it, and the call returns SGPU_E_NONFINITE.
static void raise_nonfinite(const sgpu_result_t& out) {
    throw sgpu::Error(SGPU_E_NONFINITE, "a residual became NaN or Inf at outer iteration " +
                                            std::to_string(out.iterations) + " (the run diverged)");
}

int sgpu_run(sgpu_handle* h, int maxit, double* log, int print_every, sgpu_result_t* result) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        sgpu_result_t out{};
        const auto t0 = std::chrono::steady_clock::now();
        bool diverged = false;
        if (!s.sampled && run_graphed(s, maxit, log, print_every, out, diverged)) {
            out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            s.check_pipeline();
            if (result) *result = out;
            if (diverged) raise_nonfinite(out);
            return;
        }
        double mu = 0.0, mv = 0.0, mp = 0.0;
        // Sampled timers: the host loop runs the first kSampledIterations iterations with the
        // per-phase timers on, then the graph continues the run (graphable solvers only).
        // A solver that cannot replay a graph times every iteration instead.
        const bool sampling = s.sampled && graphable(s) && maxit > kSampledIterations;
        const int host_iters = sampling ? kSampledIterations : maxit;
        if (s.sampled) s.profiling = true;
        bool stopped = false;
        for (int iter = 1; iter <= host_iters; ++iter) {
            s.iteration_enqueue(s.res_dev);
            SGPU_CUDA(cudaMemcpyAsync(s.host_res, s.res_dev, 3 * sizeof(double),
                                      cudaMemcpyDeviceToHost, s.st));
            if (s.cgs)  // CG iterations of this outer iteration (CGWork::last_iterations)
                SGPU_CUDA(cudaMemcpyAsync(s.host_res + 4, &s.cgs->k, sizeof(int),
                                          cudaMemcpyDeviceToHost, s.st));
            s.sync();
            s.collect_phases(out.phase_seconds);
            if (s.cgs) {
                int k = 0;
                std::memcpy(&k, s.host_res + 4, sizeof k);
                out.cg_iterations += k;
                s.cg_stats_pending = false;
                s.last_cg_iterations = k;
            }
            if (s.prm.pressure_solver == SGPU_P_MG) out.mg_vcycles += s.prm.mg_cycles;
            const double ru = s.host_res[0], rv = s.host_res[1], rp = s.host_res[2];
            if (log) {
                log[4 * (iter - 1) + 0] = iter;
                log[4 * (iter - 1) + 1] = ru;
                log[4 * (iter - 1) + 2] = rv;
                log[4 * (iter - 1) + 3] = rp;
            }
            out.iterations = iter;
            if (print_every > 0 && (iter == 1 || iter % print_every == 0))
                std::printf("iter %d  res_u %.6e  res_v %.6e  res_p %.6e\n", iter, ru, rv, rp);
            if (!(std::isfinite(ru) && std::isfinite(rv) && std::isfinite(rp))) {
                diverged = true;
                break;
            }
            // Stopping rule of run_outer_loop (solver.cpp:117-129).
            double tu = ru, tv = rv, tp = rp;
            if (s.prm.residual_normalisation == SGPU_NORM_RUNNING_MAX) {
                mu = mu < ru ? ru : mu;
                mv = mv < rv ? rv : mv;
                mp = mp < rp ? rp : mp;
                tu = mu > 0.0 ? ru / mu : 0.0;
                tv = mv > 0.0 ? rv / mv : 0.0;
                tp = mp > 0.0 ? rp / mp : 0.0;
            }
            double m = tu;
            if (m < tv) m = tv;
            if (m < tp) m = tp;
            if (m <= s.prm.error_tolerance && iter > 1) {
                out.converged = 1;
                break;
            }
        }
        stopped = out.converged || diverged || out.iterations < host_iters;
        if (s.sampled) s.profiling = false;
        if (sampling) {
            if (!stopped) {
                // The graph continues from iteration host_iters + 1; the sampled phase times are
                // scaled to the iterations of the whole run.
                double ph[SGPU_PH_COUNT];
                std::memcpy(ph, out.phase_seconds, sizeof ph);
                const double maxr[3] = {mu, mv, mp};
                run_graphed(s, maxit, log, print_every, out, diverged, host_iters, maxr);
                const double scale = static_cast<double>(out.iterations) / host_iters;
                for (int k = 0; k < SGPU_PH_COUNT; ++k) {
                    out.phase_seconds[k] = ph[k] * scale;
                    s.phase_acc[k] += ph[k] * (scale - 1.0);
                }
            }
        }
        out.seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        s.check_pipeline();
        if (result) *result = out;
        if (diverged) raise_nonfinite(out);
    });
}

int sgpu_download(sgpu_handle* h, int id, double* host) {
    SGPU_NEED_HANDLE(h);
    if (!host) return sgpu::fail(SGPU_E_INVALID, "sgpu_download: null buffer");
    return guarded([&] {
        double* f = h->s->field_ptr(id);
        if (!f) throw sgpu::Error(SGPU_E_INVALID, "sgpu_download: unknown field id " + std::to_string(id));
        h->s->form_p_links_if_stale(id);
        h->s->download(f, host);
    });
}

int sgpu_upload(sgpu_handle* h, int id, const double* host) {
    SGPU_NEED_HANDLE(h);
    if (!host) return sgpu::fail(SGPU_E_INVALID, "sgpu_upload: null buffer");
    return guarded([&] {
        double* f = h->s->field_ptr(id);
        if (!f) throw sgpu::Error(SGPU_E_INVALID, "sgpu_upload: unknown field id " + std::to_string(id));
        h->s->upload(f, host);
        h->s->sync();
    });
}

int sgpu_memory_bytes(sgpu_handle* h, size_t* bytes) {
    SGPU_NEED_HANDLE(h);
    if (bytes) *bytes = h->s->bytes;
    return SGPU_OK;
}

int sgpu_selftest_bounded_wait(int polls, int* gave_up) {
    if (polls < 1 || polls > (1 << 20) || !gave_up)
        return sgpu::fail(SGPU_E_INVALID, "sgpu_selftest_bounded_wait: polls in 1 .. 2^20 and an output");
    return guarded([&] {
        unsigned* err = nullptr;
        SGPU_CUDA(cudaMalloc(&err, sizeof(unsigned)));
        unsigned h = 0;
        try {
            SGPU_CUDA(cudaMemset(err, 0, sizeof(unsigned)));
            sgpu::launch_wait_selftest(polls, err, nullptr);
            SGPU_CUDA(cudaDeviceSynchronize());
            SGPU_CUDA(cudaMemcpy(&h, err, sizeof h, cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(err);
            throw;
        }
        SGPU_CUDA(cudaFree(err));
        *gave_up = h != 0 ? 1 : 0;
    });
}

int sgpu_mg_levels(int NX, int NY, int* nlevels, int* dims) {
    if (NX < 1 || NY < 1 || !nlevels) return sgpu::fail(SGPU_E_INVALID, "sgpu_mg_levels: bad arguments");
    // mg_level_dims (multigrid.cpp:143-151): halve while both are even and the result is >= 4 x 4.
    int nx = NX, ny = NY, n = 0;
    if (dims) {
        dims[0] = nx;
        dims[1] = ny;
    }
    n = 1;
    while (nx % 2 == 0 && ny % 2 == 0 && nx / 2 >= 4 && ny / 2 >= 4 && n < 64) {
        nx /= 2;
        ny /= 2;
        if (dims) {
            dims[2 * n] = nx;
            dims[2 * n + 1] = ny;
        }
        ++n;
    }
    *nlevels = n;
    return SGPU_OK;
}

int sgpu_last_solve_stats(sgpu_handle* h, int* cg_iterations, int* mg_vcycles, int* coarse_sweeps,
                          double* rel_residual) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        if (s.cg_stats_pending && s.cgs) {
            sgpu::CgScalars sc{};
            SGPU_CUDA(cudaMemcpyAsync(&sc, s.cgs, sizeof sc, cudaMemcpyDeviceToHost, s.st));
            s.sync();
            s.last_cg_iterations = sc.k;
            s.last_rel = sc.rel;
            s.cg_stats_pending = false;
        }
        s.finish_stats();
        if (cg_iterations) *cg_iterations = s.last_cg_iterations;
        if (mg_vcycles) *mg_vcycles = s.last_vcycles;
        if (coarse_sweeps) *coarse_sweeps = s.last_coarse_sweeps;
        if (rel_residual) *rel_residual = s.last_rel;
    });
}

int sgpu_ordered_sum(const double* values, int nr, int nc, double* out) {
    if (!values || !out || nr < 0 || nc < 0) return sgpu::fail(SGPU_E_INVALID, "sgpu_ordered_sum: bad arguments");
    return guarded([&] {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
            (void)cudaGetLastError();
            throw sgpu::Error(SGPU_E_NODEVICE, "GPU error: no CUDA device is visible");
        }
        const std::size_t n = static_cast<std::size_t>(nr) * nc;
        double *d = nullptr, *rows = nullptr, *res = nullptr;
        unsigned int* counter = nullptr;
        SGPU_CUDA(cudaMalloc(&d, (n ? n : 1) * sizeof(double)));
        SGPU_CUDA(cudaMalloc(&rows, (nr ? nr : 1) * sizeof(double)));
        SGPU_CUDA(cudaMalloc(&res, sizeof(double)));
        SGPU_CUDA(cudaMalloc(&counter, sizeof(unsigned int)));
        SGPU_CUDA(cudaMemset(counter, 0, sizeof(unsigned int)));
        SGPU_CUDA(cudaMemcpy(d, values, n * sizeof(double), cudaMemcpyHostToDevice));
        sgpu::SumScratch ss;
        ss.rows = rows;
        ss.counter = counter;
        ss.max_rows = nr;
        ss.max_k = 1;
        sgpu::launch_ordered_sum(d, 0, nc, nr, nc, 1, res, ss, nullptr, 0);
        SGPU_CUDA(cudaMemcpy(out, res, sizeof(double), cudaMemcpyDeviceToHost));
        cudaFree(d);
        cudaFree(rows);
        cudaFree(res);
        cudaFree(counter);
    });
}

int sgpu_set_profiling(sgpu_handle* h, int on) {
    SGPU_NEED_HANDLE(h);
    if (on < 0 || on > 2) return sgpu::fail(SGPU_E_INVALID, "sgpu_set_profiling: mode 0, 1 or 2");
    h->s->profiling = on == 1;
    h->s->sampled = on == 2;
    return SGPU_OK;
}

int sgpu_phase_seconds(sgpu_handle* h, double* out) {
    SGPU_NEED_HANDLE(h);
    if (!out) return sgpu::fail(SGPU_E_INVALID, "sgpu_phase_seconds: null output");
    for (int k = 0; k < SGPU_PH_COUNT; ++k) out[k] = h->s->phase_acc[k];
    return SGPU_OK;
}

int sgpu_sweep_seconds(sgpu_handle* h, double* seconds, long long* launches) {
    SGPU_NEED_HANDLE(h);
    if (seconds) *seconds = h->s->sweep_acc;
    if (launches) *launches = h->s->sweep_launches;
    return SGPU_OK;
}

int sgpu_stream(sgpu_handle* h, void** stream) {
    SGPU_NEED_HANDLE(h);
    if (!stream) return sgpu::fail(SGPU_E_INVALID, "sgpu_stream: null output");
    *stream = static_cast<void*>(h->s->st);
    return SGPU_OK;
}

long long sgpu_launch_count(void) { return sgpu::g_launches.load(); }

int sgpu_cnn_load(sgpu_handle* h, const char* path) {
    SGPU_NEED_HANDLE(h);
    if (!path) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_load: null path");
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        if (s.prm.pressure_solver != SGPU_P_MG)
            throw sgpu::Error(SGPU_E_INVALID, "sgpu_cnn_load: the warm start needs pressure_solver = mg");
        s.sync();
        s.own_net = sgpu::UNet::load(path);
        s.net = s.own_net.get();
    });
}

int sgpu_cnn_create(int base, int levels, unsigned seed, sgpu_cnn** out) {
    if (!out) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_create: null output");
    *out = nullptr;
    return guarded([&] {
        auto c = std::make_unique<sgpu_cnn>();
        c->net = std::make_unique<sgpu::UNet>(base, levels, seed);
        SGPU_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        *out = c.release();
    });
}

int sgpu_cnn_read(const char* path, sgpu_cnn** out) {
    if (!out || !path) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_read: null argument");
    *out = nullptr;
    return guarded([&] {
        auto c = std::make_unique<sgpu_cnn>();
        c->net = sgpu::UNet::load(path);
        SGPU_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        *out = c.release();
    });
}

int sgpu_cnn_destroy(sgpu_cnn* c) {
    if (!c) return SGPU_OK;
    const int rc = guarded([&] {
        if (c->st) cudaStreamSynchronize(c->st);
        c->net.reset();
        if (c->st) cudaStreamDestroy(c->st);
    });
    delete c;
    return rc;
}

#define SGPU_NEED_CNN(c)                                                                           \
    do {                                                                                           \
        if (!(c) || !(c)->net) return sgpu::fail(SGPU_E_INVALID, "null network");                  \
    } while (0)

int sgpu_cnn_write(sgpu_cnn* c, const char* path) {
    SGPU_NEED_CNN(c);
    if (!path) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_write: null path");
    return guarded([&] {
        SGPU_CUDA(cudaStreamSynchronize(c->st));
        c->net->save(path);
    });
}

int sgpu_cnn_info(sgpu_cnn* c, int* base, int* levels, long long* num_params, double* flops_per_pixel) {
    SGPU_NEED_CNN(c);
    if (base) *base = c->net->base();
    if (levels) *levels = c->net->levels();
    if (num_params) *num_params = c->net->num_params();
    if (flops_per_pixel) *flops_per_pixel = c->net->flops_per_pixel();
    return SGPU_OK;
}

int sgpu_cnn_get_params(sgpu_cnn* c, float* host) {
    SGPU_NEED_CNN(c);
    if (!host) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_get_params: null buffer");
    return guarded([&] { c->net->get_params(host); });
}

int sgpu_cnn_set_params(sgpu_cnn* c, const float* host) {
    SGPU_NEED_CNN(c);
    if (!host) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_set_params: null buffer");
    return guarded([&] { c->net->set_params(host); });
}

int sgpu_cnn_forward(sgpu_cnn* c, const float* in, int n, int height, int width, float* out) {
    SGPU_NEED_CNN(c);
    if (!in || !out) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_forward: null buffer");
    return guarded([&] {
        c->net->set_input(in, n, height, width, c->st);
        c->net->forward(c->st);
        c->net->get_output(out, c->st);
    });
}

int sgpu_cnn_loss_grad(sgpu_cnn* c, const float* in, const float* target, int n, int height, int width,
                       float* loss, float* grads) {
    SGPU_NEED_CNN(c);
    if (!in || !target) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_loss_grad: null buffer");
    return guarded([&] {
        c->net->set_input(in, n, height, width, c->st);
        c->net->set_target(target, c->st);
        c->net->forward(c->st);
        c->net->backward(c->st);
        const float l = c->net->loss(c->st);
        if (loss) *loss = l;
        if (grads) c->net->get_grads(grads);
    });
}

int sgpu_cnn_train_step(sgpu_cnn* c, const float* in, const float* target, int n, int height, int width,
                        float lr, float* loss) {
    SGPU_NEED_CNN(c);
    if (!in || !target) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_train_step: null buffer");
    if (!(lr > 0.0f)) return sgpu::fail(SGPU_E_INVALID, "sgpu_cnn_train_step: learning rate must be positive");
    return guarded([&] {
        c->net->set_input(in, n, height, width, c->st);
        c->net->set_target(target, c->st);
        c->net->forward(c->st);
        c->net->backward(c->st);
        c->net->adam(lr, c->st);
        const float l = c->net->loss(c->st);
        if (loss) *loss = l;
    });
}

int sgpu_attach_cnn(sgpu_handle* h, sgpu_cnn* c, int max_size) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        if (c && s.prm.pressure_solver != SGPU_P_MG)
            throw sgpu::Error(SGPU_E_INVALID, "sgpu_attach_cnn: the warm start needs pressure_solver = mg");
        if (max_size < 8) throw sgpu::Error(SGPU_E_INVALID, "sgpu_attach_cnn: max_size must be >= 8");
        s.sync();
        if (c) SGPU_CUDA(cudaStreamSynchronize(c->st));
        s.own_net.reset();
        s.net = c ? c->net.get() : nullptr;
        s.cnn_max = max_size;
    });
}

int sgpu_set_mg_mode(sgpu_handle* h, int mg_mode, double pressure_tolerance, int pressure_maxit) {
    SGPU_NEED_HANDLE(h);
    if ((mg_mode != SGPU_MG_FIXED && mg_mode != SGPU_MG_TOLERANCE) || !(pressure_tolerance > 0.0) ||
        pressure_maxit < 1)
        return sgpu::fail(SGPU_E_INVALID, "sgpu_set_mg_mode: bad arguments");
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        s.sync();
        s.prm.mg_mode = mg_mode;
        s.prm.pressure_tolerance = pressure_tolerance;
        s.prm.pressure_maxit = pressure_maxit;
    });
}

int sgpu_warm_start_stats(sgpu_handle* h, long long* used, long long* fallbacks, double* rel_initial) {
    SGPU_NEED_HANDLE(h);
    sgpu::Solver& s = *h->s;
    if (used) *used = s.ws_used;
    if (fallbacks) *fallbacks = s.ws_fallbacks;
    if (rel_initial) *rel_initial = s.last_rel_initial;
    return SGPU_OK;
}

int sgpu_cnn_sample(sgpu_handle* h, int max_size, float* in, float* target, int* nx, int* ny, int* level) {
    SGPU_NEED_HANDLE(h);
    return guarded([&] {
        sgpu::Solver& s = *h->s;
        if (s.prm.pressure_solver != SGPU_P_MG || s.lv.empty())
            throw sgpu::Error(SGPU_E_INVALID, "sgpu_cnn_sample: needs pressure_solver = mg");
        if (max_size < 8) throw sgpu::Error(SGPU_E_INVALID, "sgpu_cnn_sample: max_size must be >= 8");
        s.cnn_max = max_size;
        const int l = s.cnn_level(s.lv);
        if (nx) *nx = s.lv[l].nx;
        if (ny) *ny = s.lv[l].ny;
        if (level) *level = l;
        if (!in || !target) return; // size query
        if (s.mixed)
            throw sgpu::Error(SGPU_E_INVALID, "sgpu_cnn_sample: generate training pairs with precision = fp64");
        s.sync();
        s.sample_pair(s.lv, in, target);
    });
}


// ---- batched cavities ----

#define SGPU_NEED_BATCH(b)                                                                         \
    do {                                                                                           \
        if (!(b) || (b)->s.empty()) return sgpu::fail(SGPU_E_INVALID, "null batch");               \
    } while (0)

int sgpu_batch_create(const sgpu_params_t* params, int count, sgpu_batch** out) {
    if (!params || !out || count < 1) return sgpu::fail(SGPU_E_INVALID, "sgpu_batch_create: bad arguments");
    *out = nullptr;
    return guarded([&] {
        auto b = std::make_unique<sgpu_batch>();
        for (int c = 0; c < count; ++c) {
            const sgpu_params_t& p = params[c];
            const std::string who = "sgpu_batch_create: cavity " + std::to_string(c) + ": ";
            if (p.pressure_solver == SGPU_P_CG)
                throw sgpu::Error(SGPU_E_INVALID, who + "pressure_solver = cg is not supported in a batch");
            if (p.mg_mode == SGPU_MG_TOLERANCE)
                throw sgpu::Error(SGPU_E_INVALID, who + "mg_mode = tolerance is not supported in a batch");
            if (p.warm_start)
                throw sgpu::Error(SGPU_E_INVALID, who + "warm_start = cnn is not supported in a batch");
            b->s.push_back(std::make_unique<sgpu::Solver>(p, nullptr, nullptr, nullptr));
            b->s.back()->use_batch_shape();
        }
        SGPU_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
        b->seg_tuned.assign(count, 0);
        for (auto& sv : b->s) sv->sync();
        *out = b.release();
    });
}

int sgpu_batch_destroy(sgpu_batch* b) {
    if (!b) return SGPU_OK;
    const int rc = guarded([&] { b->s.clear(); });
    delete b;
    return rc;
}

int sgpu_batch_count(sgpu_batch* b, int* count) {
    SGPU_NEED_BATCH(b);
    if (count) *count = static_cast<int>(b->s.size());
    return SGPU_OK;
}

// Autotuner: the row-segment height of the streaming momentum sweep (the tile height of each
// CTA's strip) per distinct grid, timed on the cavity's own scratch buffers.
int sgpu_batch_autotune(sgpu_batch* b, int* chosen) {
    SGPU_NEED_BATCH(b);
    return guarded([&] {
        b->g.reset(); // captured launches carry the old segment heights
        std::map<std::tuple<int, int, int, int>, int> best;
        for (std::size_t c = 0; c < b->s.size(); ++c) {
            sgpu::Solver& sv = *b->s[c];
            if (!sv.fast) continue;
            const auto key = std::make_tuple(sv.prm.NX, sv.prm.NY, sv.dp.ncol, sv.mixed ? 1 : 0);
            auto it = best.find(key);
            if (it == best.end()) {
                const int heur = sv.seg_rows;
                std::vector<int> cand = {heur};
                for (int k : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64})
                    if (8 * sv.dp.ncol * k <= sv.dp.nrows + 8 * sv.dp.ncol) cand.push_back(8 * sv.dp.ncol * k);
                cudaEvent_t e0, e1;
                SGPU_CUDA(cudaEventCreate(&e0));
                SGPU_CUDA(cudaEventCreate(&e1));
                auto sweep = [&](int seg) {
                    if (sv.mixed)
                        sgpu::launch_corr_sweep(sv.dp, false, sv.e32[0], sv.e32[1], sv.rec32, true, seg,
                                                sv.corr_err, sv.st);
                    else sgpu::launch_mom_sweep(sv.dp, false, sv.u, sv.tmp, sv.xF, sv.v, sv.pf, seg, sv.st);
                };
                int pick = heur;
                float tbest = 1e30f;
                for (int seg : cand) {
                    sweep(seg);
                    SGPU_CUDA(cudaEventRecord(e0, sv.st));
                    for (int r = 0; r < 5; ++r) sweep(seg);
                    SGPU_CUDA(cudaEventRecord(e1, sv.st));
                    SGPU_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    SGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (ms < tbest) {
                        tbest = ms;
                        pick = seg;
                    }
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                it = best.emplace(key, pick).first;
            }
            sv.seg_rows = it->second;
            b->seg_tuned[c] = it->second;
        }
        if (chosen)
            for (std::size_t c = 0; c < b->s.size(); ++c) chosen[c] = b->seg_tuned[c];
    });
}

// All cavities in one graph launch: WHILE (any cavity active) { per cavity: IF (active) { one outer
// iteration }; stopping test }. Each cavity's iteration is captured from its own solver into the
// body of its IF node, so the cavities run as independent branches.
int sgpu_batch_run(sgpu_batch* b, int maxit, int log_cap, double* seconds) {
    SGPU_NEED_BATCH(b);
    if (maxit < 0 || log_cap < 0) return sgpu::fail(SGPU_E_INVALID, "sgpu_batch_run: bad arguments");
    return guarded([&] {
        std::vector<sgpu::Solver*> sv;
        for (auto& p : b->s) sv.push_back(p.get());
        if (!b->g) b->g = std::make_unique<sgpu::IterGraph>(sv, log_cap);
        b->g->ensure_log(log_cap);
        b->g->reset(b->st);
        b->ran = 1;
        b->last_log_cap = log_cap;
        if (maxit == 0) {
            if (seconds) *seconds = 0.0;
            SGPU_CUDA(cudaStreamSynchronize(b->st));
            return;
        }
        cudaEvent_t e0, e1;
        SGPU_CUDA(cudaEventCreate(&e0));
        SGPU_CUDA(cudaEventCreate(&e1));
        SGPU_CUDA(cudaEventRecord(e0, b->st));
        b->g->launch(maxit, b->st);
        SGPU_CUDA(cudaEventRecord(e1, b->st));
        SGPU_CUDA(cudaEventSynchronize(e1));
        {
            const int n = static_cast<int>(b->s.size());
            std::vector<int> its(n);
            SGPU_CUDA(cudaMemcpy(its.data(), b->g->bd.iters, sizeof(int) * n, cudaMemcpyDeviceToHost));
            long long total = 0, rounds = 0;
            for (int v : its) {
                total += v;
                rounds = std::max<long long>(rounds, v);
            }
            b->g->count(rounds, total); // cavities differ in kernels per iteration: an average
        }
        for (auto& p : b->s) p->check_pipeline();
        float ms = 0.0f;
        SGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (seconds) *seconds = ms * 1e-3;
    });
}

int sgpu_batch_results(sgpu_batch* b, int* iterations, int* converged, double* residuals) {
    SGPU_NEED_BATCH(b);
    if (!b->ran) return sgpu::fail(SGPU_E_INVALID, "sgpu_batch_results: the batch has not run");
    return guarded([&] {
        const int n = static_cast<int>(b->s.size());
        const sgpu::BatchDev& bd = b->g->bd;
        if (iterations)
            SGPU_CUDA(cudaMemcpyAsync(iterations, bd.iters, sizeof(int) * n, cudaMemcpyDeviceToHost, b->st));
        if (converged)
            SGPU_CUDA(cudaMemcpyAsync(converged, bd.converged, sizeof(int) * n, cudaMemcpyDeviceToHost, b->st));
        if (residuals)
            SGPU_CUDA(cudaMemcpyAsync(residuals, bd.last, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, b->st));
        SGPU_CUDA(cudaStreamSynchronize(b->st));
    });
}

int sgpu_batch_log(sgpu_batch* b, double* host) {
    SGPU_NEED_BATCH(b);
    if (!host || !b->g || !b->g->bd.log)
        return sgpu::fail(SGPU_E_INVALID, "sgpu_batch_log: no log (run with log_cap > 0)");
    return guarded([&] {
        // rows of the requested log_cap of the last run (the buffer may be longer)
        const int cap = b->g->log_cap;
        for (std::size_t c = 0; c < b->s.size(); ++c)
            SGPU_CUDA(cudaMemcpyAsync(host + c * static_cast<std::size_t>(b->last_log_cap) * 4,
                                      b->g->bd.log + c * static_cast<std::size_t>(cap) * 4,
                                      sizeof(double) * 4 * static_cast<std::size_t>(b->last_log_cap),
                                      cudaMemcpyDeviceToHost, b->st));
        SGPU_CUDA(cudaStreamSynchronize(b->st));
    });
}

int sgpu_batch_download(sgpu_batch* b, int index, int field_id, double* host) {
    SGPU_NEED_BATCH(b);
    if (index < 0 || index >= static_cast<int>(b->s.size()) || !host)
        return sgpu::fail(SGPU_E_INVALID, "sgpu_batch_download: bad arguments");
    return guarded([&] {
        SGPU_CUDA(cudaStreamSynchronize(b->st));
        sgpu::Solver& sv = *b->s[index];
        double* f = sv.field_ptr(field_id);
        if (!f) throw sgpu::Error(SGPU_E_INVALID, "sgpu_batch_download: unknown field id " + std::to_string(field_id));
        sv.form_p_links_if_stale(field_id);
        sv.download(f, host);
    });
}

} // extern "C"
