// io.cpp — the reference's output files, written from host arrays (write_outputs, src/io.cpp:43-151).
//
// Same file names, formats and number formatting as the reference, so post-processing written for
// simple-hpc reads this build's results unchanged:
//   u.csv v.csv p.csv        full stored arrays, halos included, "%.18e" comma-separated (:10-20)
//   ux_centre.csv uy_centre.csv   cell-centre velocities, NX x NY (cell_centre, :22-31)
//   alog.csv                 "Iteration,Residual_u,Residual_v,Residual_p" then "%d,%.18e,..." (:61-68)
//   timing.csv               phase,seconds,fraction with total and unaccounted rows (:71-90)
//   run_info.json            the reference's keys in the reference's order (:104-150)
// The field CSVs are formatted in parallel row blocks (each block formatted into its own buffer,
// then written in order), which gives the same bytes as the reference's sequential fprintf.
#include "common.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <thread>
#include <vector>

namespace sgpu {

namespace {

const char* phase_name(int ph) {
    static const char* names[] = {"assemble_u", "bc_u",       "residual_u", "sweep_u",
                                  "assemble_v", "bc_v",       "residual_v", "sweep_v",
                                  "assemble_p", "solve_p",    "correct",    "output"};
    return (ph >= 0 && ph < SGPU_PH_COUNT) ? names[ph] : "?";
}

// Rows [r0, r1) of a rows x cols array as the reference's write_csv formats them.
void format_rows(const double* a, int r0, int r1, int cols, std::string& out) {
    char buf[40];
    for (int i = r0; i < r1; ++i) {
        for (int j = 0; j < cols; ++j) {
            const int n = std::snprintf(buf, sizeof buf, j ? ",%.18e" : "%.18e",
                                        a[static_cast<std::size_t>(i) * cols + j]);
            out.append(buf, static_cast<std::size_t>(n));
        }
        out.push_back('\n');
    }
}

void write_csv(const std::string& path, const double* a, int rows, int cols) {
    std::FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) throw Error(SGPU_E_INVALID, "cannot open for writing: " + path);
    const int nt = std::max(1, std::min<int>(static_cast<int>(std::thread::hardware_concurrency()), 32));
    const int block = 64;
    std::vector<std::string> bufs(static_cast<std::size_t>(nt));
    for (int base = 0; base < rows; base += block * nt) {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) {
            const int r0 = base + t * block, r1 = std::min(rows, r0 + block);
            bufs[t].clear();
            if (r0 >= r1) continue;
            th.emplace_back([&, t, r0, r1] { format_rows(a, r0, r1, cols, bufs[t]); });
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < nt; ++t)
            if (!bufs[t].empty()) std::fwrite(bufs[t].data(), 1, bufs[t].size(), fp);
    }
    std::fclose(fp);
}

std::string esc(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

const char* name_conv(int c) { return c == SGPU_UDS ? "UDS" : "QUICK"; }
const char* name_backend(int b) {
    return b == SGPU_BACKEND_SERIAL ? "serial" : b == SGPU_BACKEND_OPENMP ? "openmp" : "gpu";
}
const char* name_mom(int m) {
    return m == SGPU_MOM_GS_LEX ? "gs_lex" : m == SGPU_MOM_JACOBI ? "jacobi" : "gs_multicolour";
}
const char* name_p(int s) {
    return s == SGPU_P_GS_LEX        ? "gs_lex"
           : s == SGPU_P_JACOBI      ? "jacobi"
           : s == SGPU_P_GS_REDBLACK ? "gs_redblack"
           : s == SGPU_P_CG          ? "cg"
                                     : "mg";
}

} // namespace

void write_outputs(const sgpu_params_t& p, const double* u, const double* v, const double* pf,
                   const double* log, int iterations, const sgpu_result_t& r,
                   const std::string& cfg_path, const std::string& git_hash,
                   const std::string& compiler, int threads) {
    namespace fs = std::filesystem;
    double seconds_phase[SGPU_PH_COUNT];
    std::memcpy(seconds_phase, r.phase_seconds, sizeof seconds_phase);
    const fs::path d(p.output_dir);
    const auto t_out = std::chrono::steady_clock::now();
    fs::create_directories(d);
    if (p.write_fields) {
        write_csv((d / "u.csv").string(), u, p.nrows, p.ncols);
        write_csv((d / "v.csv").string(), v, p.nrows, p.ncols);
        write_csv((d / "p.csv").string(), pf, p.nrows, p.ncols);
        // cell_centre (io.cpp:22-31).
        const int H = p.H;
        std::vector<double> ux(static_cast<std::size_t>(p.NX) * p.NY), uy(ux.size());
        for (int rr = 0; rr < p.NX; ++rr)
            for (int c = 0; c < p.NY; ++c) {
                const std::size_t k = static_cast<std::size_t>(rr) * p.NY + c;
                ux[k] = (u[static_cast<std::size_t>(H + rr) * p.ncols + H + c] +
                         u[static_cast<std::size_t>(H + rr) * p.ncols + H + c + 1]) / 2;
                uy[k] = (v[static_cast<std::size_t>(H + rr) * p.ncols + H + 1 + c] +
                         v[static_cast<std::size_t>(H + rr + 1) * p.ncols + H + 1 + c]) / 2;
            }
        write_csv((d / "ux_centre.csv").string(), ux.data(), p.NX, p.NY);
        write_csv((d / "uy_centre.csv").string(), uy.data(), p.NX, p.NY);
    }
    {
        std::FILE* al = std::fopen((d / "alog.csv").string().c_str(), "w");
        if (!al) throw Error(SGPU_E_INVALID, "cannot write alog.csv");
        std::fputs("Iteration,Residual_u,Residual_v,Residual_p\n", al);
        for (int k = 0; k < iterations; ++k)
            std::fprintf(al, "%d,%.18e,%.18e,%.18e\n", static_cast<int>(log[4 * k]), log[4 * k + 1],
                         log[4 * k + 2], log[4 * k + 3]);
        std::fclose(al);
    }
    seconds_phase[SGPU_PH_OUTPUT] +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_out).count();
    {
        double total = 0.0;
        for (double x : seconds_phase) total += x;
        const double timed = total - seconds_phase[SGPU_PH_OUTPUT];
        std::FILE* tf = std::fopen((d / "timing.csv").string().c_str(), "w");
        if (!tf) throw Error(SGPU_E_INVALID, "cannot write timing.csv");
        std::fputs("phase,seconds,fraction\n", tf);
        const double denom = total > 0.0 ? total : 1.0;
        for (int i = 0; i < SGPU_PH_COUNT; ++i)
            std::fprintf(tf, "%s,%.9f,%.6f\n", phase_name(i), seconds_phase[i], seconds_phase[i] / denom);
        std::fprintf(tf, "total,%.9f,1.000000\n", total);
        std::fprintf(tf, "unaccounted,%.9f,%.6f\n", r.seconds - timed,
                     r.seconds > 0.0 ? (r.seconds - timed) / r.seconds : 0.0);
        std::fclose(tf);
    }
    std::FILE* fp = std::fopen((d / "run_info.json").string().c_str(), "w");
    if (!fp) throw Error(SGPU_E_INVALID, "cannot write run_info.json");
    std::fprintf(fp, "{\n  \"config\": \"%s\",\n  \"git_hash\": \"%s\",\n", esc(cfg_path).c_str(),
                 git_hash.c_str());
    std::fprintf(fp, "  \"compiler\": \"%s\",\n", compiler.c_str());
    std::fprintf(fp, "  \"backend\": \"%s\",\n  \"threads\": %d,\n", name_backend(p.backend), threads);
    std::fprintf(fp, "  \"momentum_solver\": \"%s\",\n  \"pressure_solver\": \"%s\",\n",
                 name_mom(p.momentum_solver), name_p(p.pressure_solver));
    std::fprintf(fp, "  \"N_cells_x\": %d,\n  \"N_cells_y\": %d,\n  \"N_halo_x\": %d,\n", p.NX, p.NY,
                 p.N_halo_x);
    std::fprintf(fp, "  \"N_halo_y\": %d,\n  \"Re\": %.17g,\n", p.N_halo_y, p.Re);
    std::fprintf(fp, "  \"maxit_inner_u\": %d,\n  \"maxit_inner_v\": %d,\n", p.maxit_inner_u,
                 p.maxit_inner_v);
    std::fprintf(fp, "  \"maxit_inner_p\": %d,\n  \"error_tolerance\": %.17g,\n", p.maxit_inner_p,
                 p.error_tolerance);
    std::fprintf(fp, "  \"maxit\": %d,\n", p.maxit);
    std::fprintf(fp, "  \"relaxation_factor_u\": %.17g,\n  \"relaxation_factor_v\": %.17g,\n",
                 p.relaxation_factor_u, p.relaxation_factor_v);
    std::fprintf(fp, "  \"relaxation_factor_p\": %.17g,\n", p.relaxation_factor_p);
    std::fprintf(fp, "  \"convection_scheme\": \"%s\",\n  \"diffusion_order\": %d,\n",
                 name_conv(p.convection_scheme), p.diffusion_order);
    std::fprintf(fp, "  \"Hybrid_switch\": %s,\n", p.hybrid_switch ? "true" : "false");
    std::fprintf(fp, "  \"residual_normalisation\": \"%s\",\n",
                 p.residual_normalisation == SGPU_NORM_ABSOLUTE ? "absolute" : "running_max");
    std::fprintf(fp, "  \"output_dir\": \"%s\",\n", esc(p.output_dir).c_str());
    std::fprintf(fp, "  \"pressure_tolerance\": %.17g,\n  \"pressure_maxit\": %d,\n",
                 p.pressure_tolerance, p.pressure_maxit);
    std::fprintf(fp, "  \"mg_cycles\": %d,\n  \"mg_pre\": %d,\n  \"mg_post\": %d,\n", p.mg_cycles,
                 p.mg_pre, p.mg_post);
    std::fprintf(fp, "  \"mg_omega\": %.17g,\n", p.mg_omega);
    std::fprintf(fp, "  \"cg_iterations_total\": %lld,\n  \"cg_iterations_mean\": %.6f,\n",
                 r.cg_iterations,
                 r.iterations > 0 ? static_cast<double>(r.cg_iterations) / r.iterations : 0.0);
    std::fprintf(fp, "  \"ranks\": %d,\n", 1);
    std::fprintf(fp, "  \"halo_seconds_mean\": %.6f,\n  \"halo_seconds_max\": %.6f,\n", 0.0, 0.0);
    std::fprintf(fp, "  \"collective_seconds_mean\": %.6f,\n  \"collective_seconds_max\": %.6f,\n",
                 0.0, 0.0);
    std::fprintf(fp,
                 "  \"iterations\": %d,\n  \"converged\": %s,\n  \"seconds\": %.6f,\n  "
                 "\"seconds_per_iteration\": %.9f\n}\n",
                 r.iterations, r.converged ? "true" : "false", r.seconds,
                 r.iterations > 0 ? r.seconds / r.iterations : 0.0);
    std::fclose(fp);
}

// Reads a rows x cols CSV of doubles (the format write_csv writes: comma-separated, one line per
// row). Rows are parsed in parallel blocks once their line starts are known.
void read_csv(const std::string& path, double* out, int rows, int cols) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw Error(SGPU_E_INVALID, "restart: cannot read " + path);
    std::string text;
    {
        std::fseek(fp, 0, SEEK_END);
        const long n = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        text.resize(n > 0 ? static_cast<std::size_t>(n) : 0);
        const std::size_t got = n > 0 ? std::fread(&text[0], 1, text.size(), fp) : 0;
        std::fclose(fp);
        if (got != text.size()) throw Error(SGPU_E_INVALID, "restart: short read of " + path);
    }
    std::vector<std::size_t> starts;
    starts.reserve(static_cast<std::size_t>(rows) + 1);
    std::size_t pos = 0;
    while (pos < text.size()) {
        starts.push_back(pos);
        const std::size_t nl = text.find('\n', pos);
        pos = nl == std::string::npos ? text.size() : nl + 1;
    }
    if (static_cast<int>(starts.size()) != rows)
        throw Error(SGPU_E_INVALID, "restart: " + path + " has " + std::to_string(starts.size()) +
                                        " rows, the configuration needs " + std::to_string(rows));
    starts.push_back(text.size());
    const int nt = std::max(1, std::min<int>(static_cast<int>(std::thread::hardware_concurrency()), 32));
    std::vector<std::string> errors(static_cast<std::size_t>(nt));
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (int i = t; i < rows && errors[t].empty(); i += nt) {
                const char* c = text.c_str() + starts[i];
                const char* end = text.c_str() + starts[i + 1];
                for (int j = 0; j < cols; ++j) {
                    char* stop = nullptr;
                    const double val = std::strtod(c, &stop);
                    const bool sep_ok = j + 1 < cols ? (stop < end && *stop == ',')
                                                     : (stop == end || *stop == '\n' || *stop == '\r');
                    if (stop == c || !sep_ok) {
                        errors[t] = "restart: " + path + " row " + std::to_string(i + 1) +
                                    ": expected " + std::to_string(cols) + " comma-separated numbers";
                        break;
                    }
                    out[static_cast<std::size_t>(i) * cols + j] = val;
                    c = stop + 1;
                }
            }
        });
    for (auto& x : th) x.join();
    for (const auto& e : errors)
        if (!e.empty()) throw Error(SGPU_E_INVALID, e);
}

} // namespace sgpu

extern "C" int sgpu_read_fields(const sgpu_params_t* p, const char* dir, double* u, double* v, double* pf) {
    if (!p || !dir || !u || !v || !pf) return sgpu::fail(SGPU_E_INVALID, "sgpu_read_fields: null argument");
    try {
        const std::filesystem::path d(dir);
        sgpu::read_csv((d / "u.csv").string(), u, p->nrows, p->ncols);
        sgpu::read_csv((d / "v.csv").string(), v, p->nrows, p->ncols);
        sgpu::read_csv((d / "p.csv").string(), pf, p->nrows, p->ncols);
        return SGPU_OK;
    } catch (const sgpu::Error& e) {
        return sgpu::fail(e.code, e.what());
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}

extern "C" int sgpu_write_outputs(const sgpu_params_t* p, const double* u, const double* v,
                                  const double* pf, const double* log, int iterations,
                                  const sgpu_result_t* result, const char* cfg_path,
                                  const char* git_hash, const char* compiler) {
    if (!p || !u || !v || !pf || !result || (iterations > 0 && !log))
        return sgpu::fail(SGPU_E_INVALID, "sgpu_write_outputs: null argument");
    try {
        sgpu::write_outputs(*p, u, v, pf, log, iterations, *result, cfg_path ? cfg_path : "",
                            git_hash ? git_hash : "unknown", compiler ? compiler : "unknown", 1);
        return SGPU_OK;
    } catch (const sgpu::Error& e) {
        return sgpu::fail(e.code, e.what());
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}
