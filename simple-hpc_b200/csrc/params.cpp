// params.cpp — config text -> sgpu_params_t, keeping the reference's keys, defaults and messages.
//
// Parsing follows parse_config (src/config.cpp:16-39): '#' starts a comment, blank lines are
// skipped, each other line is "key = value" with surrounding whitespace trimmed, and a missing '=',
// an empty key or value, or a repeated key is an error naming the line. Building the parameters
// follows make_params (src/params.cpp:50-180): a whitelist of keys, integer / number / True|False /
// enum parsing with the reference's messages, validation, and the derived nrows, ncols, dx, dy, nu.
// Keys added by this build (precision, mg_mode, warm_start, cnn_weights, graph_batch, restart_from) are accepted
// here only; every reference key keeps its meaning and default.
#include "common.hpp"

#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace sgpu {

namespace {

std::string trim_ws(const std::string& s) {
    const char* ws = " \t\r\n";
    const std::size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return "";
    return s.substr(b, s.find_last_not_of(ws) - b + 1);
}

// Ordered (key, value) pairs of a config text.
std::vector<std::pair<std::string, std::string>> parse_lines(const std::string& text) {
    std::vector<std::pair<std::string, std::string>> kv;
    std::set<std::string> seen;
    std::size_t pos = 0;
    int lineno = 0;
    while (pos <= text.size()) {
        std::size_t nl = text.find('\n', pos);
        if (nl == std::string::npos) nl = text.size();
        std::string line = text.substr(pos, nl - pos);
        pos = nl + 1;
        ++lineno;
        const std::size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        line = trim_ws(line);
        if (line.empty()) {
            if (nl == text.size()) break;
            continue;
        }
        const std::string where = "config line " + std::to_string(lineno) + ": ";
        const std::size_t eq = line.find('=');
        if (eq == std::string::npos)
            throw std::runtime_error(where + "malformed line (expected key = value)");
        std::string key = trim_ws(line.substr(0, eq)), val = trim_ws(line.substr(eq + 1));
        if (key.empty() || val.empty())
            throw std::runtime_error(where + "malformed line (empty key or value)");
        if (!seen.insert(key).second)
            throw std::runtime_error(where + "duplicate key '" + key + "'");
        kv.emplace_back(std::move(key), std::move(val));
        if (nl == text.size()) break;
    }
    return kv;
}

int parse_int(const std::string& k, const std::string& v) {
    try {
        std::size_t used = 0;
        const int r = std::stoi(v, &used);
        if (used != v.size()) throw std::invalid_argument("trailing");
        return r;
    } catch (const std::exception&) {
        throw std::runtime_error("cannot parse integer for '" + k + "': " + v);
    }
}

double parse_num(const std::string& k, const std::string& v) {
    try {
        std::size_t used = 0;
        const double r = std::stod(v, &used);
        if (used != v.size()) throw std::invalid_argument("trailing");
        return r;
    } catch (const std::exception&) {
        throw std::runtime_error("cannot parse number for '" + k + "': " + v);
    }
}

bool parse_bool(const std::string& k, const std::string& v) {
    if (v == "True") return true;
    if (v == "False") return false;
    throw std::runtime_error("invalid boolean for '" + k + "' (use True/False): " + v);
}

int parse_choice(const std::string& k, const std::string& v,
                 std::initializer_list<std::pair<const char*, int>> options) {
    for (const auto& o : options)
        if (v == o.first) return o.second;
    throw std::runtime_error("unknown value for '" + k + "': " + v);
}

void copy_str(char* dst, std::size_t cap, const std::string& s) {
    if (s.size() + 1 > cap) throw std::runtime_error("value too long: " + s);
    std::memcpy(dst, s.c_str(), s.size() + 1);
}

} // namespace

void params_defaults(sgpu_params_t& p) {
    std::memset(&p, 0, sizeof p);
    // struct Params defaults (include/simple/params.hpp:16-36).
    p.NX = 80;
    p.NY = 80;
    p.H = 2;
    p.N_halo_x = 2;
    p.N_halo_y = 2;
    p.Re = 1000.0;
    p.maxit_inner_u = 4;
    p.maxit_inner_v = 4;
    p.maxit_inner_p = 8;
    p.error_tolerance = 1e-4;
    p.maxit = 15000;
    p.relaxation_factor_u = 0.3;
    p.relaxation_factor_v = 0.3;
    p.relaxation_factor_p = 0.2;
    p.convection_scheme = SGPU_QUICK;
    p.diffusion_order = 4;
    p.hybrid_switch = 0;
    p.residual_normalisation = SGPU_NORM_ABSOLUTE;
    p.backend = SGPU_BACKEND_SERIAL;
    p.momentum_solver = SGPU_MOM_GS_LEX;
    p.pressure_solver = SGPU_P_GS_LEX;
    p.pressure_tolerance = 1e-6;
    p.pressure_maxit = 1000;
    p.mg_cycles = 1;
    p.mg_pre = 2;
    p.mg_post = 2;
    p.mg_omega = 1.8;
    p.halo_overlap = 1;
    p.write_fields = 1;
    p.precision = SGPU_PREC_FP64;
    p.mg_mode = SGPU_MG_FIXED;
    p.warm_start = 0;
    p.graph_batch = 0;
    copy_str(p.output_dir, sizeof p.output_dir, "results/run");
}

void params_finalize(sgpu_params_t& p) {
    // Validation and derived values: src/params.cpp:152-178, in the same order.
    if (p.N_halo_x != p.N_halo_y) throw std::runtime_error("N_halo_x must equal N_halo_y");
    p.H = p.N_halo_x;
    if (p.H < 2) throw std::runtime_error("halo width H must be >= 2");
    if (p.diffusion_order != 2 && p.diffusion_order != 4)
        throw std::runtime_error("diffusion_order must be 2 or 4");
    if (p.NX < 1 || p.NY < 1) throw std::runtime_error("N_cells_x and N_cells_y must be positive");
    if (p.hybrid_switch) throw std::runtime_error("Hybrid_switch = True is not supported");
    if (!(p.pressure_tolerance > 0.0)) throw std::runtime_error("pressure_tolerance must be positive");
    if (p.pressure_maxit < 1) throw std::runtime_error("pressure_maxit must be >= 1");
    if (p.mg_cycles < 1) throw std::runtime_error("mg_cycles must be >= 1");
    if (p.mg_pre < 0 || p.mg_post < 0) throw std::runtime_error("mg_pre and mg_post must be >= 0");
    if (!(p.mg_omega > 0.0 && p.mg_omega <= 2.0)) throw std::runtime_error("mg_omega must be in (0, 2]");
    if (p.graph_batch < 0) throw std::runtime_error("graph_batch must be >= 0");
    p.nrows = p.NX + 2 * p.H + 1;
    p.ncols = p.NY + 2 * p.H + 1;
    p.dx = 1.0 / p.NY; // column spacing
    p.dy = 1.0 / p.NX; // row spacing
    p.nu = 1.0 / p.Re;
}

void params_from_config(const std::string& text, sgpu_params_t& p) {
    const auto kv = parse_lines(text);
    static const std::set<std::string> known = {
        // the reference's whitelist (src/params.cpp:51-58)
        "N_cells_x", "N_cells_y", "N_halo_x", "N_halo_y", "Re", "maxit_inner_u", "maxit_inner_v",
        "maxit_inner_p", "error_tolerance", "maxit", "relaxation_factor_u", "relaxation_factor_v",
        "relaxation_factor_p", "convection_scheme", "diffusion_order", "Hybrid_switch", "backend",
        "momentum_solver", "pressure_solver", "output_dir", "residual_normalisation",
        "pressure_tolerance", "pressure_maxit", "mg_cycles", "mg_pre", "mg_post", "mg_omega",
        "mpi_grid", "halo_overlap", "write_fields",
        // this build
        "precision", "mg_mode", "warm_start", "cnn_weights", "graph_batch", "restart_from"};
    // The reference iterates a std::map, so the first unknown key in sorted order is reported.
    std::map<std::string, std::string> sorted(kv.begin(), kv.end());
    for (const auto& e : sorted)
        if (!known.count(e.first)) throw std::runtime_error("unknown config key: " + e.first);

    params_defaults(p);
    for (const auto& e : sorted) {
        const std::string& k = e.first;
        const std::string& v = e.second;
        if (k == "N_cells_x") p.NX = parse_int(k, v);
        else if (k == "N_cells_y") p.NY = parse_int(k, v);
        else if (k == "N_halo_x") p.N_halo_x = parse_int(k, v);
        else if (k == "N_halo_y") p.N_halo_y = parse_int(k, v);
        else if (k == "Re") p.Re = parse_num(k, v);
        else if (k == "maxit_inner_u") p.maxit_inner_u = parse_int(k, v);
        else if (k == "maxit_inner_v") p.maxit_inner_v = parse_int(k, v);
        else if (k == "maxit_inner_p") p.maxit_inner_p = parse_int(k, v);
        else if (k == "error_tolerance") p.error_tolerance = parse_num(k, v);
        else if (k == "maxit") p.maxit = parse_int(k, v);
        else if (k == "relaxation_factor_u") p.relaxation_factor_u = parse_num(k, v);
        else if (k == "relaxation_factor_v") p.relaxation_factor_v = parse_num(k, v);
        else if (k == "relaxation_factor_p") p.relaxation_factor_p = parse_num(k, v);
        else if (k == "convection_scheme")
            p.convection_scheme = parse_choice(k, v, {{"UDS", SGPU_UDS}, {"QUICK", SGPU_QUICK}});
        else if (k == "diffusion_order") p.diffusion_order = parse_int(k, v);
        else if (k == "Hybrid_switch") p.hybrid_switch = parse_bool(k, v) ? 1 : 0;
        else if (k == "backend")
            p.backend = parse_choice(k, v, {{"serial", SGPU_BACKEND_SERIAL},
                                            {"openmp", SGPU_BACKEND_OPENMP},
                                            {"gpu", SGPU_BACKEND_GPU}});
        else if (k == "momentum_solver")
            p.momentum_solver = parse_choice(k, v, {{"gs_lex", SGPU_MOM_GS_LEX},
                                                    {"jacobi", SGPU_MOM_JACOBI},
                                                    {"gs_multicolour", SGPU_MOM_GS_MULTICOLOUR}});
        else if (k == "pressure_solver")
            p.pressure_solver = parse_choice(k, v, {{"gs_lex", SGPU_P_GS_LEX},
                                                    {"jacobi", SGPU_P_JACOBI},
                                                    {"gs_redblack", SGPU_P_GS_REDBLACK},
                                                    {"cg", SGPU_P_CG},
                                                    {"mg", SGPU_P_MG}});
        else if (k == "residual_normalisation")
            p.residual_normalisation = parse_choice(
                k, v, {{"absolute", SGPU_NORM_ABSOLUTE}, {"running_max", SGPU_NORM_RUNNING_MAX}});
        else if (k == "output_dir") copy_str(p.output_dir, sizeof p.output_dir, v);
        else if (k == "pressure_tolerance") p.pressure_tolerance = parse_num(k, v);
        else if (k == "pressure_maxit") p.pressure_maxit = parse_int(k, v);
        else if (k == "mg_cycles") p.mg_cycles = parse_int(k, v);
        else if (k == "mg_pre") p.mg_pre = parse_int(k, v);
        else if (k == "mg_post") p.mg_post = parse_int(k, v);
        else if (k == "mg_omega") p.mg_omega = parse_num(k, v);
        else if (k == "halo_overlap") p.halo_overlap = parse_bool(k, v) ? 1 : 0;
        else if (k == "write_fields") p.write_fields = parse_bool(k, v) ? 1 : 0;
        else if (k == "mpi_grid" && v != "auto") {
            const std::size_t x = v.find('x');
            if (x == std::string::npos)
                throw std::runtime_error("mpi_grid must be auto or RxC (e.g. 2x2): " + v);
            p.grid_rows_cfg = parse_int(k, v.substr(0, x));
            p.grid_cols_cfg = parse_int(k, v.substr(x + 1));
            if (p.grid_rows_cfg < 1 || p.grid_cols_cfg < 1)
                throw std::runtime_error("mpi_grid sizes must be positive: " + v);
        } else if (k == "precision")
            p.precision = parse_choice(k, v, {{"fp64", SGPU_PREC_FP64}, {"mixed", SGPU_PREC_MIXED}});
        else if (k == "mg_mode")
            p.mg_mode = parse_choice(k, v, {{"fixed", SGPU_MG_FIXED}, {"tolerance", SGPU_MG_TOLERANCE}});
        else if (k == "warm_start")
            p.warm_start = parse_choice(k, v, {{"zero", 0}, {"cnn", 1}});
        else if (k == "cnn_weights") copy_str(p.cnn_weights, sizeof p.cnn_weights, v);
        else if (k == "restart_from") copy_str(p.restart_from, sizeof p.restart_from, v);
        else if (k == "graph_batch") p.graph_batch = parse_int(k, v);
    }
    params_finalize(p);
}

} // namespace sgpu

extern "C" {

int sgpu_params_default(sgpu_params_t* out) {
    if (!out) return sgpu::fail(SGPU_E_INVALID, "sgpu_params_default: null output");
    try {
        sgpu::params_defaults(*out);
        sgpu::params_finalize(*out);
        return SGPU_OK;
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}

int sgpu_params_finalize(sgpu_params_t* p) {
    if (!p) return sgpu::fail(SGPU_E_INVALID, "sgpu_params_finalize: null params");
    try {
        sgpu::params_finalize(*p);
        return SGPU_OK;
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}

int sgpu_params_from_config(const char* text, sgpu_params_t* out) {
    if (!text || !out) return sgpu::fail(SGPU_E_INVALID, "sgpu_params_from_config: null argument");
    try {
        sgpu::params_from_config(text, *out);
        return SGPU_OK;
    } catch (const std::exception& e) {
        return sgpu::fail(SGPU_E_INVALID, e.what());
    }
}

} // extern "C"
