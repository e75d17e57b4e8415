// The reference's output files, written from a solver handle byte for byte as the reference writes
// them: residuals.dat (include/solver/ResidualsFile.hpp:18-48, rows from EulerSolver::PrintInfo,
// src/solver/EulerSolver.cpp:253-259), cp_part_N.dat (EulerSolver::PrintCp, :283-303), summary.txt
// (EulerSolver::WriteSummary, :169-198) and <partition>.sol (WriteSolution::writeSolutionFile,
// src/solver/WriteSolution.cpp:30-55).  Host code only.
//
// The reference formats with iostreams: `std::setw(w) << x` with std::scientific and precision p
// prints what printf's "%w.pe" prints, an int under setw(w) what "%wd" prints, a string what "%ws"
// prints; std::endl is "\n".
#include <cuda_runtime.h>

#include <cinttypes>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "solver.hpp"

namespace e3d {
namespace {

struct OutFile {
    FILE *f = nullptr;
    explicit OutFile(const char *path) {
        if (!path) throw Error(E3D_ERR_INVALID_ARG, "NULL path");
        f = std::fopen(path, "w");
        if (!f) throw Error(E3D_ERR_INVALID_ARG, std::string("cannot open ") + path + " for writing");
    }
    ~OutFile() {
        if (f) std::fclose(f);
    }
    void put(const char *fmt, ...) {
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(f, fmt, ap);
        va_end(ap);
    }
    void close() {
        if (std::fclose(f) != 0) {
            f = nullptr;
            throw Error(E3D_ERR_INVALID_ARG, "writing the output file failed");
        }
        f = nullptr;
    }
};

// A double as toml++ 2.3.1 prints it when built with GCC (extern/toml++/toml_print_to_stream.h:198-250
// with TOML_FLOAT_CHARCONV 0): an ostringstream at 16 significant digits (%.16g), ".0" appended when
// that has no decimal point or exponent; inf, -inf and nan by name.
std::string toml_float(double v) {
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.16g", v);
    std::string s(buf);
    if (s.find_first_of(".eE") == std::string::npos) s += ".0";
    return s;
}

// The width toml++ 2.3.1 estimates for a double (extern/toml++/toml_default_formatter.hpp:129-143):
// 3 for zero, else 2 + [v < 0] + size_t(log10|v|) + 1, in size_t arithmetic.  For |v| < 1 the
// logarithm is negative and its conversion to size_t wraps the way x86-64 code converts it (the
// truncated value taken as a signed 64-bit integer), so small magnitudes give "negative" widths.
// NaN converts to 2^63 and +inf to 0 there.
uint64_t toml_float_columns(double v) {
    if (v == 0.0) return 3;
    uint64_t w = 2;
    if (v < 0.0) {
        w += 1;
        v = -v;
    }
    const double l = std::log10(v);
    uint64_t c;
    if (std::isnan(l)) c = uint64_t(1) << 63;
    else if (std::isinf(l)) c = l > 0 ? 0 : uint64_t(1) << 63;
    else c = (uint64_t)(int64_t)l;
    return w + c + 1;
}

// A 3-vector as toml++ prints an array (toml_default_formatter.h:116-173): inline "[ a, b, c ]"
// unless the estimated inline width reaches the 120-column wrap (toml_default_formatter.hpp:93-106,
// 158-161; the running sum stops at the first partial sum that reaches 120 as an unsigned number,
// and the arrays here sit one indent level below the root, so the column bias is 0).  Multi-line
// arrays put each element on its own line, indented four spaces, and "]" on a line of its own.
std::string toml_vec(const double v[3]) {
    uint64_t width = 3;
    for (int k = 0; k < 3; k++) {
        width += toml_float_columns(v[k]) + 2;
        if (width >= 120) break;
    }
    if (width < 120) return "[ " + toml_float(v[0]) + ", " + toml_float(v[1]) + ", " + toml_float(v[2]) + " ]";
    std::string s = "[";
    for (int k = 0; k < 3; k++) s += std::string(k ? "," : "") + "\n    " + toml_float(v[k]);
    return s + "\n]";
}

// The last run's coefficient samples: 7 doubles each (iteration, force, moment).
std::vector<double> samples_of(Solver *S) {
    const int n = S->records_valid ? std::min(S->ctl_host->n_samples, S->sample_cap) : 0;
    std::vector<double> v(7 * (size_t)std::max(n, 0));
    if (n > 0) E3D_CUDA(cudaMemcpy(v.data(), S->samples.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost));
    return v;
}

std::vector<double> history_of(Solver *S) {
    const int n = S->records_valid ? std::min(S->ctl_host->n_rms, S->hist_cap) : 0;
    std::vector<double> v(std::max(n, 0));
    if (n > 0) E3D_CUDA(cudaMemcpy(v.data(), S->hist.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    return v;
}

Solver *writable(e3d_solver *solver) {
    if (!solver) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
    Solver *S = as_solver(solver);
    if (S->batch) throw Error(E3D_ERR_INVALID_ARG, "solver is a member of a batch (retire or remove it first)");
    E3D_CUDA(cudaSetDevice(S->device));
    E3D_CUDA(cudaStreamSynchronize(S->stream));
    return S;
}

}  // namespace
}  // namespace e3d

using namespace e3d;

extern "C" {

e3d_status e3d_solver_coefficient_history(e3d_solver *solver, double *samples, int32_t capacity, int32_t *count) {
    return guarded([&] {
        if (!count) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = writable(solver);
        std::vector<double> v = samples_of(S);
        *count = (int32_t)(v.size() / 7);
        if (samples && capacity > 0) std::copy(v.begin(), v.begin() + 7 * std::min<size_t>(capacity, v.size() / 7), samples);
    });
}

e3d_status e3d_solver_wall_cp(e3d_solver *solver, double *cp, int32_t capacity, int32_t *count) {
    return guarded([&] {
        if (!count) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        Solver *S = writable(solver);
        *count = S->n_wall;
        if (cp && capacity > 0 && S->n_wall > 0)
            E3D_CUDA(cudaMemcpy(cp, S->wall_cp.p, std::min(capacity, S->n_wall) * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

e3d_status e3d_solver_write_residuals(e3d_solver *solver, const char *path) {
    return guarded([&] {
        Solver *S = writable(solver);
        if (!S->records_valid)
            throw Error(E3D_ERR_INVALID_ARG, "the last run was e3d_solver_run_noalloc, which keeps no RMS history or "
                                             "coefficient samples in the handle");
        const Control c = *S->ctl_host;
        const std::vector<double> smp = samples_of(S), hist = history_of(S);
        OutFile o(path);
        const char *head[8] = {"iter", "Max residual", "Cx", "Cy", "Cz", "CMx", "CMy", "CMz"};
        for (const char *h : head) o.put("%30s", h);
        o.put("\n");
        auto row = [&](int it, double rms, const double *F, const double *M) {
            o.put("%30d", it);
            o.put("%30.10e", rms);
            for (int k = 0; k < 3; k++) o.put("%30.10e", F[k]);
            for (int k = 0; k < 3; k++) o.put("%30.10e", M[k]);
            o.put("\n");
        };
        // one row per sample, with the RMS of the iteration that was sampled
        for (size_t k = 0; 7 * k < smp.size(); k++) {
            const double *s = smp.data() + 7 * k;
            const int it = (int)s[0];
            const double rms = it >= 1 && (size_t)it <= hist.size() ? hist[it - 1] : c.last_rms;
            row(it, rms, s + 1, s + 4);
        }
        // the residual exit prints one more row with the last sampled coefficients (:100-108)
        if (c.stop_reason == E3D_STOP_RESIDUAL && !c.nonfinite) row(c.it, c.last_rms, c.force, c.moment);
        o.close();
    });
}

e3d_status e3d_solver_write_cp(e3d_solver *solver, const char *path) {
    return guarded([&] {
        Solver *S = writable(solver);
        std::vector<double> cp(std::max(S->n_wall, 0));
        if (S->n_wall > 0)
            E3D_CUDA(cudaMemcpy(cp.data(), S->wall_cp.p, S->n_wall * sizeof(double), cudaMemcpyDeviceToHost));
        OutFile o(path);
        o.put("%20s%20s%20s%20s\n", "Cp", "x", "y", "z");
        for (int i = 0; i < S->n_wall; i++)
            o.put("%20.10e%20.10e%20.10e%20.10e\n", cp[i], S->wall_center_host[3 * (size_t)i],
                  S->wall_center_host[3 * (size_t)i + 1], S->wall_center_host[3 * (size_t)i + 2]);
        o.close();
    });
}

e3d_status e3d_solver_write_solution(e3d_solver *solver, const char *path) {
    return guarded([&] {
        Solver *S = writable(solver);
        const int64_t T = S->state_size();
        std::vector<double> st(8 * (size_t)T);
        double *ptr[8];
        for (int k = 0; k < 8; k++) ptr[k] = st.data() + k * T;
        const e3d_status rc = e3d_solver_get_state(solver, ptr);
        if (rc != E3D_OK) throw Error(rc, e3d_last_error());
        OutFile o(path);
        const char *head[6] = {"density", "velocity_x", "velocity_y", "velocity_z", "pressure", "energy"};
        for (const char *h : head) o.put("%20s", h);
        o.put("\n");
        const int cols[6] = {0, 1, 2, 3, 4, 5};  // rho u v w p E
        for (int i = 0; i < S->N; i++) {
            for (int k : cols) o.put("%20.6e", ptr[k][i]);
            o.put("\n");
        }
        o.close();
    });
}

e3d_status e3d_solver_write_summary(e3d_solver *solver, const char *path, int64_t solver_ms, int64_t total_ms,
                                    int32_t n_cores) {
    return guarded([&] {
        Solver *S = writable(solver);
        if (n_cores < 1) throw Error(E3D_ERR_INVALID_ARG, "n_cores must be positive");
        const Control c = *S->ctl_host;
        // TimeCore_p_IterNElem_ms: double(solverTimer * nCores) / double(iterations * NElem), the
        // second product in 32-bit int arithmetic as the reference computes it (it wraps)
        const int32_t it_elem = (int32_t)((uint32_t)c.it * (uint32_t)S->N);
        const double per = (double)(solver_ms * n_cores) / (double)it_elem;
        OutFile o(path);
        o.put("Iterations = %d\n", c.it);
        o.put("Ncores = %d\n", n_cores);
        o.put("SolverLoopTime_ms = %" PRId64 "\n", solver_ms);
        o.put("TimeCore_p_IterNElem_ms = %s\n", toml_float(per).c_str());
        o.put("TotalSolverTime_ms = %" PRId64 "\n", total_ms);
        o.put("\n[Coefficients]\n");
        o.put("CD = %s\n", toml_float(c.cd).c_str());
        o.put("CL = %s\n", toml_float(c.cl).c_str());
        o.put("CM = %s\n", toml_float(c.cm).c_str());
        o.put("Force_Coeff = %s\n", toml_vec(c.force).c_str());
        o.put("Moment_Coeff = %s\n", toml_vec(c.moment).c_str());
        o.put("\n[Mesh]\n");
        o.put("NElem = %d\n", S->N);
        o.put("Wall_Face_Vector_Sum = %s\n", toml_vec(S->wall_sum).c_str());
        o.close();
    });
}

}  // extern "C"
