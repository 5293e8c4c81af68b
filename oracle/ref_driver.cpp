// C driver around the reference's own solver sources (TEST INFRASTRUCTURE ONLY).
//
// oracle/Makefile's `ref` target compiles the reference project's src/rmatrixsolver.cpp,
// src/rmatrixpreconditioner.cpp, src/riterationinfo.cpp, src/riterationinfovalue.cpp and
// src/reigenvaluesolver.cpp unchanged, from where they lie, against the stand-in headers in oracle/ref_shim/ (range-base-lib,
// range-model-lib and the few Qt classes they name are not part of the reference), together with
// this file, into oracle/_ref/libref_solver.so.  Tests use it to check the oracle's restatement and
// the CUDA library against the reference's own RMatrixSolver::solve; bench.py's reference arm
// times it.  Nothing in the product loads it.
//
// The iteration count and the last error come from RIterationInfo::printIteration, which reports
// every iteration through RLogger::info when the output frequency is 1: the logger stand-in below
// picks the values out of that one format's arguments.
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>

#include <omp.h>

#include "reigenvaluesolver.h"
#include "rmatrixsolver.h"

namespace {

const char *const kIterationFormat = "> %6u of %-6u |% 12e |% 12e |\n";

struct LogState {
    std::mutex mu;
    unsigned last_iteration = 0;  // the "iteration + 1" of the last printed line
    double error = 0.0, trend = 0.0;
    unsigned lines = 0;
    bool echo = std::getenv("REF_SHIM_ECHO") != nullptr;
} g_log;

void log_message(const char *format, va_list ap)
{
    std::lock_guard<std::mutex> lock(g_log.mu);
    if (std::strcmp(format, kIterationFormat) == 0) {
        va_list aq;
        va_copy(aq, ap);
        g_log.last_iteration = va_arg(aq, unsigned);
        (void)va_arg(aq, unsigned);
        g_log.error = va_arg(aq, double);
        g_log.trend = va_arg(aq, double);
        va_end(aq);
        g_log.lines++;
    }
    if (g_log.echo) std::vfprintf(stderr, format, ap);
}

}  // namespace

void RLogger::info(const char *format, ...)
{
    va_list ap;
    va_start(ap, format);
    log_message(format, ap);
    va_end(ap);
}

void RLogger::warning(const char *format, ...)
{
    va_list ap;
    va_start(ap, format);
    log_message(format, ap);
    va_end(ap);
}

void RLogger::error(const char *format, ...)
{
    va_list ap;
    va_start(ap, format);
    log_message(format, ap);
    va_end(ap);
}

extern "C" {

typedef struct {
    uint32_t iterations;  // CG: iterations run; GMRES: restart cycles that checked convergence
    uint32_t lines;       // iteration reports seen
    double error;         // last reference-style error ||r|| / (||A|| ||x|| + ||b||) (scaled system)
    double trend;
    double seconds;       // wall time of RMatrixSolver::solve
    char message[256];    // RError text when the call failed
} ref_result;

void *ref_matrix_create(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val)
{
    try {
        auto *A = new RSparseMatrix(n);
        for (uint32_t i = 0; i < n; i++) A->getVector(i).assign(ci + rp[i], val + rp[i], rp[i + 1] - rp[i]);
        return A;
    } catch (...) {
        return nullptr;
    }
}

// Same pattern, new values (a caller re-assembling into the same RSparseMatrix).
void ref_matrix_update(void *handle, const uint32_t *rp, const double *val)
{
    auto *A = static_cast<RSparseMatrix *>(handle);
    for (uint32_t i = 0; i < A->getNRows(); i++) {
        RSparseVector<double> &row = A->getVector(i);
        for (uint32_t j = 0; j < row.size(); j++) row.setValue(j, val[rp[i] + j]);
    }
}

void ref_matrix_destroy(void *handle) { delete static_cast<RSparseMatrix *>(handle); }

// RMatrixSolver::solve(A, b, x, prec, block) with a configuration of the given type (0 CG, 1 GMRES).
// x holds the initial guess on entry and the solution on return.  threads > 0 sets the OpenMP team
// size for this call (the reference's parallel regions take the default team size).
// Returns 0, or -1 with the RError text in out->message.
int ref_solve(void *handle, const double *b, double *x, int solver_type, int prec, unsigned block,
              unsigned n_outer, unsigned n_inner, double cvg, const char *log_file, int threads, ref_result *out)
{
    std::memset(out, 0, sizeof(*out));
    struct TeamSize {  // a requested team size holds for this call only
        int prev = omp_get_max_threads();
        ~TeamSize() { omp_set_num_threads(prev); }
    } team;
    if (threads > 0) omp_set_num_threads(threads);
    const RSparseMatrix &A = *static_cast<RSparseMatrix *>(handle);
    const uint n = A.getNRows();
    try {
        RMatrixSolverConf conf(solver_type == 1 ? RMatrixSolverConf::GMRES : RMatrixSolverConf::CG);
        conf.setNOuterIterations(n_outer);
        conf.setNInnerIterations(n_inner);
        conf.setSolverCvgValue(cvg);
        conf.setOutputFrequency(1);
        conf.setOutputFileName(QString(log_file ? log_file : ""));
        RMatrixSolver solver(conf);
        RRVector bv(n), xv(n);
        std::memcpy(bv.data(), b, sizeof(double) * n);
        std::memcpy(xv.data(), x, sizeof(double) * n);
        {
            std::lock_guard<std::mutex> lock(g_log.mu);
            g_log.last_iteration = 0;
            g_log.lines = 0;
            g_log.error = g_log.trend = 0.0;
        }
        const auto t0 = std::chrono::steady_clock::now();
        solver.solve(A, bv, xv, RMatrixPreconditionerType(prec), block);
        const auto t1 = std::chrono::steady_clock::now();
        std::memcpy(x, xv.data(), sizeof(double) * n);
        out->seconds = std::chrono::duration<double>(t1 - t0).count();
        out->iterations = g_log.last_iteration;
        out->lines = g_log.lines;
        out->error = g_log.error;
        out->trend = g_log.trend;
        return 0;
    } catch (const std::exception &e) {
        std::snprintf(out->message, sizeof(out->message), "%s", e.what());
        return -1;
    }
}

// The start values REigenValueSolver draws (src/reigenvaluesolver.cpp:125-128, 222-225, 306-311)
// after srand(seed): n values rand()/RAND_MAX, then (Rayleigh) the shift 1e9 rand()/RAND_MAX.
void ref_rand_start(unsigned seed, uint32_t n, double *start, double *mu)
{
    std::srand(seed);
    for (uint32_t i = 0; i < n; i++) start[i] = double(std::rand()) / double(RAND_MAX);
    *mu = 1.0e9 * double(std::rand()) / double(RAND_MAX);
}

// REigenValueSolver::solve(M, K, d, ev) after srand(seed), its matrix solves configured as ref_solve
// configures CG.  values: up to n_values doubles; vectors (may be NULL): rows of n doubles.
// Returns the number of values, or -1 with the RError text in out->message.
int ref_eigen(void *m_handle, void *k_handle, int method, unsigned n_eigen, unsigned n_iterations, double cvg,
              unsigned seed, unsigned n_outer, double solver_cvg, int threads, uint32_t n_values, double *values,
              double *vectors, ref_result *out)
{
    std::memset(out, 0, sizeof(*out));
    struct TeamSize {
        int prev = omp_get_max_threads();
        ~TeamSize() { omp_set_num_threads(prev); }
    } team;
    if (threads > 0) omp_set_num_threads(threads);
    const RSparseMatrix &M = *static_cast<RSparseMatrix *>(m_handle);
    const RSparseMatrix &K = *static_cast<RSparseMatrix *>(k_handle);
    try {
        REigenValueSolverConf ec;
        ec.method = REigenValueSolverConf::Method(method);
        ec.setNEigenValues(n_eigen);
        ec.setNIterations(n_iterations);
        ec.setSolverCvgValue(cvg);
        RMatrixSolverConf conf(RMatrixSolverConf::CG);
        conf.setNOuterIterations(n_outer);
        conf.setSolverCvgValue(solver_cvg);
        conf.setOutputFrequency(1);
        REigenValueSolver solver(ec, conf);
        RRVector d;
        RRMatrix ev;
        std::srand(seed);
        const auto t0 = std::chrono::steady_clock::now();
        solver.solve(M, K, d, ev);
        out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const uint32_t nd = std::min<uint32_t>(n_values, d.getNRows());
        for (uint32_t i = 0; i < nd; i++) values[i] = d[i];
        if (vectors)
            for (uint32_t r = 0; r < std::min<uint32_t>(nd, ev.getNRows()); r++)
                for (uint32_t c = 0; c < ev.getNColumns(); c++) vectors[size_t(r) * ev.getNColumns() + c] = ev[r][c];
        return int(d.getNRows());
    } catch (const std::exception &e) {
        std::snprintf(out->message, sizeof(out->message), "%s", e.what());
        return -1;
    }
}

}  // extern "C"
