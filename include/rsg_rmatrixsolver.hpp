/*
 * rsg_rmatrixsolver.hpp -- header-only C++ drop-in for the reference's
 * RMatrixSolver (include/rmatrixsolver.h:9-52) on top of the C ABI in rsg.h.
 *
 * The reference's solver takes range-model-lib / range-base-lib types
 * (RSparseMatrix, RRVector, RMatrixSolverConf), which are not part of the
 * reference repository.  This header provides minimal stand-ins with the
 * members the solve path uses, in namespace rsg::dropin; an application that
 * has the real types adapts them in RMatrixSolver::solve (row vectors of
 * (index, value) -> CSR), which is the only place they are read.
 *
 * Behaviour kept from the reference:
 *  - solve(A, b, x, preconditioner = NONE, blockSize = 1); x is resized to the
 *    number of rows and its incoming values are the initial guess
 *    (src/rmatrixsolver.cpp:158-201);
 *  - a process-wide CSR cache keyed by the address of A: a later solve with the
 *    same pattern only refreshes the values (src/rmatrixsolver.cpp:56-109);
 *  - unknown solver / preconditioner types throw RError
 *    (src/rmatrixsolver.cpp:195, src/rmatrixpreconditioner.cpp:32);
 *  - non-convergence is silent, as in RIterationInfo::hasConverged
 *    (src/riterationinfo.cpp:90-109); lastStats() exposes what happened.
 * Link with -lrsg (librsg.so).  The GPU is device 0 unless RSG_DEVICE is set.
 */
#ifndef RSG_RMATRIXSOLVER_HPP
#define RSG_RMATRIXSOLVER_HPP

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "rsg.h"

namespace rsg {
namespace dropin {

class RError : public std::runtime_error {
public:
    explicit RError(const std::string &m) : std::runtime_error(m) {}
};

/* RRVector stand-in (range-base-lib): a vector of doubles. */
class RRVector : public std::vector<double> {
public:
    RRVector() = default;
    explicit RRVector(unsigned n, double v = 0.0) : std::vector<double>(n, v) {}
    unsigned getNRows() const { return unsigned(size()); }
    void fill(double v) { std::fill(begin(), end(), v); }
    static double euclideanNorm(const RRVector &v)
    {
        double s = 0.0;
        for (double a : v) s += a * a;
        return std::sqrt(s);
    }
};

/* RSparseMatrix stand-in (range-model-lib): rows of (column, value) pairs kept sorted. */
class RSparseMatrix {
public:
    using Row = std::vector<std::pair<unsigned, double>>;
    void setNRows(unsigned n) { rows_.resize(n); }
    unsigned getNRows() const { return unsigned(rows_.size()); }
    void clear() { rows_.clear(); }
    const Row &getVector(unsigned r) const { return rows_[r]; }
    /* addValue accumulates into (row, col), inserting the entry if it is new. */
    void addValue(unsigned r, unsigned c, double v)
    {
        if (r >= rows_.size()) rows_.resize(r + 1);
        Row &row = rows_[r];
        auto it = std::lower_bound(row.begin(), row.end(), c,
                                   [](const std::pair<unsigned, double> &e, unsigned k) { return e.first < k; });
        if (it != row.end() && it->first == c) it->second += v;
        else row.insert(it, {c, v});
    }
    bool findColumnPosition(unsigned r, unsigned c, unsigned &pos) const
    {
        const Row &row = rows_[r];
        for (unsigned k = 0; k < row.size(); k++)
            if (row[k].first == c) {
                pos = k;
                return true;
            }
        return false;
    }

private:
    std::vector<Row> rows_;
};

/* RMatrixSolverConf stand-in: the fields src/rmatrixsolver.cpp reads (:125-128, :186). */
class RMatrixSolverConf {
public:
    enum Type { CG = 0, GMRES = 1 };
    explicit RMatrixSolverConf(Type t = CG) : type_(t) {}
    Type getType() const { return type_; }
    void setType(Type t) { type_ = t; }
    unsigned getNOuterIterations() const { return nOuter_; }
    void setNOuterIterations(unsigned n) { nOuter_ = n; }
    unsigned getNInnerIterations() const { return nInner_; }
    void setNInnerIterations(unsigned n) { nInner_ = n; }
    double getSolverCvgValue() const { return cvg_; }
    void setSolverCvgValue(double v) { cvg_ = v; }
    unsigned getOutputFrequency() const { return freq_; }
    void setOutputFrequency(unsigned f) { freq_ = f; }
    const std::string &getOutputFileName() const { return file_; }
    void setOutputFileName(const std::string &f) { file_ = f; }

private:
    Type type_;
    unsigned nOuter_ = 1000, nInner_ = 30, freq_ = 1;
    double cvg_ = 1.0e-13;
    std::string file_;
};

/* RMatrixPreconditionerType (include/rmatrixpreconditioner.h:7-16). */
typedef enum _RMatrixPreconditionerType {
    R_MATRIX_PRECONDITIONER_NONE = 0,
    R_MATRIX_PRECONDITIONER_JACOBI,
    R_MATRIX_PRECONDITIONER_BLOCK_JACOBI,
    R_MATRIX_PRECONDITIONER_N_TYPES
} RMatrixPreconditionerType;

namespace detail {

inline void check(rsg_context *ctx, rsg_status s, const char *what)
{
    if (s < 0) throw RError(std::string(what) + ": " + rsg_status_string(s) + ": " + rsg_last_error(ctx));
}

struct Device {
    rsg_context *ctx = nullptr;
    std::mutex mu;
    Device()
    {
        const char *d = std::getenv("RSG_DEVICE");
        rsg_status s = rsg_context_create(d ? std::atoi(d) : 0, &ctx);
        if (s != RSG_OK) throw RError(std::string("rsg_context_create: ") + rsg_status_string(s));
    }
    ~Device()
    {
        for (auto &kv : cache) rsg_csr_destroy(ctx, kv.second.A);
        rsg_context_destroy(ctx);
    }
    struct Entry {
        rsg_csr *A = nullptr;
        std::vector<uint32_t> rp, ci;
    };
    std::unordered_map<const RSparseMatrix *, Entry> cache;
    static Device &get()
    {
        static Device dev;
        return dev;
    }
};

}  // namespace detail

class RMatrixSolver {
public:
    explicit RMatrixSolver(const RMatrixSolverConf &conf) : conf_(conf) {}
    RMatrixSolver(const RMatrixSolver &o) = default;
    RMatrixSolver &operator=(const RMatrixSolver &o) = default;
    ~RMatrixSolver() = default;

    void solve(const RSparseMatrix &A, const RRVector &b, RRVector &x,
               RMatrixPreconditionerType precType = R_MATRIX_PRECONDITIONER_NONE, unsigned blockSize = 1)
    {
        if (conf_.getType() != RMatrixSolverConf::CG && conf_.getType() != RMatrixSolverConf::GMRES)
            throw RError("Unknown matrix solver type '" + std::to_string(int(conf_.getType())) + "'");
        if (precType < R_MATRIX_PRECONDITIONER_NONE || precType >= R_MATRIX_PRECONDITIONER_N_TYPES)
            throw RError("Invalid matrix preconditioner type '" + std::to_string(int(precType)) + "'");
        detail::Device &dev = detail::Device::get();
        std::lock_guard<std::mutex> lock(dev.mu);
        const unsigned n = A.getNRows();
        std::vector<uint32_t> rp(n + 1, 0), ci;
        std::vector<double> val;
        for (unsigned i = 0; i < n; i++) rp[i + 1] = rp[i] + uint32_t(A.getVector(i).size());
        ci.reserve(rp[n]);
        val.reserve(rp[n]);
        for (unsigned i = 0; i < n; i++)
            for (const auto &e : A.getVector(i)) {
                ci.push_back(e.first);
                val.push_back(e.second);
            }
        auto &entry = dev.cache[&A];
        if (entry.A && entry.rp == rp && entry.ci == ci) {
            detail::check(dev.ctx, rsg_csr_update_values(dev.ctx, entry.A, val.data(), RSG_MEM_HOST),
                          "rsg_csr_update_values");
        } else {
            if (entry.A) rsg_csr_destroy(dev.ctx, entry.A);
            entry.A = nullptr;
            detail::check(dev.ctx, rsg_csr_create(dev.ctx, n, rp.data(), ci.data(), val.data(), RSG_MEM_HOST, &entry.A),
                          "rsg_csr_create");
            entry.rp.swap(rp);
            entry.ci.swap(ci);
        }
        x.resize(b.size(), 0.0);
        rsg_solver_conf c;
        rsg_conf_default(&c);
        c.solver_type = conf_.getType() == RMatrixSolverConf::CG ? RSG_SOLVER_CG : RSG_SOLVER_GMRES;
        c.n_outer = conf_.getNOuterIterations();
        c.n_inner = conf_.getNInnerIterations();
        c.cvg = conf_.getSolverCvgValue();
        c.output_frequency = conf_.getOutputFrequency();
        c.output_file = logFile_ && !conf_.getOutputFileName().empty() ? conf_.getOutputFileName().c_str() : nullptr;
        rsg_status s = rsg_solve(dev.ctx, entry.A, &c, int32_t(precType), blockSize, b.data(), x.data(), RSG_MEM_HOST,
                                 &stats_);
        detail::check(dev.ctx, s, "rsg_solve");
    }

    void disableConvergenceLogFile() { logFile_ = false; }
    const rsg_stats &lastStats() const { return stats_; }

private:
    RMatrixSolverConf conf_;
    bool logFile_ = true;
    rsg_stats stats_ = {};
};

}  // namespace dropin
}  // namespace rsg

#endif
