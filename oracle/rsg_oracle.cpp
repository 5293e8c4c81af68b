/*
 * CPU oracle for the sparse linear-solve path (TEST INFRASTRUCTURE ONLY).
 * See rsg_oracle.h for scope.  Each function names the reference lines it
 * restates.  Loop and reduction structure of the solvers follow the
 * reference's OpenMP code so that the oracle also serves as the timed CPU
 * baseline ("port" kind) for bench.py.
 */
#include "rsg_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

namespace {

const uint32_t kEod = 0xffffffffu;

inline double row_product(const uint32_t *rp, const uint32_t *ci, const double *val, uint32_t row,
                          const double *x)
{
    /* src/rmatrixsolver.cpp:111-119 (multiplyRow) */
    double value = 0.0;
    for (uint32_t j = rp[row]; j < rp[row + 1]; j++) value += val[j] * x[ci[j]];
    return value;
}

/* src/riterationinfo.cpp:74-109 (setError / hasConverged) */
struct IterationInfo {
    double error = 0.0, trend = 0.0, cvg = 0.0, eps = 0.0;
    void set_error(double e)
    {
        trend = e - error;
        error = e;
    }
    bool has_converged() const
    {
        if (!std::isnormal(error)) return true;
        if (!std::isnormal(trend)) return true;
        if (error < cvg) return true;
        if (std::abs(trend) < eps * eps) return true;
        return false;
    }
};

/* Preconditioner state: src/rmatrixpreconditioner.cpp:16-35 */
struct Precond {
    int type = 0;          /* 0 none, 1 Jacobi, 2 block Jacobi */
    uint32_t width = 1;
    std::vector<double> data;
};

/* Gauss-Jordan inversion with partial pivoting (RRMatrix::invert stand-in). */
bool invert_dense(std::vector<double> &a, uint32_t w)
{
    std::vector<double> inv(size_t(w) * w, 0.0);
    for (uint32_t i = 0; i < w; i++) inv[size_t(i) * w + i] = 1.0;
    for (uint32_t c = 0; c < w; c++) {
        uint32_t piv = c;
        for (uint32_t r = c + 1; r < w; r++)
            if (std::abs(a[size_t(r) * w + c]) > std::abs(a[size_t(piv) * w + c])) piv = r;
        if (a[size_t(piv) * w + c] == 0.0) return false;
        if (piv != c)
            for (uint32_t k = 0; k < w; k++) {
                std::swap(a[size_t(piv) * w + k], a[size_t(c) * w + k]);
                std::swap(inv[size_t(piv) * w + k], inv[size_t(c) * w + k]);
            }
        double p = a[size_t(c) * w + c];
        for (uint32_t k = 0; k < w; k++) {
            a[size_t(c) * w + k] /= p;
            inv[size_t(c) * w + k] /= p;
        }
        for (uint32_t r = 0; r < w; r++) {
            if (r == c) continue;
            double f = a[size_t(r) * w + c];
            if (f == 0.0) continue;
            for (uint32_t k = 0; k < w; k++) {
                a[size_t(r) * w + k] -= f * a[size_t(c) * w + k];
                inv[size_t(r) * w + k] -= f * inv[size_t(c) * w + k];
            }
        }
    }
    a.swap(inv);
    return true;
}

/* src/rmatrixpreconditioner.cpp:51-76,150-190 (compute / computeJacobi / computeBlockJacobi).
 * Orphaned worksharing: must be called inside the solver's parallel region. */
void precond_apply(const Precond &P, uint32_t n, const double *x, double *y)
{
    if (P.type == 1) {
#pragma omp for
        for (int64_t i = 0; i < int64_t(n); i++) y[i] = P.data[size_t(i)] * x[i];
    } else if (P.type == 2) {
        const uint32_t w = P.width;
        const int64_t nb = n / w;
#pragma omp for
        for (int64_t blk = 0; blk < nb; blk++)
            for (uint32_t k = 0; k < w; k++) {
                size_t m = size_t(blk) * w + k;
                double value = 0.0;
                for (uint32_t l = 0; l < w; l++) value += P.data[m * w + l] * x[size_t(blk) * w + l];
                y[m] = value;
            }
    } else {
#pragma omp for
        for (int64_t i = 0; i < int64_t(n); i++) y[i] = x[i];
    }
}

bool find_diag(const uint32_t *rp, const uint32_t *ci, uint32_t row, uint32_t col, uint32_t &pos)
{
    for (uint32_t j = rp[row]; j < rp[row + 1]; j++)
        if (ci[j] == col) {
            pos = j;
            return true;
        }
    return false;
}

double true_relres_ld(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                      const double *b, const double *x)
{
    long double rr = 0.0L, bb = 0.0L;
#pragma omp parallel for reduction(+ : rr, bb)
    for (int64_t i = 0; i < int64_t(n); i++) {
        long double s = 0.0L;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) s += (long double)val[j] * (long double)x[ci[j]];
        long double r = (long double)b[i] - s;
        rr += r * r;
        bb += (long double)b[i] * (long double)b[i];
    }
    if (bb == 0.0L) return double(std::sqrt(rr));
    return double(std::sqrt(rr / bb));
}

/* src/rmatrixsolver.cpp:208-355 (solveCG).  stop_rule 1 adds the benchmark's
 * rule: when the recurrence residual reaches rtol, the true residual b - A x is
 * recomputed; the solve stops once that meets rtol, otherwise CG restarts from
 * the true residual (p = z), which cannot diverge when rtol is below the
 * attainable accuracy. */
void solve_cg(const orc_conf &conf, uint32_t m, const uint32_t *rp, const uint32_t *ci, const double *val,
              double An, const Precond &P, const double *b, double *x, orc_stats &st)
{
    std::vector<double> r(m, 0.0), z(m, 0.0), p(m, 0.0), q(m, 0.0);
    double ro0 = 0.0, ro1 = 0.0, beta = 0.0, dot = 0.0, alpha = 0.0, xn = 0.0, rn = 0.0, bn = 0.0;
    IterationInfo info;
    info.cvg = conf.cvg;
    info.eps = conf.eps;
    const double eps = conf.eps;
    bool stop = false;
    uint32_t iterations = 0;
    int converged = 0;
    double tn = 0.0;
    bool restart_dir = false;

#pragma omp parallel default(shared)
    {
#pragma omp for reduction(+ : bn)
        for (int64_t i = 0; i < int64_t(m); i++) {
            r[i] = b[i] - row_product(rp, ci, val, uint32_t(i), x);
            bn += b[i] * b[i];
        }
#pragma omp barrier
#pragma omp master
        bn = std::sqrt(bn);

        for (uint32_t it = 0; it < conf.n_outer; it++) {
#pragma omp barrier
            precond_apply(P, m, r.data(), z.data());
#pragma omp master
            ro0 = 0.0;
#pragma omp barrier
#pragma omp for reduction(+ : ro0)
            for (int64_t i = 0; i < int64_t(m); i++) ro0 += r[i] * z[i];
#pragma omp master
            {
                if (it > 0) {
                    beta = ro0 / ro1;
                    ro1 = std::max(ro1, eps);
                }
            }
#pragma omp barrier
#pragma omp for
            for (int64_t i = 0; i < int64_t(m); i++) p[i] = (it == 0 || restart_dir) ? z[i] : p[i] * beta + z[i];
#pragma omp master
            {
                dot = 0.0;
                restart_dir = false;
            }
#pragma omp barrier
#pragma omp for reduction(+ : dot)
            for (int64_t i = 0; i < int64_t(m); i++) {
                q[i] = row_product(rp, ci, val, uint32_t(i), p.data());
                dot += p[i] * q[i];
            }
#pragma omp master
            {
                if (dot > 0.0) dot = std::max(dot, eps);
                else if (dot < 0.0) dot = std::min(dot, -eps);
                else dot = eps;
                alpha = ro0 / dot;
                ro1 = ro0;
                xn = 0.0;
                rn = 0.0;
            }
#pragma omp barrier
#pragma omp for reduction(+ : xn, rn)
            for (int64_t i = 0; i < int64_t(m); i++) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
                xn += x[i] * x[i];
                rn += r[i] * r[i];
            }
#pragma omp master
            {
                xn = std::sqrt(xn);
                rn = std::sqrt(rn);
                double norm = An * xn + bn;
                if (std::abs(norm) < eps) norm = eps;
                info.set_error(rn / norm);
                iterations = it + 1;
                if (conf.stop_rule == 0) {
                    stop = info.has_converged();
                    converged = stop ? 1 : 0;
                } else {
                    stop = false;
                    if (!std::isfinite(rn)) stop = true;
                }
            }
#pragma omp barrier
            if (conf.stop_rule == 1 && !stop && rn <= conf.rtol * bn) {
                /* true residual replacement */
#pragma omp master
                tn = 0.0;
#pragma omp barrier
#pragma omp for reduction(+ : tn)
                for (int64_t i = 0; i < int64_t(m); i++) {
                    r[i] = b[i] - row_product(rp, ci, val, uint32_t(i), x);
                    tn += r[i] * r[i];
                }
#pragma omp master
                {
                    if (std::sqrt(tn) <= conf.rtol * bn) {
                        stop = true;
                        converged = 1;
                    } else {
                        restart_dir = true;  // the recurrence drifted: restart from the true residual
                    }
                }
#pragma omp barrier
            }
            if (stop) break;
        }
    }
    st.iterations = iterations;
    st.error = info.error;
    st.trend = info.trend;
    st.converged = converged;
}

/* src/rmatrixsolver.cpp:357-581 (solveGMRES): restarted GMRES(m), right
 * preconditioning with stored Z, one-pass classical Gram-Schmidt with batched
 * dot products, Givens rotations, inner exit at |g_{i+1}| < 1e-4 beta,
 * back-substitution and x += Z y. */
void solve_gmres(const orc_conf &conf, uint32_t mA, const uint32_t *rp, const uint32_t *ci, const double *val,
                 double An, const Precond &P, const double *b, double *x, orc_stats &st)
{
    const uint32_t nouter = conf.n_outer;
    const uint32_t ninner = std::max<uint32_t>(conf.n_inner, 1);
    std::vector<double> ro(mA, 0.0), w(mA, 0.0), p(ninner + 1, 0.0), y(ninner, 0.0), c(ninner, 0.0),
        s(ninner, 0.0), hValues(ninner + 1, 0.0);
    std::vector<std::vector<double>> v(ninner + 1, std::vector<double>(mA, 0.0));
    std::vector<std::vector<double>> z(ninner + 1, std::vector<double>(mA, 0.0));
    std::vector<double> h(size_t(ninner + 1) * ninner, 0.0);
    auto H = [&](uint32_t i, uint32_t j) -> double & { return h[size_t(i) * ninner + j]; };

    double bn = 0.0;
    for (uint32_t i = 0; i < mA; i++) bn += b[i] * b[i];
    bn = std::sqrt(bn);

    IterationInfo info;
    info.cvg = conf.cvg;
    info.eps = conf.eps;
    const double eps = conf.eps;
    double beta = 0.0, xn = 0.0, wNorm = 0.0;
    bool stop = false;
    int converged = 0;
    uint32_t total_inner = 0, outer_done = 0;

#pragma omp parallel default(shared)
    {
        uint32_t iti = 0;
        for (uint32_t ito = 0; ito < nouter; ito++) {
#pragma omp master
            {
                std::fill(h.begin(), h.end(), 0.0);
                beta = 0.0;
                xn = 0.0;
            }
#pragma omp barrier
#pragma omp for reduction(+ : xn, beta)
            for (int64_t i = 0; i < int64_t(mA); i++) {
                ro[i] = b[i] - row_product(rp, ci, val, uint32_t(i), x);
                xn += x[i] * x[i];
                beta += ro[i] * ro[i];
            }
#pragma omp master
            {
                xn = std::sqrt(xn);
                beta = std::sqrt(beta);
                double norm = An * xn + bn;
                if (std::fabs(norm) < eps) norm = eps;
                info.set_error(beta / norm);
                outer_done = ito;
                if (conf.stop_rule == 0) stop = info.has_converged();
                else stop = (beta <= conf.rtol * bn) || !std::isfinite(beta);
                if (stop && (conf.stop_rule == 0 || beta <= conf.rtol * bn)) converged = 1;
            }
#pragma omp barrier
            if (stop) break;
#pragma omp for
            for (int64_t i = 0; i < int64_t(mA); i++) v[0][i] = (beta == 0.0) ? 0.0 : ro[i] / beta;
#pragma omp master
            {
                std::fill(p.begin(), p.end(), 0.0);
                p[0] = beta;
            }
            for (iti = 0; iti < ninner; iti++) {
#pragma omp barrier
                precond_apply(P, mA, v[iti].data(), z[iti].data());
#pragma omp barrier
#pragma omp for
                for (int64_t i = 0; i < int64_t(mA); i++) w[i] = row_product(rp, ci, val, uint32_t(i), z[iti].data());
#pragma omp single
                std::fill(hValues.begin(), hValues.end(), 0.0);
#pragma omp barrier
                {
                    std::vector<double> hLocal(iti + 1, 0.0);
#pragma omp for nowait
                    for (int64_t j = 0; j < int64_t(mA); j++) {
                        double wj = w[j];
                        for (uint32_t i = 0; i <= iti; i++) hLocal[i] += wj * v[i][j];
                    }
#pragma omp critical
                    for (uint32_t i = 0; i <= iti; i++) hValues[i] += hLocal[i];
                }
#pragma omp barrier
#pragma omp single
                for (uint32_t i = 0; i <= iti; i++) H(i, iti) = hValues[i];
#pragma omp barrier
#pragma omp for
                for (int64_t j = 0; j < int64_t(mA); j++) {
                    double value = w[j];
                    for (uint32_t i = 0; i <= iti; i++) value -= hValues[i] * v[i][j];
                    w[j] = value;
                }
#pragma omp single
                wNorm = 0.0;
#pragma omp barrier
#pragma omp for reduction(+ : wNorm)
                for (int64_t j = 0; j < int64_t(mA); j++) wNorm += w[j] * w[j];
#pragma omp single
                H(iti + 1, iti) = std::sqrt(wNorm);
#pragma omp barrier
#pragma omp for
                for (int64_t i = 0; i < int64_t(mA); i++)
                    v[iti + 1][i] = (H(iti + 1, iti) == 0.0) ? 0.0 : w[i] / H(iti + 1, iti);
#pragma omp barrier
#pragma omp master
                {
                    for (uint32_t i = 1; i <= iti; i++) {
                        double hsave = H(i - 1, iti);
                        H(i - 1, iti) = c[i - 1] * hsave + s[i - 1] * H(i, iti);
                        H(i, iti) = -s[i - 1] * hsave + c[i - 1] * H(i, iti);
                    }
                    double g = std::sqrt(H(iti, iti) * H(iti, iti) + H(iti + 1, iti) * H(iti + 1, iti));
                    if (g == 0.0) {
                        c[iti] = s[iti] = 0.0;
                    } else {
                        c[iti] = H(iti, iti) / g;
                        s[iti] = H(iti + 1, iti) / g;
                    }
                    H(iti, iti) = g;
                    H(iti + 1, iti) = 0.0;
                    p[iti + 1] = -s[iti] * p[iti];
                    p[iti] = c[iti] * p[iti];
                    total_inner++;
                }
#pragma omp barrier
                if (std::fabs(p[iti + 1]) < beta * 1.0e-4) {
                    iti++;
                    break;
                }
            }
#pragma omp barrier
#pragma omp master
            {
                y[iti - 1] = (H(iti - 1, iti - 1) == 0.0) ? 0.0 : p[iti - 1] / H(iti - 1, iti - 1);
                for (int i = int(iti) - 2; i >= 0; i--) {
                    for (int j = int(iti) - 1; j > i; j--) p[i] -= y[j] * H(i, j);
                    y[i] = (H(i, i) == 0.0) ? 0.0 : p[i] / H(i, i);
                }
            }
#pragma omp barrier
#pragma omp for
            for (int64_t i = 0; i < int64_t(mA); i++)
                for (uint32_t j = 0; j <= iti - 1; j++) x[i] += z[j][i] * y[j];
#pragma omp master
            outer_done = ito + 1;
        }
    }
    st.iterations = total_inner;
    st.outer = outer_done;
    st.error = info.error;
    st.trend = info.trend;
    st.converged = converged;
}

/* ---------------- assembly ---------------- */

struct RowMap {
    std::vector<std::vector<std::pair<uint32_t, double>>> rows;
    explicit RowMap(uint32_t n) : rows(n) {}
    /* RSparseMatrix::addValue stand-in: accumulate into (row, col), inserting if new. */
    void add(uint32_t r, uint32_t c, double v)
    {
        auto &row = rows[r];
        for (auto &e : row)
            if (e.first == c) {
                e.second += v;
                return;
            }
        row.emplace_back(c, v);
    }
};

/* P1 tetrahedron: gradients of barycentric shape functions and signed det J. */
double tet_gradients(const double *xyz, const uint32_t *t, double G[4][3])
{
    const double *X0 = xyz + 3 * size_t(t[0]);
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; k++) {
        a[k] = xyz[3 * size_t(t[1]) + k] - X0[k];
        b[k] = xyz[3 * size_t(t[2]) + k] - X0[k];
        c[k] = xyz[3 * size_t(t[3]) + k] - X0[k];
    }
    double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
    for (int k = 0; k < 3; k++) {
        G[1][k] = bc[k] / det;
        G[2][k] = ca[k] / det;
        G[3][k] = ab[k] / det;
        G[0][k] = -(G[1][k] + G[2][k] + G[3][k]);
    }
    return det;
}

orc_system *finish_system(RowMap &rm, std::vector<double> &b);

}  // namespace

struct orc_system {
    uint32_t n = 0;
    std::vector<uint32_t> rp, ci;
    std::vector<double> val, b;
};

namespace {
orc_system *finish_system(RowMap &rm, std::vector<double> &b)
{
    auto *s = new orc_system;
    s->n = uint32_t(rm.rows.size());
    s->rp.assign(size_t(s->n) + 1, 0);
    for (uint32_t i = 0; i < s->n; i++) {
        std::sort(rm.rows[i].begin(), rm.rows[i].end(),
                  [](const std::pair<uint32_t, double> &x, const std::pair<uint32_t, double> &y) {
                      return x.first < y.first;
                  });
        s->rp[i + 1] = s->rp[i] + uint32_t(rm.rows[i].size());
    }
    s->ci.resize(s->rp.back());
    s->val.resize(s->rp.back());
    for (uint32_t i = 0; i < s->n; i++) {
        uint32_t o = s->rp[i];
        for (auto &e : rm.rows[i]) {
            s->ci[o] = e.first;
            s->val[o] = e.second;
            o++;
        }
    }
    s->b.swap(b);
    return s;
}
}  // namespace

extern "C" {

double orc_csr_frobenius(uint32_t n, const uint32_t *rp, const double *val)
{
    /* src/rmatrixsolver.cpp:37-51 */
    double norm2 = 0.0;
#pragma omp parallel for reduction(+ : norm2)
    for (int64_t i = 0; i < int64_t(n); i++)
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) norm2 += val[j] * val[j];
    return std::sqrt(norm2);
}

void orc_spmv(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val, const double *x, double *y)
{
#pragma omp parallel for
    for (int64_t i = 0; i < int64_t(n); i++) y[i] = row_product(rp, ci, val, uint32_t(i), x);
}

void orc_jacobi_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val, double *d)
{
    /* src/rmatrixpreconditioner.cpp:78-94: 1/diag, 0 if the diagonal is zero or absent */
    for (uint32_t i = 0; i < n; i++) {
        d[i] = 0.0;
        uint32_t pos;
        if (find_diag(rp, ci, i, i, pos)) d[i] = (val[pos] == 0.0) ? 0.0 : 1.0 / val[pos];
    }
}

int orc_block_jacobi_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                           uint32_t block_size, double *data, uint32_t *width_out)
{
    /* src/rmatrixpreconditioner.cpp:96-148: width shrinks until it divides n;
     * dense diagonal blocks are inverted once. */
    uint32_t width = std::max<uint32_t>(block_size, 1);
    while (n % width != 0) width--;
    *width_out = width;
    const uint32_t nb = n / width;
    int bad = 0;
#pragma omp parallel for reduction(| : bad)
    for (int64_t blk = 0; blk < int64_t(nb); blk++) {
        std::vector<double> a(size_t(width) * width, 0.0);
        for (uint32_t k = 0; k < width; k++) {
            uint32_t m = uint32_t(blk) * width + k;
            for (uint32_t l = 0; l < width; l++) {
                uint32_t pos;
                if (find_diag(rp, ci, m, uint32_t(blk) * width + l, pos)) a[size_t(k) * width + l] = val[pos];
            }
        }
        if (!invert_dense(a, width)) bad |= 1;
        for (uint32_t k = 0; k < width; k++)
            for (uint32_t l = 0; l < width; l++)
                data[(size_t(blk) * width + k) * width + l] = a[size_t(k) * width + l];
    }
    return bad ? -1 : 0;
}

double orc_true_relres(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val, const double *b,
                       const double *x)
{
    return true_relres_ld(n, rp, ci, val, b, x);
}

int orc_solve(const orc_conf *conf, uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
              int32_t prec_type, uint32_t block_size, const double *b, double *x, orc_stats *stats)
{
    /* src/rmatrixsolver.cpp:158-201 (solve) */
    orc_stats st;
    std::memset(&st, 0, sizeof(st));
    /* a requested team size holds for this call only */
    struct TeamSize {
        int prev = omp_get_max_threads();
        ~TeamSize() { omp_set_num_threads(prev); }
    } team;
    if (conf->n_threads > 0) omp_set_num_threads(conf->n_threads);

    Precond P;
    if (prec_type == 1) {
        P.type = 1;
        P.data.resize(n);
        orc_jacobi_build(n, rp, ci, val, P.data.data());
    } else if (prec_type == 2) {
        P.type = 2;
        P.data.resize(size_t(n) * std::max<uint32_t>(block_size, 1));
        if (orc_block_jacobi_build(n, rp, ci, val, block_size, P.data.data(), &P.width) != 0) {
            st.status = -3;
            *stats = st;
            return -3;
        }
    } else if (prec_type != 0) {
        st.status = -2;
        *stats = st;
        return -2;
    }
    if (conf->solver_type != 0 && conf->solver_type != 1) {
        st.status = -1;
        *stats = st;
        return -1;
    }

    const double An = orc_csr_frobenius(n, rp, val);
    double bn = 0.0;
    for (uint32_t i = 0; i < n; i++) bn += b[i] * b[i];
    bn = std::sqrt(bn);
    double scale = 1.0;
    if (conf->scale_equations && bn != 0.0 && An != 0.0) scale = 1.0e9 / std::abs(bn / An);
    st.norm_a = An;
    st.norm_b = bn;
    st.equation_scale = scale;

    std::vector<double> y(b, b + n);
    for (auto &v : y) v *= scale;
    for (uint32_t i = 0; i < n; i++) x[i] *= scale;

    auto t0 = std::chrono::steady_clock::now();
    if (conf->solver_type == 0) solve_cg(*conf, n, rp, ci, val, An, P, y.data(), x, st);
    else solve_gmres(*conf, n, rp, ci, val, An, P, y.data(), x, st);
    auto t1 = std::chrono::steady_clock::now();
    st.seconds = std::chrono::duration<double>(t1 - t0).count();

    for (uint32_t i = 0; i < n; i++) x[i] *= 1.0 / scale;
    st.true_relres = true_relres_ld(n, rp, ci, val, b, x);
    st.status = 0;
    *stats = st;
    return 0;
}

uint32_t orc_node_book(uint32_t n, const uint8_t *disabled, uint32_t *book)
{
    /* src/rsolvergeneric.cpp:565-582 (rebuildNodeBook) */
    uint32_t next = 0;
    for (uint32_t i = 0; i < n; i++) book[i] = disabled[i] ? kEod : next++;
    return next;
}

/* src/rsolvergeneric.cpp:536-558: nodes of computable elements are computable, the others disabled */
static void orc_disable_not_computable(uint32_t n_nodes, uint32_t n_elements, const uint32_t *elem_begin,
                                       const uint32_t *elem_nodes, const uint8_t *computable, uint32_t dofs,
                                       std::vector<uint8_t> &disabled)
{
    std::vector<uint8_t> computable_nodes(n_nodes, 0);
    for (uint32_t i = 0; i < n_elements; i++)
        if (!computable || computable[i])
            for (uint32_t j = elem_begin[i]; j < elem_begin[i + 1]; j++) computable_nodes[elem_nodes[j]] = 1;
    for (uint32_t i = 0; i < n_nodes; i++)
        if (!computable_nodes[i])
            for (uint32_t c = 0; c < dofs; c++) disabled[size_t(dofs) * i + c] = 1;
}

uint32_t orc_node_book_generic(uint32_t n_nodes, uint32_t n_elements, const uint32_t *elem_begin,
                               const uint32_t *elem_nodes, uint32_t n_groups, const uint32_t *group_begin,
                               const uint32_t *group_elems, const uint8_t *computable, const uint8_t *explicit_bc,
                               uint32_t *book)
{
    /* src/rsolvergeneric.cpp:508-535: every node of a group with an explicit condition is disabled */
    std::vector<uint8_t> disabled(n_nodes, 0);
    for (uint32_t g = 0; g < n_groups; g++) {
        if (!explicit_bc[g]) continue;
        for (uint32_t j = group_begin[g]; j < group_begin[g + 1]; j++) {
            const uint32_t e = group_elems[j];
            for (uint32_t k = elem_begin[e]; k < elem_begin[e + 1]; k++) disabled[elem_nodes[k]] = 1;
        }
    }
    orc_disable_not_computable(n_nodes, n_elements, elem_begin, elem_nodes, computable, 1, disabled);
    return orc_node_book(n_nodes, disabled.data(), book);
}

uint32_t orc_node_book_stress(uint32_t n_nodes, uint32_t n_elements, const uint32_t *elem_begin,
                              const uint32_t *elem_nodes, uint32_t n_groups, const uint32_t *group_begin,
                              const uint32_t *group_elems, const uint8_t *computable, const uint8_t *bc,
                              const uint8_t *is_line, uint32_t *book)
{
    /* src/rsolverstress.cpp:1569-1629: displacement / normal displacement disable x, y, z; a roller
     * disables y and z on a line group, x elsewhere; groups without any of these are skipped */
    std::vector<uint8_t> disabled(size_t(n_nodes) * 3, 0);
    for (uint32_t g = 0; g < n_groups; g++) {
        bool dx = false, dy = false, dz = false;
        if (bc[g] & 3u) dx = dy = dz = true;
        if (bc[g] & 4u) {
            if (is_line[g]) dy = dz = true;
            else dx = true;
        }
        if (!dx && !dy && !dz) continue;
        for (uint32_t j = group_begin[g]; j < group_begin[g + 1]; j++) {
            const uint32_t e = group_elems[j];
            for (uint32_t k = elem_begin[e]; k < elem_begin[e + 1]; k++) {
                const uint32_t node = elem_nodes[k];
                if (dx) disabled[3 * size_t(node) + 0] = 1;
                if (dy) disabled[3 * size_t(node) + 1] = 1;
                if (dz) disabled[3 * size_t(node) + 2] = 1;
            }
        }
    }
    /* :1630-1651 */
    orc_disable_not_computable(n_nodes, n_elements, elem_begin, elem_nodes, computable, 3, disabled);
    /* RBook::disable renumbers the enabled positions consecutively, as rebuildNodeBook does */
    return orc_node_book(3 * n_nodes, disabled.data(), book);
}

uint32_t orc_system_n(const orc_system *s) { return s->n; }
uint64_t orc_system_nnz(const orc_system *s) { return s->ci.size(); }
void orc_system_copy(const orc_system *s, uint32_t *rp, uint32_t *ci, double *val, double *b)
{
    std::memcpy(rp, s->rp.data(), s->rp.size() * sizeof(uint32_t));
    std::memcpy(ci, s->ci.data(), s->ci.size() * sizeof(uint32_t));
    std::memcpy(val, s->val.data(), s->val.size() * sizeof(double));
    std::memcpy(b, s->b.data(), s->b.size() * sizeof(double));
}
void orc_system_free(orc_system *s) { delete s; }

/* The mass integral int N_m N_n over a tetrahedron of volume V under the quadrature rule of orc_time. */
static double tet_mass(int rule, double V, int m, int n)
{
    if (rule == 1) return V / 16.0;
    if (rule == 2) return m == n ? V / 4.0 : 0.0;
    return V * (m == n ? 2.0 : 1.0) / 20.0;
}

orc_system *orc_assemble_heat(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                              const double *k_e, const double *q_e, const double *rhoc_e, const double *node_t,
                              const uint32_t *book, uint32_t n_free, const orc_time *time)
{
    (void)n_nodes;
    RowMap A(n_free);
    std::vector<double> b(n_free, 0.0);
    const bool transient = time && time->transient;
    const double alpha = time ? time->alpha : 1.0, dt = time ? time->dt : 0.0;
    for (uint32_t e = 0; e < n_tets; e++) {
        const uint32_t *t = tets + 4 * size_t(e);
        /* src/rsolverheat.cpp:397-435: Ke = k B B^T detJ w, Me = N N^T rho c detJ w, fe = Q N detJ w,
         * restated with the exact P1 integrals (constant B; int N = V/4; int N_m N_n = V(1+d_mn)/20). */
        double G[4][3];
        double V = std::abs(tet_gradients(xyz, t, G)) / 6.0;
        double Ke[4][4], Me[4][4], fe[4];
        for (int m = 0; m < 4; m++) {
            for (int n = 0; n < 4; n++) {
                Ke[m][n] = (G[m][0] * G[n][0] + G[m][1] * G[n][1] + G[m][2] * G[n][2]) * k_e[e] * V;
                Me[m][n] = transient ? rhoc_e[e] * tet_mass(time->mass_rule, V, m, n) : 0.0;
            }
            fe[m] = q_e[e] * V / 4.0;
        }
        /* src/rsolverheat.cpp:755-820 (assemblyMatrix) */
        double Ae[4][4], be[4];
        if (transient) {
            for (int m = 0; m < 4; m++) {
                be[m] = dt * fe[m];
                for (int n = 0; n < 4; n++) {
                    Ae[m][n] = Me[m][n] + alpha * dt * Ke[m][n];
                    be[m] += (Me[m][n] - (1.0 - alpha) * dt * Ke[m][n]) * node_t[t[n]];
                }
            }
        } else {
            for (int m = 0; m < 4; m++) {
                be[m] = fe[m];
                for (int n = 0; n < 4; n++) Ae[m][n] = Ke[m][n];
            }
        }
        for (int m = 0; m < 4; m++)
            if (book[t[m]] == kEod)
                for (int n = 0; n < 4; n++) be[n] -= Ae[n][m] * node_t[t[m]];
        for (int m = 0; m < 4; m++) {
            uint32_t mp = book[t[m]];
            if (mp == kEod) continue;
            b[mp] += be[m];
            for (int n = 0; n < 4; n++) {
                uint32_t np = book[t[n]];
                if (np != kEod) A.add(mp, np, Ae[m][n]);
            }
        }
    }
    return finish_system(A, b);
}

orc_system *orc_assemble_stress(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                                const double *e_mod, const double *nu, const double *rho_e, const double *gravity,
                                const double *texp_e, const double *dtemp_e, uint32_t n_tris, const uint32_t *tris,
                                const double *traction, const double *node_u, const uint32_t *book,
                                uint32_t n_free, const orc_time *time)
{
    (void)n_nodes;
    RowMap A(n_free);
    std::vector<double> b(n_free, 0.0);
    const bool transient = time && time->transient;
    const double alpha = time ? time->alpha : 1.0, dt = time ? time->dt : 0.0;

    /* src/rsolverstress.cpp:1654-1772 (assemblyMatrix); local rotations are identity here (:1774-1804). */
    auto assemble = [&](const uint32_t *nodes, int nn, const double *Ke, const double *Me, const double *fe) {
        const int nd = 3 * nn;
        double Ae[144], be[12];
        for (int i = 0; i < nd; i++) {
            be[i] = transient ? dt * fe[i] : fe[i];
            for (int j = 0; j < nd; j++) {
                double k = Ke[i * nd + j], m = Me ? Me[i * nd + j] : 0.0;
                Ae[i * nd + j] = transient ? m + alpha * dt * k : k;
            }
        }
        if (transient)
            for (int i = 0; i < nd; i++)
                for (int j = 0; j < nd; j++) {
                    double k = Ke[i * nd + j], m = Me ? Me[i * nd + j] : 0.0;
                    be[i] += (m - (1.0 - alpha) * dt * k) * node_u[3 * size_t(nodes[j / 3]) + j % 3];
                }
        for (int m = 0; m < nn; m++)
            for (int n = 0; n < nd; n++)
                for (int i = 0; i < 3; i++)
                    if (book[3 * size_t(nodes[m]) + i] == kEod)
                        be[n] -= Ae[n * nd + 3 * m + i] * node_u[3 * size_t(nodes[m]) + i];
        for (int m = 0; m < nn; m++)
            for (int i = 0; i < 3; i++) {
                uint32_t mp = book[3 * size_t(nodes[m]) + i];
                if (mp == kEod) continue;
                b[mp] += be[3 * m + i];
                for (int n = 0; n < nn; n++)
                    for (int j = 0; j < 3; j++) {
                        uint32_t np = book[3 * size_t(nodes[n]) + j];
                        if (np != kEod) A.add(mp, np, Ae[(3 * m + i) * nd + 3 * n + j]);
                    }
            }
    };

    /* Surface traction: src/rsolverstress.cpp:384-570 with thickness 0 (no stiffness);
     * force per unit area (:504-507) integrated with int N_m = Area/3. */
    for (uint32_t f = 0; f < n_tris; f++) {
        const uint32_t *t = tris + 3 * size_t(f);
        double a[3], c[3];
        for (int k = 0; k < 3; k++) {
            a[k] = xyz[3 * size_t(t[1]) + k] - xyz[3 * size_t(t[0]) + k];
            c[k] = xyz[3 * size_t(t[2]) + k] - xyz[3 * size_t(t[0]) + k];
        }
        double cr[3] = {a[1] * c[2] - a[2] * c[1], a[2] * c[0] - a[0] * c[2], a[0] * c[1] - a[1] * c[0]};
        double area = 0.5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        double Ke[81] = {0}, fe[9];
        for (int m = 0; m < 3; m++)
            for (int k = 0; k < 3; k++) fe[3 * m + k] = traction[3 * size_t(f) + k] * area / 3.0;
        assemble(t, 3, Ke, nullptr, fe);
    }

    /* Volumes: src/rsolverstress.cpp:573-715 */
    for (uint32_t e = 0; e < n_tets; e++) {
        const uint32_t *t = tets + 4 * size_t(e);
        double G[4][3];
        double V = std::abs(tet_gradients(xyz, t, G)) / 6.0;
        const double E = e_mod[e], v = nu[e];
        double De[6][6] = {{0}};
        De[0][0] = 1.0 - v; De[0][1] = v;       De[0][2] = v;
        De[1][0] = v;       De[1][1] = 1.0 - v; De[1][2] = v;
        De[2][0] = v;       De[2][1] = v;       De[2][2] = 1.0 - v;
        De[3][3] = De[4][4] = De[5][5] = (1.0 - 2.0 * v) / 2.0;
        const double f = E / ((1.0 + v) * (1.0 - 2.0 * v));
        for (auto &row : De)
            for (auto &x : row) x *= f;
        /* Be (12x6), strain order xx, yy, zz, yz, xz, xy (:643-651) */
        double Be[12][6] = {{0}};
        for (int m = 0; m < 4; m++) {
            Be[3 * m + 0][0] = G[m][0];
            Be[3 * m + 1][1] = G[m][1];
            Be[3 * m + 2][2] = G[m][2];
            Be[3 * m + 1][3] = G[m][2];
            Be[3 * m + 2][3] = G[m][1];
            Be[3 * m + 0][4] = G[m][2];
            Be[3 * m + 2][4] = G[m][0];
            Be[3 * m + 0][5] = G[m][1];
            Be[3 * m + 1][5] = G[m][0];
        }
        double BeD[12][6];
        for (int i = 0; i < 12; i++)
            for (int j = 0; j < 6; j++) {
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += Be[i][k] * De[k][j];
                BeD[i][j] = s;
            }
        double Ke[144], Me[144], fe[12];
        for (int i = 0; i < 12; i++)
            for (int j = 0; j < 12; j++) {
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += BeD[i][k] * Be[j][k];
                Ke[i * 12 + j] = s * V;
                Me[i * 12 + j] = 0.0;
            }
        if (transient)
            for (int m = 0; m < 4; m++)
                for (int n = 0; n < 4; n++) {
                    double value = rho_e[e] * tet_mass(time->mass_rule, V, m, n);
                    for (int k = 0; k < 3; k++) Me[(3 * m + k) * 12 + 3 * n + k] = value;
                }
        for (int m = 0; m < 4; m++)
            for (int k = 0; k < 3; k++) {
                /* own weight (:683-685) and thermal expansion (:688-693) */
                double val = gravity[k] * rho_e[e] * V / 4.0;
                for (int n = 0; n < 3; n++) val += texp_e[e] * dtemp_e[e] * BeD[3 * m + k][n] * V;
                fe[3 * m + k] = val;
            }
        assemble(t, 4, Ke, Me, fe);
    }
    return finish_system(A, b);
}

/* Magnetostatics (vector potential, 3 dofs per node interleaved, all three disabled together):
 * RSolverMagnetostatics::prepare volume loop (src/rsolvermagnetostatics.cpp:57-137) and
 * assemblyMatrix (:234-287).  Per tet, for node pair (m, n): Ke[3m+c][3n+c] = -(B_m . B_n) detJ w and
 * zero off the component diagonal (the zero entries are still added to the pattern, :272-282);
 * fe[3m+c] = N_m detJ w e0 (B_m x J_m)_c with J_m the current density of node m (:110-119), restated
 * with the exact P1 integrals (constant B = grad N; int N_m = V/4). */
orc_system *orc_assemble_magnetostatics(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                                        const double *node_j, const double *node_a, const uint32_t *book,
                                        uint32_t n_free)
{
    (void)n_nodes;
    const double e0 = 8.854187817e-12; /* RSolverGeneric::e0 (src/rsolvergeneric.cpp:13) */
    RowMap A(n_free);
    std::vector<double> b(n_free, 0.0);
    for (uint32_t e = 0; e < n_tets; e++) {
        const uint32_t *t = tets + 4 * size_t(e);
        double G[4][3];
        double V = std::abs(tet_gradients(xyz, t, G)) / 6.0;
        double Ke[12][12], be[12];
        for (int i = 0; i < 12; i++)
            for (int j = 0; j < 12; j++) Ke[i][j] = 0.0;
        for (int m = 0; m < 4; m++) {
            for (int n = 0; n < 4; n++) {
                const double v = (G[m][0] * G[n][0] + G[m][1] * G[n][1] + G[m][2] * G[n][2]) * V;
                for (int c = 0; c < 3; c++) Ke[3 * m + c][3 * n + c] -= v;
            }
            const double fv = V / 4.0 * e0;
            const double *J = node_j + 3 * size_t(t[m]);
            const double js[3] = {-G[m][2] * J[1] + G[m][1] * J[2], G[m][2] * J[0] - G[m][0] * J[2],
                                  -G[m][1] * J[0] + G[m][0] * J[1]};
            for (int c = 0; c < 3; c++) be[3 * m + c] = fv * js[c];
        }
        /* :240-254 -- lifting by the prescribed potential of disabled nodes */
        for (int m = 0; m < 4; m++)
            if (book[3 * size_t(t[m])] == kEod)
                for (int n = 0; n < 12; n++)
                    for (int c = 0; c < 3; c++) be[n] -= Ke[n][3 * m + c] * node_a[3 * size_t(t[m]) + c];
        /* :256-286 */
        for (int m = 0; m < 4; m++) {
            if (book[3 * size_t(t[m])] == kEod) continue;
            for (int i = 0; i < 3; i++) {
                const uint32_t mp = book[3 * size_t(t[m]) + i];
                b[mp] += be[3 * m + i];
                for (int n = 0; n < 4; n++) {
                    if (book[3 * size_t(t[n])] == kEod) continue;
                    for (int j = 0; j < 3; j++) A.add(mp, book[3 * size_t(t[n]) + j], Ke[3 * m + i][3 * n + j]);
                }
            }
        }
    }
    return finish_system(A, b);
}

}  // extern "C"

/* ------------------------------------------------------------------------------------------------
 * Multilevel aggregation preconditioner (no reference counterpart).  Serial restatement of the
 * CUDA library's set-up (range-solver-lib_b200/csrc/amg.cu): every integer decision and every
 * floating-point sum is taken in the same order, so the hierarchy is identical bit for bit; the
 * cycle (levels 1..2 as K-cycle levels: two flexible-CG steps) runs in FP64 here (FP32 on the GPU).
 * ------------------------------------------------------------------------------------------------ */
namespace {

constexpr uint32_t kAmgCoarsest = 128, kAmgMaxEntries = 4096, kAmgUnset = 0xffffffffu;
constexpr double kAmgTheta = 0.08, kAmgOmega = 2.0 / 3.0, kAmgScale1 = 1.6, kAmgScale2 = 1.8;
constexpr size_t kAmgKLevels = 2;  /* levels 1..2 are solved by two flexible-CG steps (K-cycle) */

uint32_t amg_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
uint64_t amg_key(uint32_t i) { return (uint64_t(amg_hash(i) >> 2) << 32) | i; }

struct AmgLev {
    uint32_t n = 0;
    std::vector<uint32_t> rp, ci, agg, agg_ptr, agg_rows;
    std::vector<double> val, diag, dw;
};

}  // namespace

struct orc_amg {
    std::vector<AmgLev> L;
    bool dense = false;
    std::vector<double> inv;  /* dense inverse of the last level */
};

namespace {

void amg_level_diag(AmgLev &l)
{
    l.diag.assign(l.n, 0.0);
    l.dw.assign(l.n, 0.0);
    for (uint32_t i = 0; i < l.n; i++) {
        double d = 0.0;
        for (uint32_t j = l.rp[i]; j < l.rp[i + 1]; j++)
            if (l.ci[j] == i) d = l.val[j];
        l.diag[i] = d;
        l.dw[i] = d != 0.0 ? kAmgOmega / d : 0.0;
    }
}

/* aggregates of level F; returns the coarse size, the largest entry count of a coarse row and the
 * largest aggregate */
uint32_t amg_aggregate(AmgLev &F, uint32_t &emax, uint32_t &smax)
{
    const uint32_t n = F.n;
    std::vector<uint8_t> strong(F.ci.size(), 0);
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++) {
            const uint32_t c = F.ci[j];
            strong[j] = (c != i && c < n && std::abs(F.val[j]) >= kAmgTheta * std::sqrt(std::abs(F.diag[i] * F.diag[c])) &&
                         F.val[j] != 0.0) ? 1 : 0;
        }
    /* synchronous rounds: state 0 out, 1 undecided, 2 root */
    std::vector<uint64_t> T(n), M1(n), M2(n);
    for (uint32_t i = 0; i < n; i++) T[i] = (uint64_t(1) << 62) | amg_key(i);
    auto nbmax = [&](const std::vector<uint64_t> &in, std::vector<uint64_t> &out) {
        for (uint32_t i = 0; i < n; i++) {
            uint64_t m = in[i];
            for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++)
                if (strong[j]) m = std::max(m, in[F.ci[j]]);
            out[i] = m;
        }
    };
    for (;;) {
        nbmax(T, M1);
        nbmax(M1, M2);
        uint32_t left = 0;
        for (uint32_t i = 0; i < n; i++) {
            if ((T[i] >> 62) != 1) continue;
            if (M2[i] == T[i]) T[i] = (uint64_t(2) << 62) | amg_key(i);
            else if ((M2[i] >> 62) == 2) T[i] = amg_key(i);
            else left++;
        }
        if (!left) break;
    }
    std::vector<uint32_t> rank(n, 0);
    uint32_t nc = 0;
    for (uint32_t i = 0; i < n; i++) {
        rank[i] = nc;
        if ((T[i] >> 62) == 2) nc++;
    }
    std::vector<uint32_t> a1(n, kAmgUnset);
    for (uint32_t i = 0; i < n; i++) {
        if ((T[i] >> 62) == 2) {
            a1[i] = rank[i];
            continue;
        }
        uint64_t best = 0;
        for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++)
            if (strong[j] && (T[F.ci[j]] >> 62) == 2) best = std::max(best, T[F.ci[j]]);
        if (best) a1[i] = rank[uint32_t(best & 0xffffffffu)];
    }
    F.agg.assign(n, kAmgUnset);
    uint32_t left = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t a = a1[i];
        if (a == kAmgUnset) {
            uint64_t best = 0;
            for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++) {
                const uint32_t c = F.ci[j];
                if (!strong[j] || a1[c] == kAmgUnset) continue;
                if (amg_key(c) + 1 > best) {
                    best = amg_key(c) + 1;
                    a = a1[c];
                }
            }
            if (a == kAmgUnset) left++;
        }
        F.agg[i] = a;
    }
    if (left) {
        uint32_t next = nc;
        for (uint32_t i = 0; i < n; i++)
            if (F.agg[i] == kAmgUnset) F.agg[i] = next++;
        nc = next;
    }
    F.agg_ptr.assign(size_t(nc) + 1, 0);
    for (uint32_t i = 0; i < n; i++) F.agg_ptr[F.agg[i] + 1]++;
    for (uint32_t a = 0; a < nc; a++) F.agg_ptr[a + 1] += F.agg_ptr[a];
    F.agg_rows.assign(n, 0);
    std::vector<uint32_t> cur(F.agg_ptr.begin(), F.agg_ptr.end() - 1);
    for (uint32_t i = 0; i < n; i++) F.agg_rows[cur[F.agg[i]]++] = i;  /* ascending within each aggregate */
    emax = smax = 0;
    for (uint32_t a = 0; a < nc; a++) {
        uint32_t e = 0;
        for (uint32_t k = F.agg_ptr[a]; k < F.agg_ptr[a + 1]; k++) e += F.rp[F.agg_rows[k] + 1] - F.rp[F.agg_rows[k]];
        emax = std::max(emax, e);
        smax = std::max(smax, F.agg_ptr[a + 1] - F.agg_ptr[a]);
    }
    return nc;
}

/* C = P^T A P: entries of coarse row I in (J ascending, then the order of the aggregate's rows and
 * of the entries within each row), each run of equal J added serially */
void amg_galerkin(const AmgLev &F, AmgLev &C, uint32_t nc)
{
    C.n = nc;
    C.rp.assign(size_t(nc) + 1, 0);
    C.ci.clear();
    C.val.clear();
    std::vector<std::pair<uint32_t, uint32_t>> ent;  /* (J, staging position) */
    std::vector<double> v;
    for (uint32_t I = 0; I < nc; I++) {
        ent.clear();
        v.clear();
        for (uint32_t k = F.agg_ptr[I]; k < F.agg_ptr[I + 1]; k++) {
            const uint32_t i = F.agg_rows[k];
            for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++) {
                ent.emplace_back(F.agg[F.ci[j]], uint32_t(v.size()));
                v.push_back(F.val[j]);
            }
        }
        std::sort(ent.begin(), ent.end());
        for (size_t t = 0; t < ent.size();) {
            const uint32_t J = ent[t].first;
            double s = 0.0;
            for (; t < ent.size() && ent[t].first == J; t++) s += v[ent[t].second];
            C.ci.push_back(J);
            C.val.push_back(s);
        }
        C.rp[I + 1] = uint32_t(C.ci.size());
    }
}

/* in-place Gauss-Jordan inverse without pivoting (SPD); a non-positive pivot zeroes its row and column */
void amg_dense_inverse(const AmgLev &l, std::vector<double> &a)
{
    const uint32_t n = l.n;
    a.assign(size_t(n) * n, 0.0);
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = l.rp[i]; j < l.rp[i + 1]; j++)
            if (l.ci[j] < n) a[size_t(i) * n + l.ci[j]] = l.val[j];
    for (uint32_t k = 0; k < n; k++) {
        const double p = a[size_t(k) * n + k];
        if (!(p > 0.0)) {
            for (uint32_t t = 0; t < n; t++) a[size_t(k) * n + t] = a[size_t(t) * n + k] = 0.0;
            continue;
        }
        const double pinv = 1.0 / p;
        for (uint32_t j = 0; j < n; j++) a[size_t(k) * n + j] = (j == k) ? pinv : a[size_t(k) * n + j] * pinv;
        for (uint32_t i = 0; i < n; i++) {
            if (i == k) continue;
            for (uint32_t j = 0; j < n; j++)
                if (j != k) a[size_t(i) * n + j] -= a[size_t(i) * n + k] * a[size_t(k) * n + j];
        }
        for (uint32_t i = 0; i < n; i++)
            if (i != k) a[size_t(i) * n + k] = -a[size_t(i) * n + k] * pinv;
    }
}

/* out = x + dw (b - A x) (smooth) or b - A x (residual) */
void amg_sweep(const AmgLev &l, const std::vector<double> &b, const std::vector<double> &x, std::vector<double> &out,
               bool smooth)
{
    for (uint32_t i = 0; i < l.n; i++) {
        double ax = 0.0;
        for (uint32_t j = l.rp[i]; j < l.rp[i + 1]; j++) ax += l.val[j] * x[l.ci[j]];
        const double res = b[i] - ax;
        out[i] = smooth ? x[i] + l.dw[i] * res : res;
    }
}

bool amg_k_level(const orc_amg &H, size_t l) { return l >= 1 && l <= kAmgKLevels && l + 1 < H.L.size(); }

void amg_solve_level(const orc_amg &H, size_t lv, const std::vector<double> &b, std::vector<double> &e,
                     uint32_t sweeps);

/* one cycle on level lv: smoothing from zero, residual, restriction, the coarser level, prolongation
 * (scaled by 1.6 / 1.8 unless the coarser level is a K-cycle level), smoothing */
void amg_cycle(const orc_amg &H, size_t lv, const std::vector<double> &b, std::vector<double> &e, uint32_t sweeps)
{
    const AmgLev &F = H.L[lv];
    const uint32_t n = F.n;
    const double s = amg_k_level(H, lv + 1) ? 1.0 : (sweeps == 2 ? kAmgScale2 : kAmgScale1);
    std::vector<double> x(n, 0.0), t(n), r(n);
    amg_sweep(F, b, x, t, true);           /* x = dw b */
    x.swap(t);
    for (uint32_t k = 1; k < sweeps; k++) {
        amg_sweep(F, b, x, t, true);
        x.swap(t);
    }
    amg_sweep(F, b, x, r, false);
    const AmgLev &C = H.L[lv + 1];
    std::vector<double> bc(C.n, 0.0), ec;
    for (uint32_t I = 0; I < C.n; I++) {
        double acc = 0.0;
        for (uint32_t k = F.agg_ptr[I]; k < F.agg_ptr[I + 1]; k++) acc += r[F.agg_rows[k]];
        bc[I] = acc;
    }
    amg_solve_level(H, lv + 1, bc, ec, sweeps);
    for (uint32_t i = 0; i < n; i++) x[i] += s * ec[F.agg[i]];
    for (uint32_t k = 0; k < sweeps; k++) {
        amg_sweep(F, b, x, t, true);
        x.swap(t);
    }
    e = x;
}

double amg_dot(const std::vector<double> &u, const std::vector<double> &v)
{
    double s = 0.0;
    for (size_t i = 0; i < u.size(); i++) s += u[i] * v[i];
    return s;
}

/* e ~ A_lv^-1 b: the dense inverse on the last level, two flexible-CG steps preconditioned by the
 * cycle on a K-cycle level (Notay's K-cycle), one cycle otherwise */
void amg_solve_level(const orc_amg &H, size_t lv, const std::vector<double> &b, std::vector<double> &e,
                     uint32_t sweeps)
{
    const AmgLev &F = H.L[lv];
    const uint32_t n = F.n;
    if (lv + 1 == H.L.size()) {
        e.assign(n, 0.0);
        if (H.dense) {
            for (uint32_t i = 0; i < n; i++) {
                double s = 0.0;
                for (uint32_t j = 0; j < n; j++) s += H.inv[size_t(i) * n + j] * b[j];
                e[i] = s;
            }
        } else {  /* coarsening stalled: nine damped-Jacobi sweeps from zero */
            std::vector<double> x(n, 0.0), y(n);
            for (int k = 0; k < 9; k++) {
                amg_sweep(F, b, x, y, true);
                x.swap(y);
            }
            e = x;
        }
        return;
    }
    if (!amg_k_level(H, lv)) {
        amg_cycle(H, lv, b, e, sweeps);
        return;
    }
    std::vector<double> c1, c2, v1(n), v2(n), r2(n);
    auto mul = [&](const std::vector<double> &c, std::vector<double> &v) {
        for (uint32_t i = 0; i < n; i++) {
            double acc = 0.0;
            for (uint32_t j = F.rp[i]; j < F.rp[i + 1]; j++) acc += F.val[j] * c[F.ci[j]];
            v[i] = acc;
        }
    };
    amg_cycle(H, lv, b, c1, sweeps);
    mul(c1, v1);
    const double d1 = amg_dot(c1, v1), t1 = amg_dot(c1, b);
    const double a1 = d1 > 0.0 ? t1 / d1 : 0.0;
    for (uint32_t i = 0; i < n; i++) r2[i] = b[i] - a1 * v1[i];
    amg_cycle(H, lv, r2, c2, sweeps);
    mul(c2, v2);
    const double d2 = amg_dot(c2, v2), g = amg_dot(c2, v1), t2 = amg_dot(c2, r2);
    double g1 = 0.0, a2 = 0.0;
    if (d1 > 0.0) {
        const double b2 = d2 - g * g / d1;
        a2 = b2 > 0.0 ? t2 / b2 : 0.0;
        g1 = t1 / d1 - g * a2 / d1;
    }
    e.assign(n, 0.0);
    for (uint32_t i = 0; i < n; i++) e[i] = g1 * c1[i] + a2 * c2[i];
}

}  // namespace

extern "C" {

orc_amg *orc_amg_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val)
{
    auto *H = new orc_amg;
    H->L.emplace_back();
    AmgLev &L0 = H->L.back();
    L0.n = n;
    L0.rp.assign(rp, rp + n + 1);
    L0.ci.assign(ci, ci + rp[n]);
    L0.val.assign(val, val + rp[n]);
    amg_level_diag(L0);
    while (H->L.size() < 12) {
        AmgLev &F = H->L.back();
        if (F.n <= kAmgCoarsest) {
            H->dense = true;
            break;
        }
        uint32_t emax = 0, smax = 0;
        const uint32_t nc = amg_aggregate(F, emax, smax);
        if (nc == 0 || uint64_t(nc) * 10 > uint64_t(F.n) * 9 || emax > kAmgMaxEntries || smax > kAmgMaxEntries) {
            F.agg.clear();
            break;
        }
        AmgLev C;
        amg_galerkin(F, C, nc);
        amg_level_diag(C);
        H->L.push_back(std::move(C));
    }
    if (H->dense) amg_dense_inverse(H->L.back(), H->inv);
    return H;
}

uint32_t orc_amg_levels(const orc_amg *h) { return uint32_t(h->L.size()); }
int32_t orc_amg_dense_coarsest(const orc_amg *h) { return h->dense ? 1 : 0; }
uint32_t orc_amg_rows(const orc_amg *h, uint32_t level) { return h->L[level].n; }
uint64_t orc_amg_nnz(const orc_amg *h, uint32_t level) { return h->L[level].ci.size(); }

void orc_amg_level(const orc_amg *h, uint32_t level, uint32_t *agg, uint32_t *row_ptr, uint32_t *col_idx,
                   double *values)
{
    const AmgLev &l = h->L[level];
    if (agg && !l.agg.empty()) std::memcpy(agg, l.agg.data(), l.agg.size() * sizeof(uint32_t));
    if (row_ptr) std::memcpy(row_ptr, l.rp.data(), l.rp.size() * sizeof(uint32_t));
    if (col_idx) std::memcpy(col_idx, l.ci.data(), l.ci.size() * sizeof(uint32_t));
    if (values) std::memcpy(values, l.val.data(), l.val.size() * sizeof(double));
}

void orc_amg_apply(const orc_amg *h, const double *r, double *z, uint32_t sweeps)
{
    const AmgLev &F = h->L[0];
    std::vector<double> b(r, r + F.n), e;
    if (h->L.size() == 1 && !h->dense) {  /* no coarse level: damped Jacobi */
        for (uint32_t i = 0; i < F.n; i++) z[i] = F.dw[i] * r[i];
        return;
    }
    if (h->L.size() == 1) amg_solve_level(*h, 0, b, e, sweeps);  /* one dense level */
    else amg_cycle(*h, 0, b, e, sweeps);
    std::memcpy(z, e.data(), F.n * sizeof(double));
}

void orc_amg_free(orc_amg *h) { delete h; }

// RSolverFluid::buildSparseMatrixPattern (src/rsolverfluid.cpp:2305-2397) and assemblyMatrix (:2399-2419):
// rows as ordered maps column -> value; the pattern pass inserts zeros for every pair of an active
// element's enabled DOFs, the assembly pass adds each active element's matrix and vector in element
// order.  Ae / fe hold the active elements' blocks concatenated in element order.
uint64_t orc_scatter_assemble(uint32_t d, uint32_t ne, const uint32_t *elem_begin, const uint32_t *elem_nodes,
                              const uint8_t *elem_active, uint32_t n_nodes, const uint32_t *book, uint32_t n_free,
                              const double *Ae, const double *fe, uint32_t *rp, uint32_t *ci, double *val, double *b)
{
    (void)n_nodes;
    std::vector<std::map<uint32_t, double>> A(n_free);
    std::vector<double> bp(n_free, 0.0);
    std::vector<std::vector<uint32_t>> active(ne), vpos(ne);  // local DOF, equation row
    for (uint32_t e = 0; e < ne; e++) {
        if (elem_active && !elem_active[e]) continue;
        for (uint32_t m = 0; m < elem_begin[e + 1] - elem_begin[e]; m++)
            for (uint32_t i = 0; i < d; i++) {
                const uint32_t mp = book[size_t(elem_nodes[elem_begin[e] + m]) * d + i];
                if (mp == 0xffffffffu) continue;
                active[e].push_back(m * d + i);
                vpos[e].push_back(mp);
            }
        for (uint32_t r : vpos[e])
            for (uint32_t c : vpos[e]) A[r].emplace(c, 0.0);
    }
    if (Ae && fe) {
        size_t ae_off = 0, fe_off = 0;
        for (uint32_t e = 0; e < ne; e++) {
            if (elem_active && !elem_active[e]) continue;
            const size_t nd = size_t(elem_begin[e + 1] - elem_begin[e]) * d;
            for (size_t a = 0; a < active[e].size(); a++) {
                bp[vpos[e][a]] += fe[fe_off + active[e][a]];
                for (size_t c = 0; c < active[e].size(); c++)
                    A[vpos[e][a]][vpos[e][c]] += Ae[ae_off + active[e][a] * nd + active[e][c]];
            }
            ae_off += nd * nd;
            fe_off += nd;
        }
    }
    uint64_t nnz = 0;
    for (uint32_t r = 0; r < n_free; r++) {
        if (rp) rp[r] = uint32_t(nnz);
        for (const auto &kv : A[r]) {
            if (ci) ci[nnz] = kv.first;
            if (val) val[nnz] = kv.second;
            nnz++;
        }
    }
    if (rp) rp[n_free] = uint32_t(nnz);
    if (b) std::copy(bp.begin(), bp.end(), b);
    return nnz;
}

}  // extern "C"
