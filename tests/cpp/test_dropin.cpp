// C++ drop-in check: the reference's own matrix-solver tests
// (tests/tst_matrix_solver.cpp:33-77 in the reference project) written
// against rsg::dropin::RMatrixSolver, plus a cache-refresh case.
#include <cmath>
#include <cstdio>

#include "rsg_rmatrixsolver.hpp"

using namespace rsg::dropin;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            failures++;                                            \
        }                                                          \
    } while (0)

static RMatrixSolverConf makeCgConf()
{
    RMatrixSolverConf conf(RMatrixSolverConf::CG);
    conf.setNInnerIterations(1000);
    conf.setNOuterIterations(1000);
    conf.setSolverCvgValue(1.0e-13);
    conf.setOutputFrequency(0);
    return conf;
}

int main()
{
    const double tol = 1.0e-6;
    {
        RSparseMatrix a;
        a.setNRows(2);
        a.addValue(0, 0, 4.0);
        a.addValue(0, 1, 1.0);
        a.addValue(1, 0, 1.0);
        a.addValue(1, 1, 3.0);
        RRVector b(2, 0.0);
        b[0] = 1.0;
        b[1] = 2.0;
        RRVector x;
        RMatrixSolver solver(makeCgConf());
        solver.solve(a, b, x);
        CHECK(x.getNRows() == 2u);
        CHECK(std::fabs(x[0] - 1.0 / 11.0) < tol);
        CHECK(std::fabs(x[1] - 7.0 / 11.0) < tol);
    }
    {
        RSparseMatrix a;
        a.setNRows(3);
        a.addValue(0, 0, 2.0);
        a.addValue(1, 1, 4.0);
        a.addValue(2, 2, 5.0);
        RRVector b(3, 0.0);
        b[0] = 6.0;
        b[1] = 8.0;
        b[2] = 10.0;
        RRVector x;
        RMatrixSolver solver(makeCgConf());
        solver.solve(a, b, x);
        CHECK(std::fabs(x[0] - 3.0) < tol);
        CHECK(std::fabs(x[1] - 2.0) < tol);
        CHECK(std::fabs(x[2] - 2.0) < tol);
        // same matrix object, new values, same pattern: cache refresh path
        a.addValue(0, 0, 2.0);  // 4
        RRVector x2;
        solver.solve(a, b, x2, R_MATRIX_PRECONDITIONER_JACOBI);
        CHECK(std::fabs(x2[0] - 1.5) < tol);
    }
    {
        // 1-D Laplacian, GMRES with Jacobi
        const unsigned n = 200;
        RSparseMatrix a;
        a.setNRows(n);
        for (unsigned i = 0; i < n; i++) {
            a.addValue(i, i, 2.0);
            if (i) a.addValue(i, i - 1, -1.0);
            if (i + 1 < n) a.addValue(i, i + 1, -1.0);
        }
        RRVector b(n, 1.0), x;
        RMatrixSolverConf conf(RMatrixSolverConf::GMRES);
        conf.setNInnerIterations(50);
        conf.setNOuterIterations(500);
        conf.setSolverCvgValue(1.0e-14);
        conf.setOutputFrequency(0);
        RMatrixSolver solver(conf);
        solver.solve(a, b, x, R_MATRIX_PRECONDITIONER_JACOBI);
        double worst = 0.0;
        for (unsigned i = 0; i < n; i++) {
            const double exact = 0.5 * (i + 1) * (n - i);
            worst = std::fmax(worst, std::fabs(x[i] - exact) / exact);
        }
        CHECK(worst < 1e-7);
    }
    {
        bool threw = false;
        try {
            RSparseMatrix a;
            a.setNRows(1);
            a.addValue(0, 0, 1.0);
            RRVector b(1, 1.0), x;
            RMatrixSolver solver(makeCgConf());
            solver.solve(a, b, x, RMatrixPreconditionerType(7));
        } catch (const RError &) {
            threw = true;
        }
        CHECK(threw);
    }
    std::printf(failures ? "dropin: %d failures\n" : "dropin: all passed\n", failures);
    return failures ? 1 : 0;
}
