// Stand-ins for range-base-lib's RRVector and RRMatrix (TEST INFRASTRUCTURE): dense FP64 vector
// and row-major matrix with the members the reference's solver and eigenvalue sources call.
// invert() is Gauss-Jordan elimination with partial pivoting (range-base-lib's own method is not
// published with the reference); a singular matrix throws RError.  dot / norm / mlt sum in index
// order; normalize() divides by the norm.
#ifndef REF_SHIM_RBL_RMATRIX_H
#define REF_SHIM_RBL_RMATRIX_H

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "rbl_utils.h"

class RRVector
{
    protected:
        std::vector<double> v;

    public:
        RRVector() = default;
        explicit RRVector(uint n, double value = 0.0) : v(n, value) {}

        double &operator[](uint i) { return v[i]; }
        const double &operator[](uint i) const { return v[i]; }

        uint getNRows() const { return uint(v.size()); }
        uint size() const { return uint(v.size()); }
        void resize(uint n) { v.resize(n); }
        void resize(uint n, double value) { v.resize(n, value); }
        void fill(double value) { std::fill(v.begin(), v.end(), value); }
        double *data() { return v.data(); }
        const double *data() const { return v.data(); }

        RRVector &operator*=(double s)
        {
            for (double &e : v) e *= s;
            return *this;
        }

        //! sqrt of the sum of squares, accumulated in index order.
        static double euclideanNorm(const RRVector &x)
        {
            double s = 0.0;
            for (double e : x.v) s += e * e;
            return std::sqrt(s);
        }

        //! Sum of products in index order.
        static double dot(const RRVector &x, const RRVector &y)
        {
            double s = 0.0;
            for (size_t i = 0; i < x.v.size(); i++) s += x.v[i] * y.v[i];
            return s;
        }

        //! Divides every element by the Euclidean norm (left as is when the norm is zero); returns the norm.
        double normalize()
        {
            const double nrm = euclideanNorm(*this);
            if (nrm != 0.0)
                for (double &e : v) e /= nrm;
            return nrm;
        }
};

class RRMatrix
{
    protected:
        std::vector<RRVector> rows;
        uint nColumns = 0;

    public:
        RRMatrix() = default;
        RRMatrix(uint nRows, uint nCols, double value = 0.0) { this->resize(nRows, nCols, value); }

        RRVector &operator[](uint i) { return rows[i]; }
        const RRVector &operator[](uint i) const { return rows[i]; }

        uint getNRows() const { return uint(rows.size()); }
        uint getNColumns() const { return nColumns; }

        void resize(uint nRows, uint nCols) { this->resize(nRows, nCols, 0.0); }
        void resize(uint nRows, uint nCols, double value)
        {
            rows.assign(nRows, RRVector(nCols, value));
            nColumns = nCols;
        }
        void fill(double value)
        {
            for (RRVector &r : rows) r.fill(value);
        }

        void transpose()
        {
            RRMatrix t(nColumns, uint(rows.size()), 0.0);
            for (uint i = 0; i < rows.size(); i++)
                for (uint j = 0; j < nColumns; j++) t[j][i] = rows[i][j];
            *this = t;
        }

        //! c = a b, each entry summed over the inner index in ascending order.
        static void mlt(const RRMatrix &a, const RRMatrix &b, RRMatrix &c)
        {
            RRMatrix r(a.getNRows(), b.getNColumns(), 0.0);
            for (uint i = 0; i < a.getNRows(); i++)
                for (uint j = 0; j < b.getNColumns(); j++) {
                    double s = 0.0;
                    for (uint k = 0; k < a.getNColumns(); k++) s += a[i][k] * b[k][j];
                    r[i][j] = s;
                }
            c = r;
        }

        void invert()
        {
            const uint w = nColumns;
            if (w != rows.size())
                throw RError(RError::Type::Application, R_ERROR_REF, "Matrix is not square.");
            RRMatrix inv(w, w, 0.0);
            for (uint i = 0; i < w; i++) inv[i][i] = 1.0;
            for (uint c = 0; c < w; c++) {
                uint piv = c;
                for (uint r = c + 1; r < w; r++)
                    if (std::abs(rows[r][c]) > std::abs(rows[piv][c])) piv = r;
                if (rows[piv][c] == 0.0)
                    throw RError(RError::Type::Application, R_ERROR_REF, "Matrix is singular.");
                if (piv != c) {
                    std::swap(rows[piv], rows[c]);
                    std::swap(inv.rows[piv], inv.rows[c]);
                }
                const double p = rows[c][c];
                for (uint k = 0; k < w; k++) {
                    rows[c][k] /= p;
                    inv[c][k] /= p;
                }
                for (uint r = 0; r < w; r++) {
                    if (r == c) continue;
                    const double f = rows[r][c];
                    if (f == 0.0) continue;
                    for (uint k = 0; k < w; k++) {
                        rows[r][k] -= f * rows[c][k];
                        inv[r][k] -= f * inv[c][k];
                    }
                }
            }
            *this = inv;
        }
};

#endif
