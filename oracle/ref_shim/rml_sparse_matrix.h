// Stand-ins for range-model-lib's RSparseVector and RSparseMatrix (TEST INFRASTRUCTURE): one
// sparse row per matrix row, (column index, value) pairs in ascending column order, filled from
// a CSR matrix by the driver.  findColumnPosition is a binary search over the row's columns.
#ifndef REF_SHIM_RML_SPARSE_MATRIX_H
#define REF_SHIM_RML_SPARSE_MATRIX_H

#include <vector>

#include "rbl_rmatrix.h"
#include "rbl_utils.h"

template <typename T>
class RSparseVector
{
    protected:
        std::vector<uint> indexes;
        std::vector<T> values;

    public:
        uint size() const { return uint(indexes.size()); }
        uint getIndex(uint position) const { return indexes[position]; }
        const T &getValue(uint position) const { return values[position]; }
        void assign(const uint *idx, const T *val, uint n)
        {
            indexes.assign(idx, idx + n);
            values.assign(val, val + n);
        }
        void setValue(uint position, const T &value) { values[position] = value; }
        void insert(uint index, const T &value)
        {
            uint p = 0;
            while (p < indexes.size() && indexes[p] < index) p++;
            indexes.insert(indexes.begin() + p, index);
            values.insert(values.begin() + p, value);
        }
};

class RSparseMatrix
{
    protected:
        std::vector<RSparseVector<double>> rows;

    public:
        RSparseMatrix() = default;
        explicit RSparseMatrix(uint nRows) : rows(nRows) {}

        uint getNRows() const { return uint(rows.size()); }
        const RSparseVector<double> &getVector(uint row) const { return rows[row]; }
        RSparseVector<double> &getVector(uint row) { return rows[row]; }

        bool findColumnPosition(uint row, uint column, uint &position) const
        {
            const RSparseVector<double> &r = rows[row];
            uint lo = 0, hi = r.size();
            while (lo < hi) {
                const uint mid = lo + (hi - lo) / 2;
                if (r.getIndex(mid) < column) lo = mid + 1;
                else hi = mid;
            }
            if (lo < r.size() && r.getIndex(lo) == column) {
                position = lo;
                return true;
            }
            return false;
        }
        double getValue(uint row, uint position) const { return rows[row].getValue(position); }

        std::vector<uint> getRowIndexes(uint row) const
        {
            std::vector<uint> out(rows[row].size());
            for (uint j = 0; j < out.size(); j++) out[j] = rows[row].getIndex(j);
            return out;
        }

        //! Adds value to entry (row, column), inserting it in column order when it is not stored.
        void addValue(uint row, uint column, double value)
        {
            uint position = 0;
            if (findColumnPosition(row, column, position)) {
                RSparseVector<double> &r = rows[row];
                r.setValue(position, r.getValue(position) + value);
            } else {
                rows[row].insert(column, value);
            }
        }

        //! y = A x, every row summed over its stored entries in column order.
        static void mlt(const RSparseMatrix &a, const RRVector &x, RRVector &y)
        {
            y.resize(a.getNRows());
            for (uint i = 0; i < a.getNRows(); i++) {
                const RSparseVector<double> &r = a.rows[i];
                double s = 0.0;
                for (uint j = 0; j < r.size(); j++) s += r.getValue(j) * x[r.getIndex(j)];
                y[i] = s;
            }
        }
};

#endif
