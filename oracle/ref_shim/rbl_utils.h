// Stand-in for range-base-lib's rbl_utils.h (TEST INFRASTRUCTURE): the names the reference's
// solver sources take from it -- RConstants::eps, RError with R_ERROR_REF / R_ERROR_ASSERT, RLogger,
// RUtil::qSort and `uint`.
// RConstants::eps is not published with the reference; 1e-14 is the value this project's solver
// configuration uses by default for it.
#ifndef REF_SHIM_RBL_UTILS_H
#define REF_SHIM_RBL_UTILS_H

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "rbl_logger.h"

typedef unsigned int uint;

namespace RConstants
{
    constexpr double eps = 1.0e-14;
    constexpr unsigned int eod = 0xffffffffu;
}

#define R_ERROR_REF __FILE__, __LINE__, __func__

class RError : public std::runtime_error
{
    public:
        enum class Type { None = 0, Application, InvalidInput, InvalidOutput, Unknown };

        RError(Type, const char *file, int line, const char *function, const char *format, ...)
            : std::runtime_error(RError::format(file, line, function, format))
        {
        }

        //! The message, as an object with toUtf8().constData() (the reference formats it into a new RError).
        struct Message {
            std::string s;
            const Message &toUtf8() const { return *this; }
            const char *constData() const { return s.c_str(); }
        };
        Message getMessage() const { return Message{what()}; }

    private:
        static std::string format(const char *file, int line, const char *function, const char *fmt)
        {
            char buf[512];
            std::snprintf(buf, sizeof(buf), "%s:%d (%s): %s", file, line, function, fmt);
            return buf;
        }
};

// |a| with the sign of b (the sign-transfer macro of range-base-lib).
#define R_SAME_SIGN(a, b) ((b) >= 0.0 ? std::fabs(a) : -std::fabs(a))

#define R_ERROR_ASSERT(_condition)                                                              \
    {                                                                                           \
        if (!(_condition))                                                                      \
            throw RError(RError::Type::Application, R_ERROR_REF, "Assertion failed: " #_condition); \
    }

// RUtil::qSort (used by REigenValueSolver::solve): not published with the reference; this stand-in
// sorts ascending, stably, and returns in `indexes` the original position of each sorted value.
namespace RUtil
{
    template <typename V>
    void qSort(V &values, std::vector<uint> &indexes)
    {
        const uint n = uint(values.size());
        indexes.resize(n);
        std::iota(indexes.begin(), indexes.end(), 0u);
        std::stable_sort(indexes.begin(), indexes.end(), [&](uint a, uint b) { return values[a] < values[b]; });
        std::vector<double> sorted(n);
        for (uint i = 0; i < n; i++) sorted[i] = values[indexes[i]];
        for (uint i = 0; i < n; i++) values[i] = sorted[i];
    }
}

#endif
