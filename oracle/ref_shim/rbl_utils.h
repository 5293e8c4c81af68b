// Stand-in for range-base-lib's rbl_utils.h (TEST INFRASTRUCTURE): the names the reference's
// solver sources take from it -- RConstants::eps, RError with R_ERROR_REF, RLogger and `uint`.
// RConstants::eps is not published with the reference; 1e-14 is the value this project's solver
// configuration uses by default for it.
#ifndef REF_SHIM_RBL_UTILS_H
#define REF_SHIM_RBL_UTILS_H

#include <cstdarg>
#include <cstdio>
#include <stdexcept>
#include <string>

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

    private:
        static std::string format(const char *file, int line, const char *function, const char *fmt)
        {
            char buf[512];
            std::snprintf(buf, sizeof(buf), "%s:%d (%s): %s", file, line, function, fmt);
            return buf;
        }
};

#endif
