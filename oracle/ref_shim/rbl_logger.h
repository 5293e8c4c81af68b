// Stand-in for range-base-lib's RLogger (TEST INFRASTRUCTURE: lets the reference's own solver
// sources compile here).  Messages are formatted printf-style; the driver (ref_driver.cpp) picks the
// iteration reports out of them; nothing is printed unless REF_SHIM_ECHO is set.
#ifndef REF_SHIM_RBL_LOGGER_H
#define REF_SHIM_RBL_LOGGER_H

class RLogger
{
    public:
        static void info(const char *format, ...) __attribute__((format(printf, 1, 2)));
        static void warning(const char *format, ...) __attribute__((format(printf, 1, 2)));
        static void error(const char *format, ...) __attribute__((format(printf, 1, 2)));
        static void indent() {}
        static void unindent() {}
};

#endif
