// TEST INFRASTRUCTURE ONLY — stand-in for the reference's include/host/logger.hpp (which needs a
// formatting library that is not installed here) when oracle/build_ref_sppm.py compiles the
// reference's own host sources.  Log lines are dropped; LOG_FATAL and ASSERT, which end the
// reference program, throw instead, so that a C entry point can turn them into a status code.
#pragma once

#include <stdexcept>

#define LOG_INFO(...) ((void)0)
#define LOG_WARN(...) ((void)0)
#define LOG_ERROR(...) ((void)0)
#define LOG_DEBUG(...) ((void)0)
#define LOG_FATAL(...) throw std::runtime_error("reference LOG_FATAL")
#define ASSERT(cond, ...)                                                                                              \
    do {                                                                                                               \
        if (!(cond))                                                                                                   \
            throw std::runtime_error("reference ASSERT");                                                              \
    } while (0)
