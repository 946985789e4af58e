// Hand-written configuration for compiling reference sources as a checker
// (TEST INFRASTRUCTURE ONLY): Eigen on, no MPI, no TBB, no asserts, the
// same macros configuration.h.in defines for that choice.
#pragma once
#define ZEPHYR_EIGEN
#include <iostream>
#include <stdexcept>
#define PYTHONHOME L""
#define if_mpi(...)
#define mpi_cond(expr1, expr2) expr2
#define z_assert(...)
#define if_debug(...) if constexpr (false)
#define debug_code if constexpr (false)
