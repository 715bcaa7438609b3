/* Clarity.h -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Stands in for the header CMake would configure from the reference's
 * Clarity.h.in when building the reference CPU sources for the oracle:
 * OpenMP on, CUDA off, no timers (CMakeLists.txt:8-16).  The declarations
 * come from this project's own ABI header, which carries the same names,
 * types and enum values. */
#ifndef CLARITY_ORACLE_CONFIG_H_
#define CLARITY_ORACLE_CONFIG_H_
#define BUILD_WITH_OPENMP
#ifdef __cplusplus
#define C_FUNC_DEF extern "C"
#else
#define C_FUNC_DEF
#endif
#ifndef NULL
#define NULL 0L
#endif
#include "../../include/clarity.h"
#endif
