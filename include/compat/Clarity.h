/*
 * Clarity.h -- the header name the reference's callers include
 * (`#include <Clarity.h>`, configured from the reference's Clarity.h.in).
 * Put this directory on the include path (-I<repo>/include/compat) and an
 * existing caller compiles unchanged against libclarity.so: the declarations
 * are this library's own (clarity.h: same names, signatures, result codes and
 * Clarity_Dim3 layout).
 */
#ifndef CLARITY_B200_COMPAT_CLARITY_H_
#define CLARITY_B200_COMPAT_CLARITY_H_
#include "../clarity.h"
#endif
