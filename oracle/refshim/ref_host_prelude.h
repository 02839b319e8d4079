// ref_host_prelude.h -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref), force-included before the reference's DPE.cpp.  The reference compiles DPE.cpp
// with the host compiler against the CUDA runtime headers, which include <math.h>; in C++ that
// header also makes the float overloads of the std math functions (exp(float), fabs(float),
// isnan ...) visible unqualified.  Including it here gives DPE.cpp the same overload set.
#ifndef REFSHIM_REF_HOST_PRELUDE_H_
#define REFSHIM_REF_HOST_PRELUDE_H_
#include <math.h>
#include <stdlib.h>
#endif
