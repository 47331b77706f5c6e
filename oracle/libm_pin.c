/*
 * Single-precision elementary functions pinned to the correctly rounded result.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference core calls std::exp, std::log,
 * std::log1p and std::pow on floats (src/core/core.cpp:187, 267, 312, 322,
 * 344, 355).  Their last bit depends on the C library of the build machine
 * (glibc's expf/logf are within about 0.5 ulp, not always correctly rounded).
 * oracle/Makefile links this file into the reference build with -Bsymbolic so
 * that those calls resolve here, which pins the oracle to one platform-
 * independent definition: evaluate in double precision (error below one
 * double ulp) and round once to float.  That equals the correctly rounded
 * float result except when the exact value lies within 2^-29 float-ulp of a
 * rounding midpoint.  The GPU plain path evaluates the same way.
 *
 * The build without this pin is kept as oracle/_ref/libvnlb_ref_glibc.so so
 * the size of the platform effect can be measured.
 */
#include <math.h>

float expf(float x) { return (float)exp((double)x); }
float logf(float x) { return (float)log((double)x); }
float log1pf(float x) { return (float)log1p((double)x); }
float powf(float x, float y) { return (float)pow((double)x, (double)y); }
