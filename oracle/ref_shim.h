/* Force-included into every reference C++ translation unit compiled by
 * oracle/Makefile.  The reference's Commons.h defines its own
 * `inline bool isnan(double)` when no `isnan` macro exists, which collides
 * with glibc's declarations under a modern g++; defining the macro here makes
 * the reference take its `#ifndef isnan` branch and use the standard one.
 * Test infrastructure only: nothing in the product includes this file. */
#ifndef CFD_ORACLE_REF_SHIM_H
#define CFD_ORACLE_REF_SHIM_H
#ifdef __cplusplus
#include <cmath>
#define isnan(x) std::isnan(x)
#endif
#endif
