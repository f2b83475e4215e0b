/* Forced-include prelude for compiling the reference's singlestep/Direct/
 * direct.cpp (+ DirectCPUKernels.cc, direct.h) outside its build system.
 * TEST INFRASTRUCTURE ONLY.  It supplies the two type names that abacus'
 * config.h / header.cpp normally provide in a float build (FLOAT, FLOAT3 as
 * include/threevector.hh's float3); nothing of the reference is changed. */
#ifndef NF_REF_PRELUDE_H
#define NF_REF_PRELUDE_H
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include "threevector.hh"
#define FLOAT float
#define FLOAT3 float3
#endif
