/*
 * Forced-include shim for compiling the reference solver without an OpenACC
 * compiler (test infrastructure only).  The pragmas are ignored (no
 * -fopenacc), so every `#pragma acc kernels` region runs serially on the
 * host in FP64.  The two device-selection calls in Solver::initialize
 * (src/solver.h:560-562) are replaced: without them `rank % 0` would raise
 * SIGFPE on a machine with no OpenACC device.
 */
#pragma once
#include <openacc.h>
#define acc_get_num_devices(t) 1
#define acc_set_device_num(n, t) ((void)0)
